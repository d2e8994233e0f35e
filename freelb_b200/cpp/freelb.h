// freelb.h -- C++17 host classes with the reference FreeLB names, backed by the
// B200 C ABI (include/flb.h, libflb_b200.so).
//
// A FreeLB program written against the reference's cavity interface
// (benchmarks/cavity3d/cavity3d.cpp, examples/cavity3d/cavity3d.cpp) compiles
// against this header by changing only its include path: the geometry, flag
// field, unit converter, task selector and lattice manager types keep their
// reference names and signatures, while every lattice operation runs on the
// GPU through the C ABI.  Policy types (collision::BGK, ...) are compile-time
// tags mapped to the ABI's op codes; a policy without a device op fails to
// compile (there is no CPU fallback).
//
// Device mapping of the reference calls:
//   BlockLatticeManager ctor            -> flb_create (single device block)
//   ApplyCellDynamics<NSTask>(FlagFM)   -> flb_set_tasks; the collision is
//                                          fused into the following Stream()
//   Stream()                            -> flb_step(1)
//   ApplyCellDynamics<rhoU<CELL,true>>  -> flb_compute_rhou (RHO, VELOCITY)
//   getToleranceU                       -> flb_tolerance_u
//   field forEach / SetField            -> host mirrors uploaded before the next
//                                          device call; reads download first.
// The block count passed to BlockGeometry3D is recorded but the domain is one
// device block: on one GPU the reference's block split (there for OpenMP / MPI
// work sharing) brings no benefit, and fluid-cell results are identical
// (multi-block equivalence is tested on the C ABI).
#pragma once

#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/flb.h"

#ifdef _OPENMP
#include <omp.h>
#endif

// ---------------------------------------------------------------------------
// errors
namespace flbcpp {
inline void check(int rc, const char* what) {
  if (rc != FLB_OK)
    throw std::runtime_error(std::string(what) + ": " + flb_last_error());
}
}  // namespace flbcpp

// ---------------------------------------------------------------------------
// Vector (src/data_struct/Vector.h)
template <typename T, unsigned int D>
class Vector {
  std::array<T, D> v_{};

 public:
  Vector() = default;
  explicit Vector(T a) { v_.fill(a); }
  template <typename... A, typename = std::enable_if_t<sizeof...(A) == D && (D > 1)>>
  Vector(A... a) : v_{T(a)...} {}
  T& operator[](unsigned int i) { return v_[i]; }
  const T& operator[](unsigned int i) const { return v_[i]; }
  const T* data() const { return v_.data(); }
  Vector operator+(const Vector& o) const {
    Vector r;
    for (unsigned i = 0; i < D; ++i) r[i] = v_[i] + o[i];
    return r;
  }
  Vector operator-(const Vector& o) const {
    Vector r;
    for (unsigned i = 0; i < D; ++i) r[i] = v_[i] - o[i];
    return r;
  }
  Vector operator*(T s) const {
    Vector r;
    for (unsigned i = 0; i < D; ++i) r[i] = v_[i] * s;
    return r;
  }
  Vector operator/(T s) const {
    Vector r;
    for (unsigned i = 0; i < D; ++i) r[i] = v_[i] / s;
    return r;
  }
  T operator*(const Vector& o) const {  // dot product, as the reference's operator*
    T s{};
    for (unsigned i = 0; i < D; ++i) s += v_[i] * o[i];
    return s;
  }
  Vector& operator+=(const Vector& o) { return *this = *this + o; }
  void clear() { v_.fill(T{}); }
};

// ---------------------------------------------------------------------------
// utilities
namespace util {
template <typename F>
inline bool isFlag(F flag, F key) { return (flag & key) != F(0); }
}  // namespace util

struct Printer {
  static void Print_BigBanner(const std::string& s) {
    std::cout << "\n----------------" << s << "----------------\n" << std::endl;
  }
  static void Print_Banner(const std::string& s) { std::cout << "---" << s << "---" << std::endl; }
  template <typename T>
  static void Print(const std::string& s, T v) { std::cout << s << ": " << v << std::endl; }
  template <typename T>
  static void Print_Res(T r) { std::cout << "Res: " << r << " "; }
  static void Endl() { std::cout << std::endl; }
};

struct Counter {
  std::int64_t count = 0;
  void reset() { count = 0; }
  void operator++() { ++count; }
  std::int64_t operator()() const { return count; }
};

// Timer with the reference's MLUPs report (src/utils/timer.h:50-112).
struct Timer : public Counter {
  std::chrono::high_resolution_clock::time_point START, END;
  Timer() { START_TIMER(); }
  void START_TIMER() { START = std::chrono::high_resolution_clock::now(); }
  void END_TIMER() { END = std::chrono::high_resolution_clock::now(); }
  std::int64_t GetDurationCount() {
    END_TIMER();
    return std::chrono::duration_cast<std::chrono::milliseconds>(END - START).count();
  }
  double GetTimeElapsed() { return GetDurationCount() / 1000.0; }
  void Print_MainLoopPerformance(std::size_t n) {
    END_TIMER();
    const double ms = std::max<double>(
        1.0, double(std::chrono::duration_cast<std::chrono::milliseconds>(END - START).count()));
    std::cout << "[Main_Loop Performance]:\nTime Elapsed:  " << ms / 1000.0
              << " s\nTotal Step:    " << count
              << "\nAverage_MLUPs: " << double(count) * double(n) / ms / 1000.0 << std::endl;
  }
  void Print_InnerLoopPerformance(std::size_t n, std::size_t steps) {
    END_TIMER();
    const double ms = std::max<double>(
        1.0, double(std::chrono::duration_cast<std::chrono::milliseconds>(END - START).count()));
    std::cout << "[Step: " << count << "]  MLUPs: " << double(steps) * double(n) / ms / 1000.0
              << "  ";
    START_TIMER();
  }
};

// Minimal INI reader with the reference's getValue<T>(section, key)
// (src/io/ini_reader.h:54): `;` and `//` start comments.
class iniReader {
  std::map<std::string, std::map<std::string, std::string>> data_;
  static std::string trim(std::string s) {
    const auto a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return {};
    return s.substr(a, s.find_last_not_of(" \t\r\n") - a + 1);
  }

 public:
  explicit iniReader(const std::string& file) {
    std::ifstream in(file);
    if (!in) throw std::runtime_error("iniReader: cannot open " + file);
    std::string line, sec;
    while (std::getline(in, line)) {
      for (const char* c : {";", "//", "#"}) {
        const auto p = line.find(c);
        if (p != std::string::npos) line = line.substr(0, p);
      }
      line = trim(line);
      if (line.empty()) continue;
      if (line.front() == '[') {
        sec = trim(line.substr(1, line.find(']') - 1));
        continue;
      }
      const auto eq = line.find('=');
      if (eq == std::string::npos) continue;
      data_[sec][trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
  }
  template <typename T>
  T getValue(const std::string& sec, const std::string& key) const {
    const auto s = data_.find(sec);
    if (s == data_.end() || s->second.find(key) == s->second.end())
      throw std::runtime_error("iniReader: missing [" + sec + "] " + key);
    std::istringstream is(s->second.at(key));
    T v{};
    is >> v;
    return v;
  }
};

// MPI is out of scope: single-process stand-ins for the calls examples make.
struct MpiManagerStub {
  void init(int*, char***) {}
  int getRank() const { return 0; }
  int getSize() const { return 1; }
  void barrier() const {}
};
inline MpiManagerStub& mpi() {
  static MpiManagerStub m;
  return m;
}
#ifndef MPI_DEBUG_WAIT
#define MPI_DEBUG_WAIT
#endif

// ---------------------------------------------------------------------------
// lattice set (src/lbm/lattice_set.h:259-296)
template <typename T>
struct D3Q19 {
  using FloatType = T;
  static constexpr unsigned int d = 3;
  static constexpr unsigned int q = 19;
  static constexpr T cs2 = T(1) / T(3);
  static constexpr T InvCs2 = T(3);
  static constexpr T InvCs4 = T(9);
};

// unit conversion (src/lbm/unit_converter.h:120-235)
template <typename T>
struct AbstractConverter {
  virtual ~AbstractConverter() = default;
  virtual T getOMEGA() const = 0;
  virtual T getLatRhoInit() const = 0;
};

template <typename T>
struct BaseConverter final : public AbstractConverter<T> {
  T deltaX{}, deltaT{}, charL{}, charU{}, VisKine{}, rho{}, Re{};
  T Conv_L{}, Conv_Time{}, Conv_U{}, Conv_rho{}, Conv_VisKine{};
  T Lattice_charU{}, Lattice_charL{}, Lattice_VisKine{}, Lattice_Re{}, Lattice_RT{}, OMEGA{};
  T cs2;
  explicit BaseConverter(T cs2_) : cs2(cs2_) {}
  T getOMEGA() const override { return OMEGA; }
  T getLattice_RT() const { return Lattice_RT; }
  T getLatRhoInit() const override { return T(1); }
  T getLatticeU(T u) const { return u / Conv_U; }
  T getPhysU(T u) const { return u * Conv_U; }
  template <unsigned int D>
  Vector<T, D> getLatticeU(const Vector<T, D>& u) const { return u / Conv_U; }
  template <unsigned int D>
  Vector<T, D> getPhysU(const Vector<T, D>& u) const { return u * Conv_U; }
  T getPhysRho(T r) const { return r * Conv_rho; }
  T getPhysTime(T t) const { return t * deltaT; }
  void Converter(T dx, T dt, T rho_, T L, T U, T nu) {
    deltaX = dx;
    deltaT = dt;
    charL = L;
    charU = U;
    VisKine = nu;
    rho = rho_;
    Re = U * L / nu;
    Conv_L = dx;
    Conv_Time = dt;
    Conv_rho = rho_;
    Conv_U = Conv_L / Conv_Time;
    Conv_VisKine = Conv_L * Conv_L / Conv_Time;
    Lattice_charU = charU / Conv_U;
    Lattice_charL = charL / Conv_L;
    Lattice_VisKine = VisKine / Conv_VisKine;
    Lattice_Re = Lattice_charU / Lattice_VisKine;
    OMEGA = T(1) / Lattice_RT;
  }
  void ConvertFromRT(T dx, T RT, T rho_, T L, T U, T nu) {
    Lattice_RT = RT;
    Converter(dx, (RT - T(0.5)) * cs2 * dx * dx / nu, rho_, L, U, nu);
  }
  void SimplifiedConverterFromRT(int Ni, T U, T RT) {
    Lattice_RT = RT;
    Converter(T(1), T(1), T(1), T(Ni), U, (RT - T(0.5)) * cs2);
  }
};

template <typename T>
struct UnitConvManager {
  BaseConverter<T>* base;
  explicit UnitConvManager(BaseConverter<T>* b) : base(b) {}
  void Check_and_Print() const {
    std::cout << "[Unit conversion] tau = " << base->Lattice_RT << ", omega = " << base->OMEGA
              << ", lattice U = " << base->Lattice_charU << ", Re = " << base->Lattice_Re
              << std::endl;
  }
};

// ---------------------------------------------------------------------------
// geometry (src/geometry/basic_geometry.h, block_geometry3d.h)
template <typename T, unsigned int D>
class AABB {
  Vector<T, D> min_, max_;

 public:
  AABB() = default;
  AABB(const Vector<T, D>& a, const Vector<T, D>& b) : min_(a), max_(b) {}
  const Vector<T, D>& getMin() const { return min_; }
  const Vector<T, D>& getMax() const { return max_; }
  // basic_geometry.hh:39-48
  bool isInside(const Vector<T, D>& p) const {
    constexpr T eps = std::numeric_limits<T>::epsilon();
    for (unsigned i = 0; i < D; ++i)
      if (!(p[i] >= min_[i] - eps && p[i] <= max_[i] + eps)) return false;
    return true;
  }
};

// One device block covering the domain plus its one-cell overlap layer
// (block_geometry3d.hh:157-171); cell centres as the reference computes them.
template <typename T>
class BlockGeometry3D {
  int nx_, ny_, nz_;
  int blocknum_;
  T voxel_;
  Vector<T, 3> min_ext_;

 public:
  BlockGeometry3D(int Nx, int Ny, int Nz, int blocknum, const AABB<T, 3>& block, T voxelSize,
                  int overlap = 1)
      : nx_(Nx + 2 * overlap), ny_(Ny + 2 * overlap), nz_(Nz + 2 * overlap),
        blocknum_(blocknum), voxel_(voxelSize),
        min_ext_(block.getMin() - Vector<T, 3>(voxelSize * T(overlap))) {
    std::cout << "[BlockGeometry3D]:\n  Total CellNum: " << getTotalCellNum()
              << "\n  BlockNum: 1 (device block; requested " << blocknum << ")" << std::endl;
  }
  int getNx() const { return nx_; }
  int getNy() const { return ny_; }
  int getNz() const { return nz_; }
  std::size_t getTotalCellNum() const { return std::size_t(nx_) * ny_ * nz_; }
  std::size_t getN() const { return getTotalCellNum(); }
  int getBlockNum() const { return 1; }
  T getVoxelSize() const { return voxel_; }
  // MinCenter + VoxelSize * (i, j, k) (basic_geometry.h:245, 310-311)
  Vector<T, 3> getVoxel(int i, int j, int k) const {
    const T h = T(0.5) * voxel_;
    return Vector<T, 3>((min_ext_[0] + h) + voxel_ * T(i), (min_ext_[1] + h) + voxel_ * T(j),
                        (min_ext_[2] + h) + voxel_ * T(k));
  }
  std::size_t index(int i, int j, int k) const {
    return std::size_t(i) + std::size_t(nx_) * (std::size_t(j) + std::size_t(ny_) * k);
  }
  // visit the cells whose centre is inside `box` (basic_geometry.hh:484-505)
  template <typename F>
  void forEachInside(const AABB<T, 3>& box, F&& f) const {
    for (int k = 0; k < nz_; ++k)
      for (int j = 0; j < ny_; ++j)
        for (int i = 0; i < nx_; ++i)
          if (box.isInside(getVoxel(i, j, k))) f(index(i, j, k));
  }
};

// ---------------------------------------------------------------------------
// field types and packs (src/utils/alias.h).  A field is the host array the
// reference's forEach lambdas receive (GenericField<GenericArray<V>, Tag>);
// the tag keeps RHO, SMAGORINSKY and POP distinct as in the reference.
template <typename V, typename Tag>
class HostField {
 public:
  using value_type = V;
  std::vector<V> data;
  bool dirty = false;  // host newer than device
  explicit HostField(std::size_t n = 0, V init = V{}) : data(n, init) {}
  void SetField(std::size_t id, const V& v) {
    data[id] = v;
    dirty = true;
  }
  const V& get(std::size_t id) const { return data[id]; }
  V& get(std::size_t id) { return data[id]; }
  const V& operator[](std::size_t id) const { return data[id]; }
  HostField& getField(int = 0) { return *this; }
  const HostField& getField(int = 0) const { return *this; }
};
struct FLAGBase {};
struct RHOBase {};
struct VELOCITYBase {};
struct SMAGORINSKYBase {};
template <unsigned int Q>
struct POPBase {};
using FLAG = HostField<std::uint8_t, FLAGBase>;
template <typename T>
using RHO = HostField<T, RHOBase>;
template <typename T, unsigned int D>
using VELOCITY = HostField<Vector<T, D>, VELOCITYBase>;
template <typename T, unsigned int Q>
using POP = HostField<T, POPBase<Q>>;
template <typename T>
using SMAGORINSKY = HostField<T, SMAGORINSKYBase>;
template <typename... F>
struct TypePack {};
template <typename... V>
struct ValuePack {
  std::tuple<V...> values;
  explicit ValuePack(V... v) : values(v...) {}
};
template <typename T, typename LatSet, typename FIELDS>
struct Cell {
  using FloatType = T;
  using LatticeSet = LatSet;
};

// BlockFieldManager<FLAG, T, 3> (src/data_struct/field_struct.h:39-335)
template <typename FieldType, typename T, unsigned int Dim>
class BlockFieldManager {
 public:
  using field_t = FieldType;
  BlockFieldManager(const BlockGeometry3D<T>& geo, typename FieldType::value_type init)
      : geo_(geo), field_(geo.getTotalCellNum(), init) {
    field_.dirty = true;
  }
  // forEach(AABB, func(field, id)): cells whose centre is inside
  template <typename F>
  void forEach(const AABB<T, Dim>& box, F&& f) {
    geo_.forEachInside(box, [&](std::size_t id) { f(field_, id); });
  }
  template <typename F>
  void forEach(F&& f) {
    for (std::size_t id = 0; id < field_.data.size(); ++id) f(field_, id);
  }
  // forEach(AABB, FlagFM, flag, func): inside the box and flag matching
  // (basic_geometry.hh:507-533)
  template <typename FlagManager, typename F>
  void forEach(const AABB<T, Dim>& box, const FlagManager& flags, std::uint8_t flag, F&& f) {
    const auto& fl = flags.field();
    geo_.forEachInside(box, [&](std::size_t id) {
      if (util::isFlag(fl.get(id), flag)) f(field_, id);
    });
  }
  // Block3D::SetupBoundary (block_geometry3d.hh:78-104): interior cells with
  // any D3Q19 neighbour centre outside `box` get `bdvalue`.
  template <typename LatSet>
  void SetupBoundary(const AABB<T, Dim>& box, typename FieldType::value_type bdvalue) {
    static const int C[19][3] = {{0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},
                                 {0, 0, 1},  {0, 0, -1},  {1, 1, 0},  {-1, -1, 0}, {1, 0, 1},
                                 {-1, 0, -1}, {0, 1, 1},  {0, -1, -1}, {1, -1, 0}, {-1, 1, 0},
                                 {1, 0, -1}, {-1, 0, 1},  {0, 1, -1}, {0, -1, 1}};
    std::vector<std::size_t> mark;
    for (int k = 1; k < geo_.getNz() - 1; ++k)
      for (int j = 1; j < geo_.getNy() - 1; ++j)
        for (int i = 1; i < geo_.getNx() - 1; ++i) {
          const Vector<T, 3> v = geo_.getVoxel(i, j, k);
          for (int q = 1; q < 19; ++q) {
            const T s = geo_.getVoxelSize();
            const Vector<T, 3> n(v[0] + T(C[q][0]) * s, v[1] + T(C[q][1]) * s,
                                 v[2] + T(C[q][2]) * s);
            if (!box.isInside(n)) {
              mark.push_back(geo_.index(i, j, k));
              break;
            }
          }
        }
    for (std::size_t id : mark) field_.SetField(id, bdvalue);
  }
  field_t& getBlockField(int) { return field_; }
  const field_t& getBlockField(int) const { return field_; }
  field_t& field() { return field_; }
  const field_t& field() const { return field_; }
  const BlockGeometry3D<T>& geo() const { return geo_; }
  void copyToDevice() { field_.dirty = true; }

 private:
  const BlockGeometry3D<T>& geo_;
  field_t field_;
};

// ---------------------------------------------------------------------------
// policies (src/lbm/collision.h, collisionMRT.h, collisionLES.h, moment.h,
// equilibrium.h) as compile-time tags with their device op
namespace equilibrium {
template <typename CELL>
struct SecondOrder {};
}  // namespace equilibrium
namespace moment {
template <typename CELL, bool WriteToField = false>
struct rhoU {
  static constexpr bool flb_is_moment = WriteToField;
};
template <typename CELL>
struct useFieldrhoU {};
}  // namespace moment
namespace collision {
template <typename M, typename E>
struct BGK {};
template <typename CELL>
struct BounceBack {};
template <typename CELL>
struct BounceBackMovingWall {};
template <typename CELL, bool WriteToField = false>
struct MRT_Feq_RhoU {};
template <typename M, typename E, bool WriteToField = false>
struct SmagorinskyBGK {};
}  // namespace collision

namespace flbcpp {
// op / model of a policy; kind: 0 collision, 1 moment task
template <typename P>
struct PolicyOp {
  static_assert(sizeof(P) == 0, "policy without a device op (no CPU fallback)");
};
template <typename C, bool W>
struct PolicyOp<moment::rhoU<C, W>> {
  static constexpr int op = FLB_OP_NONE, model = -1, kind = 1;
};
template <typename C, typename E>
struct PolicyOp<collision::BGK<moment::rhoU<C>, E>> {
  static constexpr int op = FLB_OP_BULK, model = FLB_MODEL_BGK, kind = 0;
};
template <typename C, typename E>
struct PolicyOp<collision::BGK<moment::rhoU<C, true>, E>> {
  static constexpr int op = FLB_OP_BULK, model = FLB_MODEL_BGK, kind = 0;
};
template <typename C, typename E>
struct PolicyOp<collision::BGK<moment::useFieldrhoU<C>, E>> {
  static constexpr int op = FLB_OP_FIELD_BGK, model = -1, kind = 0;
};
template <typename C>
struct PolicyOp<collision::BounceBack<C>> {
  static constexpr int op = FLB_OP_BOUNCEBACK, model = -1, kind = 0;
};
template <typename C>
struct PolicyOp<collision::BounceBackMovingWall<C>> {
  static constexpr int op = FLB_OP_MOVINGWALL, model = -1, kind = 0;
};
template <typename C, bool W>
struct PolicyOp<collision::MRT_Feq_RhoU<C, W>> {
  static constexpr int op = FLB_OP_BULK, model = FLB_MODEL_MRT, kind = 0;
};
template <typename M, typename E, bool W>
struct PolicyOp<collision::SmagorinskyBGK<M, E, W>> {
  static constexpr int op = FLB_OP_BULK, model = FLB_MODEL_LES, kind = 0;
};
}  // namespace flbcpp

// task selection (src/utils/tmp.h:194-309)
namespace tmp {
template <auto Key, typename Policy>
struct Key_TypePair {
  static constexpr auto key = Key;
  using type = Policy;
};
template <typename... Pairs>
struct TupleWrapper {};
template <typename TUPLE, typename FlagType, typename CELL>
struct TaskSelector;
template <typename... Pairs, typename FlagType, typename CELL>
struct TaskSelector<TupleWrapper<Pairs...>, FlagType, CELL> {
  using pairs = std::tuple<Pairs...>;
};
}  // namespace tmp
template <typename FlagType, typename CELL, typename... Pairs>
struct TaskSelector {
  using pairs = std::tuple<Pairs...>;
};

namespace flbcpp {
struct TaskList {
  int n = 0, model = -1, kind = 0;
  std::uint8_t keys[FLB_MAX_TASKS]{}, ops[FLB_MAX_TASKS]{};
};
template <typename Tuple, std::size_t... I>
TaskList task_list_impl(std::index_sequence<I...>) {
  TaskList t;
  static_assert(sizeof...(I) <= FLB_MAX_TASKS, "too many tasks");
  (([&] {
     using P = std::tuple_element_t<I, Tuple>;
     using Op = PolicyOp<typename P::type>;
     t.keys[t.n] = std::uint8_t(P::key);
     t.ops[t.n] = std::uint8_t(Op::op);
     if (Op::model >= 0) t.model = Op::model;
     if (Op::kind == 1) t.kind = 1;
     ++t.n;
   }()),
   ...);
  return t;
}
template <typename Selector>
TaskList task_list() {
  using Tuple = typename Selector::pairs;
  return task_list_impl<Tuple>(std::make_index_sequence<std::tuple_size<Tuple>::value>{});
}
}  // namespace flbcpp

// ---------------------------------------------------------------------------
// BlockLatticeManager (src/data_struct/block_lattice.h:234-433), one device block
template <typename T, typename LatSet, typename FIELDS>
class BlockLatticeManager {
  static_assert(std::is_same<LatSet, D3Q19<T>>::value, "the device path is D3Q19");
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value,
                "FP32 or FP64 populations");

 public:
  using FloatType = T;
  using VelField = BlockFieldManager<VELOCITY<T, 3>, T, 3>;
  using RhoField = BlockFieldManager<RHO<T>, T, 3>;

  template <typename INIT>
  BlockLatticeManager(BlockGeometry3D<T>& geo, INIT& init, AbstractConverter<T>& conv)
      : geo_(geo), vel_(geo, Vector<T, 3>{}), rho_(geo, conv.getLatRhoInit()) {
    flb_lattice_desc d;
    flbcpp::check(flb_desc_default(&d, geo.getNx(), geo.getNy(), geo.getNz(),
                                   1.0 / double(conv.getOMEGA())),
                  "flb_desc_default");
    d.omega = double(conv.getOMEGA());
    d.storage = std::is_same<T, double>::value ? FLB_STORAGE_FP64 : FLB_STORAGE_FP32;
    d.rho0 = double(conv.getLatRhoInit());
    d.ntasks = 0;
    init_smagorinsky(d, init);
    flbcpp::check(flb_create(&d, &h_), "flb_create");
  }
  ~BlockLatticeManager() { flb_destroy(h_); }
  BlockLatticeManager(const BlockLatticeManager&) = delete;
  BlockLatticeManager& operator=(const BlockLatticeManager&) = delete;

  template <typename F>
  auto& getField() {
    if constexpr (std::is_same<F, VELOCITY<T, 3>>::value) {
      pull_fields();
      return vel_;
    } else if constexpr (std::is_same<F, RHO<T>>::value) {
      pull_fields();
      return rho_;
    } else {
      static_assert(sizeof(F) == 0, "field not mirrored on the host");
    }
  }

  // ApplyCellDynamics<TaskSelector>(FlagFM) (block_lattice.hh:766-778)
  template <typename Selector, typename FlagManager>
  void ApplyCellDynamics(FlagManager& flags) {
    push(flags);
    const flbcpp::TaskList t = flbcpp::task_list<Selector>();
    if (t.kind == 1) {  // moment::rhoU<CELL,true> as a task: device RHO/VELOCITY
      std::uint8_t key = 0;
      for (int i = 0; i < t.n; ++i) key |= t.keys[i];
      flbcpp::check(flb_compute_rhou(h_, key, nullptr), "flb_compute_rhou");
      fields_stale_ = true;
      return;
    }
    if (pending_) throw std::logic_error("ApplyCellDynamics twice without Stream()");
    const int model = t.model >= 0 ? t.model : FLB_MODEL_BGK;
    flbcpp::check(flb_set_tasks(h_, t.n, t.keys, t.ops, model), "flb_set_tasks");
    pending_ = true;
  }
  template <typename Selector, typename FlagManager>
  void CuDevApplyCellDynamics(FlagManager& flags) { ApplyCellDynamics<Selector>(flags); }

  // Stream() (block_lattice.hh:744-747): runs the fused collide + stream.
  void Stream() {
    if (!pending_) {  // streaming alone: no task matches any flag
      flbcpp::check(flb_set_tasks(h_, 0, nullptr, nullptr, FLB_MODEL_BGK), "flb_set_tasks");
    }
    flbcpp::check(flb_step(h_, 1, nullptr), "flb_step");
    pending_ = false;
    fields_stale_ = true;
  }
  void CuDevStream() { Stream(); }
  // one device block: the halo exchange between blocks has nothing to do
  void NormalCommunicate() {}
  void Communicate() {}

  void EnableToleranceU() { tolerance_on_ = true; }
  T getToleranceU(int = -1) {
    double v = 0;
    flbcpp::check(flb_tolerance_u(h_, 2, &v, nullptr), "flb_tolerance_u");
    return T(v);
  }
  flb_lattice* handle() { return h_; }

 private:
  template <typename INIT>
  void init_smagorinsky(flb_lattice_desc& d, const INIT& init) {
    constexpr std::size_t n = std::tuple_size<decltype(init.values)>::value;
    if constexpr (n >= 4) d.smagorinsky = double(std::get<3>(init.values));
  }
  template <typename FlagManager>
  void push(FlagManager& flags) {
    auto& f = flags.field();
    if (f.dirty) {
      flbcpp::check(flb_upload_flags(h_, f.data.data(), nullptr), "flb_upload_flags");
      f.dirty = false;
    }
    if (vel_.field().dirty) {
      std::vector<T> buf(3 * vel_.field().data.size());
      for (std::size_t i = 0; i < vel_.field().data.size(); ++i)
        for (int c = 0; c < 3; ++c) buf[3 * i + c] = vel_.field().data[i][c];
      flbcpp::check(flb_upload_field(h_, FLB_FIELD_VELOCITY, buf.data(), dtype(), nullptr),
                    "upload VELOCITY");
      vel_.field().dirty = false;
    }
    if (rho_.field().dirty) {
      flbcpp::check(flb_upload_field(h_, FLB_FIELD_RHO, rho_.field().data.data(), dtype(),
                                     nullptr),
                    "upload RHO");
      rho_.field().dirty = false;
    }
  }
  void pull_fields() {
    if (!fields_stale_) return;
    std::vector<T> buf(3 * vel_.field().data.size());
    flbcpp::check(flb_download_field(h_, FLB_FIELD_VELOCITY, buf.data(), dtype(), nullptr),
                  "download VELOCITY");
    for (std::size_t i = 0; i < vel_.field().data.size(); ++i)
      for (int c = 0; c < 3; ++c) vel_.field().data[i][c] = buf[3 * i + c];
    flbcpp::check(flb_download_field(h_, FLB_FIELD_RHO, rho_.field().data.data(), dtype(),
                                     nullptr),
                  "download RHO");
    fields_stale_ = false;
  }
  static constexpr int dtype() {
    return std::is_same<T, double>::value ? FLB_DTYPE_F64 : FLB_DTYPE_F32;
  }

  BlockGeometry3D<T>& geo_;
  VelField vel_;
  RhoField rho_;
  flb_lattice* h_ = nullptr;
  bool pending_ = false;
  bool fields_stale_ = false;
  bool tolerance_on_ = false;
};

// ---------------------------------------------------------------------------
// post-stream boundary managers (src/boundary/boundary.h:34-222) are the
// halfway bounce-back of the reference; the cavity programs construct them but
// run their wall physics through the BounceBack / BounceBackMovingWall tasks.
namespace bounceback {
template <typename CELL>
struct normal {};
template <typename CELL>
struct movingwall {};
}  // namespace bounceback

template <typename BBType, typename LatticeManager, typename FlagManager>
class BBLikeFixedBlockBdManager {
 public:
  BBLikeFixedBlockBdManager(std::string name, LatticeManager&, FlagManager&, std::uint8_t,
                            std::uint8_t)
      : name_(std::move(name)) {}
  void Apply() {
    throw std::logic_error(name_ + ": post-stream bounce-back managers are not built on the "
                                   "device; use the BounceBack / BounceBackMovingWall tasks");
  }

 private:
  std::string name_;
};

class BlockBoundaryManager {
 public:
  template <typename... B>
  explicit BlockBoundaryManager(B*...) {}
  void Apply() {
    throw std::logic_error("post-stream bounce-back managers are not built on the device");
  }
};
