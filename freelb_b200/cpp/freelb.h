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

#include <sys/stat.h>

#include <array>
#include <functional>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
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
#include "../../include/flb_boundary.h"
#include "../../include/flb_vtk.h"

#ifdef _OPENMP
#include <omp.h>
#endif

// The reference's build-time float type (src/head.h:43-48: -DFLOAT_TYPE=...,
// double by default).
#ifdef FLOAT_TYPE
using FLOAT = FLOAT_TYPE;
#else
using FLOAT = double;
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
// the rank guards of src/parallel/mpi_manager.h:80-81 without MPI_ENABLED
#ifndef MPI_RANK
#define MPI_RANK(x)
#define IF_MPI_RANK(x)
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
  int overlap_;

 public:
  BlockGeometry3D(int Nx, int Ny, int Nz, int blocknum, const AABB<T, 3>& block, T voxelSize,
                  int overlap = 1)
      : nx_(Nx + 2 * overlap), ny_(Ny + 2 * overlap), nz_(Nz + 2 * overlap),
        blocknum_(blocknum), voxel_(voxelSize),
        min_ext_(block.getMin() - Vector<T, 3>(voxelSize * T(overlap))), overlap_(overlap) {
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
  int getOverlap() const { return overlap_; }
  Vector<int, 3> getMesh() const { return Vector<int, 3>(nx_, ny_, nz_); }
  // centre of the first stored cell (basic_geometry.hh:298: _min + VoxelSize / 2)
  Vector<T, 3> getMinCenter() const { return min_ext_ + Vector<T, 3>(T(0.5) * voxel_); }
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
// The reference's device field packs and cells (benchmarks/cavity3d_cu/
// cavity3d.cu:158-162): on this path every lattice field already lives on the
// device, so the device pack is the field pack and the device cell the cell tag.
template <typename FIELDS>
struct ExtractCudevFieldPack {
  using cudev_pack = FIELDS;
};
namespace cudev {
template <typename T, typename LatSet, typename FIELDS>
using Cell = ::Cell<T, LatSet, FIELDS>;
}  // namespace cudev

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
  // For the RHO and VELOCITY managers of a BlockLatticeManager: the device
  // copy the VTK writers encode from, and the call that uploads host edits
  // to it first.
  struct DeviceView {
    flb_lattice* lat = nullptr;
    int field = -1;
    std::function<void()> sync;
  };
  DeviceView device;

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
    rho0_ = d.rho0;
    d.ntasks = 0;
    init_smagorinsky(d, init);
    flbcpp::check(flb_create(&d, &h_), "flb_create");
    vel_.device = {h_, FLB_FIELD_VELOCITY, [this] { push_fields(); }};
    rho_.device = {h_, FLB_FIELD_RHO, [this] { push_fields(); }};
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
    } else if constexpr (std::is_same<F, POP<T, 19>>::value) {
      return pops_;
    } else {
      static_assert(sizeof(F) == 0, "field not mirrored on the host");
    }
  }
  // getField<POP<T, 19>>(): the populations live only on the device (created
  // at their equilibrium by the constructor), so copyToDevice() has nothing to
  // send; read them through flb_download_pops(handle(), ...).
  struct DevicePopulations {
    void copyToDevice() {}
  };

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
    // periodic managers whose Apply() came between ApplyCellDynamics and this
    // Stream(): their copies act on the post-collision populations, which the
    // fused step has just produced
    for (flb_periodic* per : periodic_)
      flbcpp::check(flb_periodic_apply(per, h_, nullptr), "flb_periodic_apply");
    periodic_.clear();
    pending_ = false;
    fields_stale_ = true;
  }
  // FixedPeriodicBoundaryManager::Apply(): runs after the next collision
  void arm_periodic(flb_periodic* per) { periodic_.push_back(per); }
  const BlockGeometry3D<T>& getGeo() const { return geo_; }
  void CuDevStream() { Stream(); }
  // one device block: the halo exchange between blocks has nothing to do
  void NormalCommunicate() {}
  void NormalCommunicate(std::int64_t) {}
  void NormalFullCommunicate() {}
  void NormalFullCommunicate(std::int64_t) {}
  void NormalAllCommunicate() {}
  void NormalAllCommunicate(std::int64_t) {}
  void Communicate() {}

  void EnableToleranceU() { tolerance_on_ = true; }
  T getToleranceU(int = -1) {
    double v = 0;
    flbcpp::check(flb_tolerance_u(h_, 2, &v, nullptr), "flb_tolerance_u");
    return T(v);
  }
  flb_lattice* handle() { return h_; }
  // Bring the device copies of the flags and fields up to date (what the
  // next ApplyCellDynamics would do); used by the boundary managers.
  template <typename FlagManager>
  void sync(FlagManager& flags) { push(flags); }
  double rho0() const { return rho0_; }

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
    push_fields();
  }
  void push_fields() {
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
  double rho0_ = 1.0;
  bool pending_ = false;
  bool fields_stale_ = false;
  bool tolerance_on_ = false;
  std::vector<flb_periodic*> periodic_;
  DevicePopulations pops_;
};

// ---------------------------------------------------------------------------
// post-stream boundary managers (src/boundary/boundary.h:34-222): halfway
// bounce-back after Stream() on the device (flb_boundary.h).  The policy tags
// carry the device kind of bounce_back_boundary.h:167-256.
namespace bounceback {
template <typename CELL>
struct normal { static constexpr int kind = FLB_BB_NORMAL; };
template <typename CELL>
struct movingwall { static constexpr int kind = FLB_BB_MOVINGWALL; };
template <typename CELL>
struct anti_simple { static constexpr int kind = FLB_BB_ANTI_SIMPLE; };
template <typename CELL>
struct anti_O1 { static constexpr int kind = FLB_BB_ANTI_O1; };
template <typename CELL>
struct anti_O2 { static constexpr int kind = FLB_BB_ANTI_O2; };
template <typename CELL>
struct anti_pressure { static constexpr int kind = FLB_BB_ANTI_PRESSURE; };
}  // namespace bounceback

class AbstractBlockBoundary {
 public:
  virtual ~AbstractBlockBoundary() = default;
  virtual void Apply() = 0;
  virtual void Apply(std::int64_t) { Apply(); }
};

// BBLikeFixedBlockBdManager (boundary.h:86-140): the boundary cells and their
// outflow directions are found from the flags at construction, like
// BlockFixedBoundary::Setup; Apply() runs after Stream().
template <typename BBType, typename LatticeManager, typename FlagManager>
class BBLikeFixedBlockBdManager final : public AbstractBlockBoundary {
 public:
  BBLikeFixedBlockBdManager(std::string name, LatticeManager& lat, FlagManager& flags,
                            std::uint8_t cellflag, std::uint8_t voidflag = std::uint8_t(1))
      : name_(std::move(name)), lat_(lat) {
    lat.sync(flags);
    flbcpp::check(flb_bb_create(lat.handle(), cellflag, voidflag, BBType::kind, lat.rho0(), &h_),
                  "flb_bb_create");
  }
  ~BBLikeFixedBlockBdManager() override { flb_bb_destroy(h_); }
  BBLikeFixedBlockBdManager(const BBLikeFixedBlockBdManager&) = delete;
  BBLikeFixedBlockBdManager& operator=(const BBLikeFixedBlockBdManager&) = delete;

  void Apply() override {
    flbcpp::check(flb_bb_apply(h_, lat_.handle(), nullptr), "flb_bb_apply");
  }
  void Apply(std::int64_t) override { Apply(); }  // one refinement level
  void getinfo() const {
    long long cells = 0;
    flb_bb_count(h_, &cells, nullptr);
    std::cout << std::setw(18) << std::left << name_ << std::setw(10) << std::left << cells
              << std::endl;
  }

 private:
  std::string name_;
  LatticeManager& lat_;
  flb_bb* h_ = nullptr;
};

// NbrDirection (parallel/communicator.h:37-52)
enum NbrDirection : std::uint8_t {
  NONE = 0,
  XN = FLB_NBR_XN,
  XP = FLB_NBR_XP,
  YN = FLB_NBR_YN,
  YP = FLB_NBR_YP,
  ZN = FLB_NBR_ZN,
  ZP = FLB_NBR_ZP
};

// FixedPeriodicBoundaryManager (boundary/periodic_boundary.h:136-321).
// Setup(box0, dir0, box1, dir1) turns the two AABBs into stored-cell ranges
// the way BasicBlock::getLocIdxRange does (basic_geometry.hh:448-472:
// round((min - block min) / h) .. round((max - block min) / h) - 1, block min
// = the domain's minimum less the overlap layer) and builds the device copy
// list (flb_periodic_create); Apply(), called between ApplyCellDynamics and
// Stream as in examples/couette2d/couette2d.cpp:212-214, makes the next
// Stream() copy the post-collision populations box1 -> box0 over
// getCommPopDir(dir0) and box0 -> box1 over getCommPopDir(dir1).
template <typename LatticeManager, typename FlagManager>
class FixedPeriodicBoundaryManager {
 public:
  using T = typename LatticeManager::FloatType;
  FixedPeriodicBoundaryManager(std::string name, LatticeManager& lat, FlagManager& flags,
                               std::uint8_t cellflag, std::uint8_t voidflag = std::uint8_t(1))
      : name_(std::move(name)), lat_(lat), flags_(flags), cellflag_(cellflag),
        voidflag_(voidflag) {}
  ~FixedPeriodicBoundaryManager() { flb_periodic_destroy(h_); }
  FixedPeriodicBoundaryManager(const FixedPeriodicBoundaryManager&) = delete;
  FixedPeriodicBoundaryManager& operator=(const FixedPeriodicBoundaryManager&) = delete;

  void Setup(const AABB<T, 3>& box0, NbrDirection dir0, const AABB<T, 3>& box1,
             NbrDirection dir1) {
    lat_.sync(flags_);
    int b0[6], b1[6];
    range(box0, b0);
    range(box1, b1);
    flb_periodic_destroy(h_);
    h_ = nullptr;
    flbcpp::check(flb_periodic_create(lat_.handle(), b0, int(dir0), b1, int(dir1), cellflag_, &h_),
                  "flb_periodic_create");
  }
  void Apply() {
    if (h_) lat_.arm_periodic(h_);
  }
  void getinfo() const {
    long long pairs = 0;
    if (h_) flb_periodic_count(h_, &pairs, nullptr);
    std::cout << std::setw(18) << std::left << name_ << std::setw(10) << std::left << pairs
              << std::endl;
  }

 private:
  void range(const AABB<T, 3>& box, int* out) const {
    const auto& g = lat_.getGeo();
    const T h = g.getVoxelSize();
    const Vector<T, 3> lo = g.getMinCenter() - Vector<T, 3>(T(0.5) * h);
    const int n[3] = {g.getNx(), g.getNy(), g.getNz()};
    for (int a = 0; a < 3; ++a) {
      const int i0 = int(std::round((box.getMin()[a] - lo[a]) / h));
      const int i1 = int(std::round((box.getMax()[a] - lo[a]) / h)) - 1;
      out[2 * a] = i0 < 0 ? 0 : i0;
      out[2 * a + 1] = i1 > n[a] - 1 ? n[a] - 1 : i1;
    }
  }
  std::string name_;
  LatticeManager& lat_;
  FlagManager& flags_;
  std::uint8_t cellflag_, voidflag_;
  flb_periodic* h_ = nullptr;
};

// BlockBoundaryManager (basic_boundary.h:331-348): applies its managers in order.
class BlockBoundaryManager {
 public:
  explicit BlockBoundaryManager(std::vector<AbstractBlockBoundary*> bds) : bds_(std::move(bds)) {}
  template <typename... B>
  explicit BlockBoundaryManager(B*... bs) : bds_{static_cast<AbstractBlockBoundary*>(bs)...} {}
  void Apply() {
    for (AbstractBlockBoundary* b : bds_) b->Apply();
  }
  void Apply(std::int64_t count) {
    for (AbstractBlockBoundary* b : bds_) b->Apply(count);
  }

 private:
  std::vector<AbstractBlockBoundary*> bds_;
};

// ---------------------------------------------------------------------------
// VTK output (src/io/vtm_writer.h:288-663, namespace vtmo; src/io/vti_writer.h:
// 424-986, namespace vtino): one .vti per block plus a .vtm index under
// ./vtkoutput/vtidata/, written byte for byte as the reference writes them.
// Fields resident on the device (the lattice's RHO and VELOCITY) are cropped,
// converted and base64-encoded on the GPU (flb_vtk_field_base64); host fields
// (the flag field) are encoded here.
namespace flbcpp {
inline void mkdir_one(const std::string& d) { ::mkdir(d.c_str(), 0755); }
template <typename X>
struct ident {  // keeps a parameter out of class template argument deduction
  using type = X;
};
inline void make_dir(const std::string& d) {
  std::string cur;
  for (char c : d) {
    cur += c;
    if (c == '/') mkdir_one(cur);
  }
  mkdir_one(cur);
}
// RFC 4648 base64 with '=' padding, one stream (src/io/base64.h Base64Encoder)
inline void base64_append(std::string& out, const unsigned char* p, std::size_t n) {
  static const char* a = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
  std::size_t i = 0;
  for (; i + 3 <= n; i += 3) {
    out += a[p[i] >> 2];
    out += a[((p[i] & 3) << 4) | (p[i + 1] >> 4)];
    out += a[((p[i + 1] & 15) << 2) | (p[i + 2] >> 6)];
    out += a[p[i + 2] & 63];
  }
  if (i < n) {
    const unsigned b0 = p[i], b1 = i + 1 < n ? p[i + 1] : 0u;
    out += a[b0 >> 2];
    out += a[((b0 & 3) << 4) | (b1 >> 4)];
    out += i + 1 < n ? a[(b1 & 15) << 2] : '=';
    out += '=';
  }
}
// DataArray body of host values: size block, then the data
template <typename V>
std::string base64_body(const std::vector<V>& v) {
  std::string s;
  const unsigned size = unsigned(v.size() * sizeof(V));
  base64_append(s, reinterpret_cast<const unsigned char*>(&size), sizeof size);
  base64_append(s, reinterpret_cast<const unsigned char*>(v.data()), v.size() * sizeof(V));
  return s;
}
template <typename V>
std::string device_body(flb_lattice* lat, int field, int overlap, int map, double scale,
                        double offset) {
  const int dt = std::is_same<V, double>::value ? FLB_DTYPE_F64 : FLB_DTYPE_F32;
  std::size_t len = 0;
  check(flb_vtk_field_base64(lat, 0, field, overlap, dt, map, scale, offset, nullptr, 0, &len,
                             nullptr),
        "flb_vtk_field_base64");
  std::string s(len, '\0');
  check(flb_vtk_field_base64(lat, 0, field, overlap, dt, map, scale, offset, &s[0], len, &len,
                             nullptr),
        "flb_vtk_field_base64");
  return s;
}
template <typename V>
const char* vtk_type() {
  if constexpr (std::is_same<V, double>::value) return "Float64";
  else if constexpr (std::is_same<V, float>::value) return "Float32";
  else if constexpr (std::is_same<V, std::uint8_t>::value) return "UInt8";
  else if constexpr (std::is_same<V, std::int8_t>::value) return "Int8";
  else if constexpr (std::is_same<V, std::int32_t>::value) return "Int32";
  else static_assert(sizeof(V) == 0, "no VTK type for this value type");
}
// cells [ov, n - ov) of a host array, x fastest (util::CopyFromFieldArray)
template <typename V, typename F>
std::vector<V> crop(const Vector<int, 3>& mesh, int ov, std::size_t n, F&& at) {
  std::vector<V> out;
  out.reserve(n);
  for (int k = ov; k < mesh[2] - ov; ++k)
    for (int j = ov; j < mesh[1] - ov; ++j)
      for (int i = ov; i < mesh[0] - ov; ++i)
        at(out, std::size_t(i) + std::size_t(mesh[0]) * (std::size_t(j) + std::size_t(mesh[1]) * k));
  return out;
}
// f(x) == x * scale + offset (offset 0: x * scale) for probe values, bit for bit
template <typename V>
bool affine(const std::function<V(V)>& f, double& scale, double& offset) {
  const V o = f(V(0)), sc = f(V(1)) - o;
  for (V x : {V(0.5), V(2), V(-3), V(1.25e-3), V(7.75)}) {
    const V want = o == V(0) ? x * sc : x * sc + o;
    if (!(f(x) == want)) return false;
  }
  scale = double(sc);
  offset = double(o);
  return true;
}
}  // namespace flbcpp

namespace vtmo {
class AbstractWriter {
 public:
  virtual ~AbstractWriter() = default;
  virtual void writeBinary(const std::string& fName, int Overlap) const = 0;
};
class AbstWriterSet {
 public:
  virtual ~AbstWriterSet() = default;
  virtual const AbstractWriter& getWriter(int i) const = 0;
};

namespace detail {
inline void open_array(const std::string& fName, const char* type, const std::string& name,
                       unsigned ncomp) {
  std::ofstream f(fName, std::ios::out | std::ios::app);
  f << "<DataArray type=\"" << type << "\" Name=\"" << name << "\" "
    << "format=\"binary\" encoding=\"base64\" " << "NumberOfComponents=\"" << ncomp
    << "\">\n";
}
inline void body_and_close(const std::string& fName, const std::string& body) {
  {
    std::ofstream fb(fName, std::ios::out | std::ios::app | std::ios::binary);
    fb.write(body.data(), std::streamsize(body.size()));
  }
  std::ofstream ff(fName, std::ios::out | std::ios::app);
  ff << "\n</DataArray>\n";
}
}  // namespace detail

// Scalar field of one block; Phys form maps values through `f` first.
template <typename Manager, typename V>
class ScalarArrayWriter final : public AbstractWriter {
 public:
  ScalarArrayWriter(std::string name, const Manager& fm, std::function<V(V)> f)
      : name_(std::move(name)), fm_(fm), f_(std::move(f)) {}
  void writeBinary(const std::string& fName, int Overlap) const override {
    detail::open_array(fName, flbcpp::vtk_type<V>(), name_, 1);
    detail::body_and_close(fName, body(Overlap));
  }

 private:
  std::string body(int ov) const {
    double scale = 1, offset = 0;
    const bool phys = bool(f_);
    if (fm_.device.lat && (!phys || flbcpp::affine<V>(f_, scale, offset))) {
      fm_.device.sync();
      return flbcpp::device_body<V>(fm_.device.lat, fm_.device.field, ov, phys ? 1 : 0, scale,
                                    offset);
    }
    const auto& d = fm_.field().data;
    const Vector<int, 3> mesh = fm_.geo().getMesh();
    return flbcpp::base64_body(flbcpp::crop<V>(mesh, ov, d.size(), [&](std::vector<V>& o, std::size_t id) {
      o.push_back(phys ? f_(V(d[id])) : V(d[id]));
    }));
  }
  std::string name_;
  const Manager& fm_;
  std::function<V(V)> f_;
};

template <typename Manager, typename V>
class VectorArrayWriter final : public AbstractWriter {
 public:
  using Vec = Vector<V, 3>;
  VectorArrayWriter(std::string name, const Manager& fm, std::function<Vec(Vec)> f)
      : name_(std::move(name)), fm_(fm), f_(std::move(f)) {}
  void writeBinary(const std::string& fName, int Overlap) const override {
    detail::open_array(fName, flbcpp::vtk_type<V>(), name_, 3);
    detail::body_and_close(fName, body(Overlap));
  }

 private:
  std::string body(int ov) const {
    double scale = 1, offset = 0;
    const bool phys = bool(f_);
    bool dev = fm_.device.lat != nullptr;
    if (dev && phys) {
      // component-wise affine map with the same factor on every component
      const std::function<V(V)> g = [this](V x) { return f_(Vec(x))[0]; };
      dev = flbcpp::affine<V>(g, scale, offset);
      for (V x : {V(0.5), V(-2)})
        for (int c = 0; c < 3; ++c) {
          Vec in(V(0));
          in[c] = x;
          const Vec out = f_(in);
          for (int e = 0; e < 3; ++e)
            if (!(out[e] == (e == c ? g(x) : g(V(0))))) dev = false;
        }
    }
    if (dev) {
      fm_.device.sync();
      return flbcpp::device_body<V>(fm_.device.lat, fm_.device.field, ov, phys ? 1 : 0, scale,
                                    offset);
    }
    const auto& d = fm_.field().data;
    const Vector<int, 3> mesh = fm_.geo().getMesh();
    return flbcpp::base64_body(
        flbcpp::crop<V>(mesh, ov, 3 * d.size(), [&](std::vector<V>& o, std::size_t id) {
          const Vec v = phys ? f_(d[id]) : d[id];
          for (int c = 0; c < 3; ++c) o.push_back(V(v[c]));
        }));
  }
  std::string name_;
  const Manager& fm_;
  std::function<Vec(Vec)> f_;
};

// vtmo::ScalarWriter / PhysScalarWriter / VectorWriter / PhysVectorWriter:
// one array writer per block (one device block here).
template <typename FieldType, typename FloatType, unsigned int Dim>
class ScalarWriter final : public AbstWriterSet {
  using Manager = BlockFieldManager<FieldType, FloatType, Dim>;

 public:
  ScalarWriter(std::string varname, const BlockFieldManager<FieldType, FloatType, Dim>& fm)
      : w_(std::move(varname), fm, nullptr) {}
  const AbstractWriter& getWriter(int) const override { return w_; }

 private:
  ScalarArrayWriter<Manager, typename FieldType::value_type> w_;
};
template <typename FieldType, typename FloatType, unsigned int Dim>
class PhysScalarWriter final : public AbstWriterSet {
  using Manager = BlockFieldManager<FieldType, FloatType, Dim>;
  using V = typename FieldType::value_type;

 public:
  PhysScalarWriter(std::string varname, const BlockFieldManager<FieldType, FloatType, Dim>& fm,
                   typename flbcpp::ident<std::function<V(V)>>::type f)
      : w_(std::move(varname), fm, std::move(f)) {}
  const AbstractWriter& getWriter(int) const override { return w_; }

 private:
  ScalarArrayWriter<Manager, V> w_;
};
template <typename FieldType, typename FloatType, unsigned int Dim>
class VectorWriter final : public AbstWriterSet {
  using Manager = BlockFieldManager<FieldType, FloatType, Dim>;

 public:
  VectorWriter(std::string varname, const BlockFieldManager<FieldType, FloatType, Dim>& fm)
      : w_(std::move(varname), fm, nullptr) {}
  const AbstractWriter& getWriter(int) const override { return w_; }

 private:
  VectorArrayWriter<Manager, FloatType> w_;
};
template <typename FieldType, typename FloatType, unsigned int Dim>
class PhysVectorWriter final : public AbstWriterSet {
  using Manager = BlockFieldManager<FieldType, FloatType, Dim>;
  using Vec = Vector<FloatType, 3>;

 public:
  PhysVectorWriter(std::string varname, const BlockFieldManager<FieldType, FloatType, Dim>& fm,
                   typename flbcpp::ident<std::function<Vec(Vec)>>::type f)
      : w_(std::move(varname), fm, std::move(f)) {}
  const AbstractWriter& getWriter(int) const override { return w_; }

 private:
  VectorArrayWriter<Manager, FloatType> w_;
};

// vtino::vtiManager with overlap (vti_writer.h:438-548)
template <typename T, unsigned int Dim>
class vtiManager {
 public:
  vtiManager(std::string filename, int id, T voxsize, Vector<T, Dim> min, Vector<int, Dim> ext,
             int Overlap)
      : filename_(std::move(filename)), id_(id), voxel_(voxsize), overlap_(Overlap),
        min_(min + Vector<T, Dim>(T(Overlap) * voxsize)),
        ext_(ext - Vector<int, Dim>(2 * Overlap)) {
    flbcpp::make_dir(dirname_);
  }
  void addWriter(const AbstractWriter& w) { writers_.push_back(&w); }
  void WriteBinary() { write(dirname_ + filename_ + "_B" + std::to_string(id_) + ".vti"); }
  void WriteBinary(int step) {
    write(dirname_ + filename_ + "_T" + std::to_string(step) + "_B" + std::to_string(id_) +
          ".vti");
  }

 private:
  void write(const std::string& fullName) {
    {
      std::ofstream f(fullName);
      f << "<?xml version=\"1.0\"?>\n";
      f << "<VTKFile type=\"ImageData\" version=\"0.1\" " << "byte_order=\"LittleEndian\">\n";
      f << "<ImageData WholeExtent=\"" << 0 << " " << ext_[0] << " " << 0 << " " << ext_[1] << " "
        << 0 << " " << ext_[2] << "\" Origin=\"" << min_[0] << " " << min_[1] << " " << min_[2]
        << "\" Spacing=\"" << voxel_ << " " << voxel_ << " " << voxel_ << "\">\n";
      f << "<Piece Extent=\"" << 0 << " " << ext_[0] << " " << 0 << " " << ext_[1] << " " << 0
        << " " << ext_[2] << "\">\n";
      f << "<PointData>\n";
    }
    for (const AbstractWriter* w : writers_) w->writeBinary(fullName, overlap_);
    std::ofstream f(fullName, std::ios::app);
    f << "</PointData>\n";
    f << "</Piece>\n";
    f << "</ImageData>\n";
    f << "</VTKFile>\n";
  }
  std::string dirname_ = "./vtkoutput/vtidata/";
  std::string filename_;
  int id_;
  T voxel_;
  int overlap_;
  Vector<T, Dim> min_;
  Vector<int, Dim> ext_;
  std::vector<const AbstractWriter*> writers_;
};

// vtmo::vtmWriter (vtm_writer.h:291-437)
template <typename T, unsigned int Dim>
class vtmWriter {
 public:
  // overlapth: -1 writes the whole stored block; otherwise blocks whose overlap
  // exceeds it drop (overlap - overlapth) layers on each side
  vtmWriter(std::string filename, BlockGeometry3D<T>& geo, int overlapth = -1)
      : filename_(std::move(filename)) {
    flbcpp::make_dir(dirname_);
    flbcpp::make_dir(vtidirname_);
    int ov = 0;
    if (overlapth != -1 && overlapth < geo.getOverlap()) ov = geo.getOverlap() - overlapth;
    vtis_.emplace_back(filename_, 0, geo.getVoxelSize(), geo.getMinCenter(),
                       geo.getMesh() - Vector<int, Dim>(1), ov);
  }
  void addWriterSet(const AbstWriterSet& ws) {
    int i = 0;
    for (auto& v : vtis_) v.addWriter(ws.getWriter(i++));
  }
  template <typename... Args>
  void addWriterSet(const AbstWriterSet& ws, const Args&... args) {
    addWriterSet(ws);
    addWriterSet(args...);
  }
  void WriteBinary() {
    for (auto& v : vtis_) v.WriteBinary();
    write_vtm(vtidirname_ + filename_ + ".vtm", [&](std::size_t i) {
      return filename_ + "_B" + std::to_string(i) + ".vti";
    });
  }
  void WriteBinary(int step) {
    for (auto& v : vtis_) v.WriteBinary(step);
    write_vtm(vtidirname_ + filename_ + std::to_string(step) + ".vtm", [&](std::size_t i) {
      return filename_ + "_T" + std::to_string(step) + "_B" + std::to_string(i) + ".vti";
    });
  }

 private:
  template <typename F>
  void write_vtm(const std::string& fullName, F&& vti_name) {
    std::ofstream f(fullName, std::ios::trunc);
    f << "<?xml version=\"1.0\"?>\n";
    f << "<VTKFile type=\"vtkMultiBlockDataSet\" version=\"1.0\" "
      << "byte_order=\"LittleEndian\">\n"
      << "<vtkMultiBlockDataSet>\n";
    for (std::size_t i = 0; i < vtis_.size(); ++i) {
      f << "<Block index=\"" << i << "\" >\n";
      f << "<DataSet index= \"0\" " << "file=\"" << vti_name(i) << "\">\n" << "</DataSet>\n";
      f << "</Block>\n";
    }
    f << "</vtkMultiBlockDataSet>\n";
    f << "</VTKFile>\n";
  }
  std::string dirname_ = "./vtkoutput/";
  std::string vtidirname_ = "./vtkoutput/vtidata/";
  std::string filename_;
  std::vector<vtiManager<T, Dim>> vtis_;
};
}  // namespace vtmo
