// Oracle harness (test infrastructure only): drives the reference FreeLB CPU
// path, compiled from the reference's own headers, on the lid-driven cavity and
// dumps what the parity tests compare against.
//
// It reproduces benchmarks/cavity3d/cavity3d.cpp:111-223 (flag setup, lattice
// construction, moving-lid velocity, NSTask = first-matching-key selector over
// {2: bulk collision, 4: BounceBack, 8: BounceBackMovingWall},
// ApplyCellDynamics + Stream per step) with lattice parameters taken from the
// command line instead of an ini file:
//
//   ref_cavity <model> <Ni> <RT> <u_lid> <steps> <warmup> <outdir|-> [Cs] [blockfile]
//
//   model     bgk | les | mrt
//             bgk: collision::BGK<moment::rhoU, equilibrium::SecondOrder>
//             les: collision::SmagorinskyBGK<moment::rhoU<CELL,true>, SecondOrder>
//                  (rhoU writes RHO, so the RHO field read at collisionLES.h:50
//                   holds the local density of this step)
//             mrt: collision::MRT_Feq_RhoU with the D3Q19 basis specialised in
//                  mrt_d3q19_table.h (the reference ships only D2Q9 data)
//             brinkman: BGK with a Brinkman drag F = -alpha u built from the
//                  reference's own pieces (BrinkmanBGK below); per-cell alpha
//                  read from the file named by FLB_ALPHA_FILE (N values of T,
//                  reference cell order; zero when unset)
//   Ni        interior cells per axis (stored mesh is (Ni+2)^3, one void layer)
//   RT        relaxation time tau (lattice units; dx = dt = 1 so u_lid is lattice)
//   FLB_VTK_NAME=<name> (environment): after the main loop, the reference's
//             vtmo writers write flag, rho, velocity, physRho, physVelocity
//             into ./vtkoutput/vtidata/ (FLB_VTK_OVERLAP: overlap threshold).
//   FLB_FIELDS_FILE (environment, single block): RHO (N values of T) and
//             VELOCITY (3N, x y z per cell) replacing both fields after setup.
//   FLB_POSTSTREAM_BB=<k> (environment): wall and lid cells collide with the
//             bulk policy and the reference's post-stream managers
//             BBLikeFixedBlockBdManager (boundary/boundary.h:86-140) run after
//             every Stream(), as in examples/couette2d/couette2d.cpp:212-216:
//             the lid (8) with bounceback::movingwall and the walls (4) with
//             bounceback::normal (k=1), anti_simple (2), anti_O1 (3),
//             anti_O2 (4) or anti_pressure (5) (bounce_back_boundary.h:167-256).
//   FLB_PERIODIC=1 (environment): the wall cells of the x = 0 and x = Ni-1
//             interior columns (y, z inside [1, Nj-1] x [1, Nk-1]) take flag 16,
//             which no task matches (no collision), and a
//             FixedPeriodicBoundaryManager (boundary/periodic_boundary.h:136-321)
//             on those two boxes, Setup(left, XN, right, XP), runs Apply()
//             between ApplyCellDynamics and Stream as in
//             examples/couette2d/couette2d.cpp:171-214.  Use a block file whose
//             first block holds the x = 0 column and a later block the
//             x = Ni-1 column (the manager's cross-block pairing).
//   blockfile optional BlockReader file (io/block_reader.h) for a multi-block run;
//             NormalCommunicate() (FLB_COMM=full / all: NormalFullCommunicate /
//             NormalAllCommunicate) follows Stream() as in
//             examples/cavity3d/cavity3d.cpp:220.
//
// Output (when outdir != "-"): meta.txt, flags.u8, pops.bin (19 x N, logical
// order after the PS rotation), rho.bin (N), u.bin (3N, AoS) -- per block with
// suffix _b<k> -- where rho/u are refreshed on fluid cells with
// moment::rhoU<CELL,true> after the last step (examples/cavity3d/cavity3d.cpp:191-194).
// It always prints one line "MLUPS <value> CELLS <n> STEPS <k> SECONDS <t> THREADS <p>"
// using the reference's Timer (utils/timer.h:50-112).

#include "freelb.h"
#include "freelb.hh"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <fstream>

#include "mrt_d3q19_table.h"

#ifdef _OPENMP
#include <omp.h>
#endif

int Thread_Num = 1;

#ifndef REF_T
#define REF_T float
#endif
using T = REF_T;
using LatSet = D3Q19<T>;

constexpr std::uint8_t VoidFlag = std::uint8_t(1);
constexpr std::uint8_t AABBFlag = std::uint8_t(2);
constexpr std::uint8_t BouncebackFlag = std::uint8_t(4);
constexpr std::uint8_t BBMovingWallFlag = std::uint8_t(8);
constexpr std::uint8_t PeriodicFlag = std::uint8_t(16);

// Per-cell Brinkman porosity for the single-block run (FLB_ALPHA_FILE).
static std::vector<T> g_alpha;

// BGK with Brinkman drag F = -alpha u, assembled from the reference's own
// components: the forced moment of moment::forcerhoUImpl (moment.h:408-422),
// u = (sum c f + F/2) / rho, solved for F = -alpha u as u = sum c f / (rho + alpha/2);
// force::ForcePop (force.h:29-36) for the discrete force; equilibrium::SecondOrder;
// the update of collision::BGKForce (collision.h:61-90).
template <typename CELL>
struct BrinkmanBGK {
  using LS = typename CELL::LatticeSet;
  static void apply(CELL& cell) {
    const T alpha = g_alpha.empty() ? T{} : g_alpha[cell.getId()];
    T rho{};
    Vector<T, LS::d> m{};
    for (unsigned int i = 0; i < LS::q; ++i) {
      rho += cell[i];
      m += latset::c<LS>(i) * cell[i];
    }
    const Vector<T, LS::d> u = m / (rho + T{0.5} * alpha);
    const Vector<T, LS::d> F = u * (-alpha);
    std::array<T, LS::q> fi{};
    force::ForcePop<T, LS>::compute(fi, u, F);
    std::array<T, LS::q> feq{};
    equilibrium::SecondOrder<CELL>::apply(feq, rho, u);
    const T omega = cell.getOmega();
    const T _omega = cell.get_Omega();
    const T fomega = cell.getfOmega();
    for (unsigned int i = 0; i < LS::q; ++i)
      cell[i] = omega * feq[i] + _omega * cell[i] + fomega * fi[i];
  }
};

struct Params {
  std::string model;
  int Ni;
  T RT;
  T ulid;
  int steps;
  int warmup;
  std::string outdir;
  T Cs;
  std::string blockfile;
};

template <typename V>
static void dump(const std::string& path, const V* data, std::size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(data), sizeof(V) * n);
}

template <typename FIELDS, typename GEO>
struct Runner {
  using CELL = Cell<T, LatSet, FIELDS>;

  template <typename BulkPolicy, typename INITVALUES>
  static void run(const Params& p, GEO& Geo, BaseConverter<T>& BaseConv, INITVALUES& InitValues,
                  const AABB<T, 3>& cavity, const AABB<T, 3>& toplid) {
    BlockFieldManager<FLAG, T, 3> FlagFM(Geo, VoidFlag);
    FlagFM.forEach(cavity, [&](FLAG& field, std::size_t id) { field.SetField(id, AABBFlag); });
    FlagFM.template SetupBoundary<LatSet>(cavity, BouncebackFlag);
    FlagFM.forEach(toplid, [&](FLAG& field, std::size_t id) {
      if (util::isFlag(field.get(id), BouncebackFlag)) field.SetField(id, BBMovingWallFlag);
    });
    const char* pe = std::getenv("FLB_PERIODIC");
    const bool periodic = pe && std::atoi(pe) == 1;
    const T nx = cavity.getMax()[0], ny = cavity.getMax()[1], nz = cavity.getMax()[2];
    const AABB<T, 3> left(Vector<T, 3>(T(0), T(1), T(1)), Vector<T, 3>(T(1), ny - 1, nz - 1));
    const AABB<T, 3> right(Vector<T, 3>(nx - 1, T(1), T(1)), Vector<T, 3>(nx, ny - 1, nz - 1));
    if (periodic) {
      FlagFM.forEach(left, [&](FLAG& field, std::size_t id) {
        if (util::isFlag(field.get(id), BouncebackFlag)) field.SetField(id, PeriodicFlag);
      });
      FlagFM.forEach(right, [&](FLAG& field, std::size_t id) {
        if (util::isFlag(field.get(id), BouncebackFlag)) field.SetField(id, PeriodicFlag);
      });
    }

    BlockLatticeManager<T, LatSet, FIELDS> NSLattice(Geo, InitValues, BaseConv);
    Vector<T, 3> U_Wall{p.ulid, T{}, T{}};
    Vector<T, 3> LatU_Wall = BaseConv.getLatticeU(U_Wall);
    NSLattice.template getField<VELOCITY<T, LatSet::d>>().forEach(
      toplid, FlagFM, BBMovingWallFlag,
      [&](auto& field, std::size_t id) { field.SetField(id, LatU_Wall); });
    // FLB_FIELDS_FILE (single block): N values of T for RHO, then 3N for
    // VELOCITY (x y z per cell), replacing both fields on every cell.
    if (const char* ff = std::getenv("FLB_FIELDS_FILE")) {
      auto& blat = NSLattice.getBlockLat(0);
      const std::size_t N = blat.getN();
      std::vector<T> buf(4 * N);
      std::ifstream in(ff, std::ios::binary);
      in.read(reinterpret_cast<char*>(buf.data()), std::streamsize(buf.size() * sizeof(T)));
      if (!in) {
        std::fprintf(stderr, "FLB_FIELDS_FILE: short read\n");
        std::exit(2);
      }
      auto& rhof = blat.template getField<RHO<T>>().getField(0);
      auto& uf = blat.template getField<VELOCITY<T, LatSet::d>>().getField(0);
      for (std::size_t id = 0; id < N; ++id) {
        rhof[id] = buf[id];
        for (int d = 0; d < 3; ++d) uf[id][d] = buf[N + 3 * id + d];
      }
    }

    using BulkTask = tmp::Key_TypePair<AABBFlag, BulkPolicy>;
    using BBTask = tmp::Key_TypePair<BouncebackFlag, collision::BounceBack<CELL>>;
    using BBMVTask = tmp::Key_TypePair<BBMovingWallFlag, collision::BounceBackMovingWall<CELL>>;
    using NSTask = TaskSelector<std::uint8_t, CELL, BulkTask, BBTask, BBMVTask>;
    using AllBulkTask =
      tmp::Key_TypePair<AABBFlag | BouncebackFlag | BBMovingWallFlag, BulkPolicy>;
    using HWTask = TaskSelector<std::uint8_t, CELL, AllBulkTask>;
    using RhoUtask = tmp::Key_TypePair<AABBFlag, moment::rhoU<CELL, true>>;
    using RhoUTask = TaskSelector<std::uint8_t, CELL, RhoUtask>;
    using LM = BlockLatticeManager<T, LatSet, FIELDS>;
    using FM = BlockFieldManager<FLAG, T, 3>;
    BBLikeFixedBlockBdManager<bounceback::normal<CELL>, LM, FM> NS_BB("NS_BB", NSLattice, FlagFM,
                                                                      BouncebackFlag, VoidFlag);
    BBLikeFixedBlockBdManager<bounceback::anti_simple<CELL>, LM, FM> NS_ABB1(
      "NS_ABB1", NSLattice, FlagFM, BouncebackFlag, VoidFlag);
    BBLikeFixedBlockBdManager<bounceback::anti_O1<CELL>, LM, FM> NS_ABB2(
      "NS_ABB2", NSLattice, FlagFM, BouncebackFlag, VoidFlag);
    BBLikeFixedBlockBdManager<bounceback::anti_O2<CELL>, LM, FM> NS_ABB3(
      "NS_ABB3", NSLattice, FlagFM, BouncebackFlag, VoidFlag);
    BBLikeFixedBlockBdManager<bounceback::anti_pressure<CELL>, LM, FM> NS_ABB4(
      "NS_ABB4", NSLattice, FlagFM, BouncebackFlag, VoidFlag);
    BBLikeFixedBlockBdManager<bounceback::movingwall<CELL>, LM, FM> NS_BBMW(
      "NS_BBMW", NSLattice, FlagFM, BBMovingWallFlag, VoidFlag);
    FixedPeriodicBoundaryManager<LM, FM> NS_Peri("NS_Peri", NSLattice, FlagFM, PeriodicFlag,
                                                 VoidFlag);
    if (periodic) NS_Peri.Setup(left, NbrDirection::XN, right, NbrDirection::XP);
    // FLB_COMM=full / all: NormalFullCommunicate / NormalAllCommunicate
    const char* cm = std::getenv("FLB_COMM");
    const int comm = cm ? (std::string(cm) == "full" ? 1 : (std::string(cm) == "all" ? 2 : 0)) : 0;
    const char* hw = std::getenv("FLB_POSTSTREAM_BB");
    const int wallkind = hw ? std::atoi(hw) : 0;
    const bool poststream = wallkind >= 1 && wallkind <= 5;

    const bool multi = Geo.getBlockNum() > 1;
    auto step = [&]() {
      if (poststream) {
        NSLattice.template ApplyCellDynamics<HWTask>(FlagFM);
        NSLattice.Stream();
        switch (wallkind) {
          case 1: NS_BB.Apply(); break;
          case 2: NS_ABB1.Apply(); break;
          case 3: NS_ABB2.Apply(); break;
          case 4: NS_ABB3.Apply(); break;
          default: NS_ABB4.Apply(); break;
        }
        NS_BBMW.Apply();
      } else {
        NSLattice.template ApplyCellDynamics<NSTask>(FlagFM);
        if (periodic) NS_Peri.Apply();
        NSLattice.Stream();
      }
      if (multi) {
        if (comm == 1) NSLattice.NormalFullCommunicate();
        else if (comm == 2) NSLattice.NormalAllCommunicate();
        else NSLattice.NormalCommunicate();
      }
    };
    for (int i = 0; i < p.warmup; ++i) step();
    Timer MainLoopTimer;
    MainLoopTimer.START_TIMER();
    while (MainLoopTimer() < p.steps) {
      step();
      ++MainLoopTimer;
    }
    MainLoopTimer.END_TIMER();
    // FLB_VTK_NAME (environment): write the fields with the reference's vtmo
    // writers into ./vtkoutput/vtidata/ of the working directory, before the
    // rhoU output task (FLB_VTK_OVERLAP: the writers' overlap threshold).
    if (const char* vn = std::getenv("FLB_VTK_NAME")) {
      const char* vo = std::getenv("FLB_VTK_OVERLAP");
      const int overlapth = vo ? std::atoi(vo) : -1;
      vtmo::ScalarWriter FlagWriter("flag", FlagFM);
      vtmo::ScalarWriter RhoWriter("rho", NSLattice.template getField<RHO<T>>());
      vtmo::VectorWriter VecWriter("velocity", NSLattice.template getField<VELOCITY<T, LatSet::d>>());
      vtmo::PhysScalarWriter PhysRhoWriter(
        "physRho", NSLattice.template getField<RHO<T>>(),
        std::bind(&BaseConverter<T>::getPhysRho, &BaseConv, std::placeholders::_1));
      vtmo::PhysVectorWriter PhysVecWriter(
        "physVelocity", NSLattice.template getField<VELOCITY<T, LatSet::d>>(),
        std::bind(&BaseConverter<T>::template getPhysU<LatSet::d>, &BaseConv, std::placeholders::_1));
      vtmo::vtmWriter<T, LatSet::d> Writer(vn, Geo, overlapth);
      Writer.addWriterSet(FlagWriter, RhoWriter, VecWriter, PhysRhoWriter, PhysVecWriter);
      Writer.WriteBinary(p.steps);
    }
    const double ms = double(std::chrono::duration_cast<std::chrono::microseconds>(
                               MainLoopTimer.END - MainLoopTimer.START).count()) / 1000.0;
    const double cells = double(Geo.getTotalCellNum());
    const double mlups = ms > 0 ? double(p.steps) * cells / ms / 1000.0 : 0.0;
    std::printf("MLUPS %.6f CELLS %.0f STEPS %d SECONDS %.6f THREADS %d\n", mlups, cells,
                p.steps, ms / 1000.0, Thread_Num);

    if (p.outdir == "-") return;
    NSLattice.template ApplyCellDynamics<RhoUTask>(FlagFM);
    {
      std::ofstream meta(p.outdir + "/meta.txt");
      meta.precision(17);
      meta << "model " << p.model << "\nNi " << p.Ni << "\nRT " << p.RT << "\nulid " << p.ulid
           << "\nsteps " << p.steps << "\nwarmup " << p.warmup << "\nblocks " << Geo.getBlockNum()
           << "\nsizeofT " << sizeof(T) << "\nomega " << BaseConv.getOMEGA() << "\n";
      for (int ib = 0; ib < Geo.getBlockNum(); ++ib) {
        const auto& blk = Geo.getBlock(ib);
        meta << "block " << ib << " mesh " << blk.getNx() << " " << blk.getNy() << " "
             << blk.getNz() << " min " << blk.getMin()[0] << " " << blk.getMin()[1] << " "
             << blk.getMin()[2] << " overlap " << blk.getOverlap() << "\n";
      }
    }
    for (int ib = 0; ib < Geo.getBlockNum(); ++ib) {
      auto& blat = NSLattice.getBlockLat(ib);
      const std::size_t N = blat.getN();
      const std::string sfx = multi ? ("_b" + std::to_string(ib)) : std::string();
      const auto& flagarr = FlagFM.getBlockField(ib).getField(0);
      std::vector<std::uint8_t> flags(N);
      for (std::size_t id = 0; id < N; ++id) flags[id] = flagarr[id];
      dump(p.outdir + "/flags" + sfx + ".u8", flags.data(), N);
      std::vector<T> pops(19 * N);
      auto& popf = blat.template getField<POP<T, LatSet::q>>();
      for (int i = 0; i < 19; ++i)
        for (std::size_t id = 0; id < N; ++id) pops[i * N + id] = popf.getField(i)[id];
      dump(p.outdir + "/pops" + sfx + ".bin", pops.data(), 19 * N);
      std::vector<T> rho(N), u(3 * N);
      auto& rhof = blat.template getField<RHO<T>>().getField(0);
      auto& uf = blat.template getField<VELOCITY<T, LatSet::d>>().getField(0);
      for (std::size_t id = 0; id < N; ++id) {
        rho[id] = rhof[id];
        for (int d = 0; d < 3; ++d) u[3 * id + d] = uf[id][d];
      }
      dump(p.outdir + "/rho" + sfx + ".bin", rho.data(), N);
      dump(p.outdir + "/u" + sfx + ".bin", u.data(), 3 * N);
    }
  }
};

template <typename GEO>
static void dispatch(const Params& p, GEO& Geo, BaseConverter<T>& BaseConv,
                     const AABB<T, 3>& cavity, const AABB<T, 3>& toplid) {
  if (p.model == "bgk") {
    using FIELDS = TypePack<RHO<T>, VELOCITY<T, LatSet::d>, POP<T, LatSet::q>>;
    using CELL = Cell<T, LatSet, FIELDS>;
    ValuePack InitValues(BaseConv.getLatRhoInit(), Vector<T, 3>{}, T{});
    Runner<FIELDS, GEO>::template run<
      collision::BGK<moment::rhoU<CELL>, equilibrium::SecondOrder<CELL>>>(
        p, Geo, BaseConv, InitValues, cavity, toplid);
  } else if (p.model == "mrt") {
    using FIELDS = TypePack<RHO<T>, VELOCITY<T, LatSet::d>, POP<T, LatSet::q>>;
    using CELL = Cell<T, LatSet, FIELDS>;
    ValuePack InitValues(BaseConv.getLatRhoInit(), Vector<T, 3>{}, T{});
    Runner<FIELDS, GEO>::template run<collision::MRT_Feq_RhoU<CELL>>(p, Geo, BaseConv,
                                                                      InitValues, cavity, toplid);
  } else if (p.model == "brinkman") {
    using FIELDS = TypePack<RHO<T>, VELOCITY<T, LatSet::d>, POP<T, LatSet::q>>;
    using CELL = Cell<T, LatSet, FIELDS>;
    ValuePack InitValues(BaseConv.getLatRhoInit(), Vector<T, 3>{}, T{});
    if (const char* af = std::getenv("FLB_ALPHA_FILE")) {
      std::ifstream in(af, std::ios::binary);
      in.seekg(0, std::ios::end);
      const std::size_t n = std::size_t(in.tellg()) / sizeof(T);
      in.seekg(0);
      g_alpha.resize(n);
      in.read(reinterpret_cast<char*>(g_alpha.data()), n * sizeof(T));
    }
    Runner<FIELDS, GEO>::template run<BrinkmanBGK<CELL>>(p, Geo, BaseConv, InitValues, cavity,
                                                         toplid);
  } else if (p.model == "les") {
    using FIELDS =
      TypePack<RHO<T>, VELOCITY<T, LatSet::d>, POP<T, LatSet::q>, SMAGORINSKY<T>>;
    using CELL = Cell<T, LatSet, FIELDS>;
    ValuePack InitValues(BaseConv.getLatRhoInit(), Vector<T, 3>{}, T{}, p.Cs);
    Runner<FIELDS, GEO>::template run<
      collision::SmagorinskyBGK<moment::rhoU<CELL, true>, equilibrium::SecondOrder<CELL>>>(
        p, Geo, BaseConv, InitValues, cavity, toplid);
  } else {
    std::fprintf(stderr, "unknown model %s\n", p.model.c_str());
    std::exit(2);
  }
}

int main(int argc, char** argv) {
  if (argc < 8) {
    std::fprintf(stderr,
                 "usage: %s <bgk|les|mrt> <Ni> <RT> <u_lid> <steps> <warmup> <outdir|-> [Cs] "
                 "[blockfile]\n",
                 argv[0]);
    return 2;
  }
  Params p;
  p.model = argv[1];
  p.Ni = std::atoi(argv[2]);
  p.RT = T(std::atof(argv[3]));
  p.ulid = T(std::atof(argv[4]));
  p.steps = std::atoi(argv[5]);
  p.warmup = std::atoi(argv[6]);
  p.outdir = argv[7];
  p.Cs = argc > 8 ? T(std::atof(argv[8])) : T(0.1);
  p.blockfile = argc > 9 ? argv[9] : "";
#ifdef _OPENMP
  Thread_Num = omp_get_max_threads();
#endif
  const T Cell_Len = T(1);
  // dx = dt = 1: lattice and physical units coincide (unit_converter.h:225-228)
  BaseConverter<T> BaseConv(LatSet::cs2);
  BaseConv.SimplifiedConverterFromRT(p.Ni, p.ulid, p.RT);

  const int Ni = p.Ni, Nj = p.Ni, Nk = p.Ni;
  AABB<T, 3> cavity(Vector<T, 3>{},
                    Vector<T, 3>(T(Ni * Cell_Len), T(Nj * Cell_Len), T(Nk * Cell_Len)));
  AABB<T, 3> toplid(Vector<T, 3>(Cell_Len, Cell_Len, T((Nk - 1) * Cell_Len)),
                    Vector<T, 3>(T((Ni - 1) * Cell_Len), T((Nj - 1) * Cell_Len), T(Nk * Cell_Len)));
  if (p.blockfile.empty()) {
    BlockGeometry3D<T> Geo(Ni, Nj, Nk, 1, cavity, Cell_Len);
    dispatch(p, Geo, BaseConv, cavity, toplid);
  } else {
    BlockReader<T, 3> reader(p.blockfile);
    BlockGeometry3D<T> Geo(reader, true);
    dispatch(p, Geo, BaseConv, cavity, toplid);
  }
  return 0;
}
