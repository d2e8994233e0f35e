// cavity3d_b200.cpp -- the lid-driven cavity through the C++17 host classes.
//
//   cavity3d_b200 <Ni> <tau> <u_lid> <steps> [model: bgk|mrt|les|halfway] [out.bin]
//
// Written against the reference's programming interface (geometry, flag
// field, converter, task selector, BlockLatticeManager): the same calls a
// FreeLB cavity program makes, executed on the GPU.  With an output path it
// writes rho (N values) then u (3N values) as float64 after refreshing them on
// the fluid cells with the moment::rhoU<CELL,true> task.  Model "halfway"
// collides wall and lid cells like fluid (BGK) and applies the post-stream
// halfway bounce-back managers after every Stream(), as
// examples/couette2d/couette2d.cpp does.
#include <cstdlib>
#include <string>

#include "../freelb.h"

int Thread_Num = 1;

template <typename Bulk, typename CELL, typename FIELDS, bool Halfway = false>
int run(int Ni, double tau, double ulid, int steps, const char* out) {
  using T = float;
  using LatSet = D3Q19<T>;
  constexpr std::uint8_t VoidFlag = 1, AABBFlag = 2, BouncebackFlag = 4, BBMovingWallFlag = 8;
  BaseConverter<T> conv(LatSet::cs2);
  conv.SimplifiedConverterFromRT(Ni, T(ulid), T(tau));
  AABB<T, 3> cavity(Vector<T, 3>{}, Vector<T, 3>(T(Ni), T(Ni), T(Ni)));
  AABB<T, 3> toplid(Vector<T, 3>(T(1), T(1), T(Ni - 1)), Vector<T, 3>(T(Ni - 1), T(Ni - 1), T(Ni)));
  BlockGeometry3D<T> Geo(Ni, Ni, Ni, 1, cavity, T(1));
  BlockFieldManager<FLAG, T, 3> FlagFM(Geo, VoidFlag);
  FlagFM.forEach(cavity, [&](FLAG& f, std::size_t id) { f.SetField(id, AABBFlag); });
  FlagFM.template SetupBoundary<LatSet>(cavity, BouncebackFlag);
  FlagFM.forEach(toplid, [&](FLAG& f, std::size_t id) {
    if (util::isFlag(f.get(id), BouncebackFlag)) f.SetField(id, BBMovingWallFlag);
  });
  ValuePack Init(conv.getLatRhoInit(), Vector<T, 3>{}, T{}, T(0.1));
  BlockLatticeManager<T, LatSet, FIELDS> NS(Geo, Init, conv);
  const Vector<T, 3> uw = conv.getLatticeU(Vector<T, 3>(T(ulid), T(0), T(0)));
  NS.template getField<VELOCITY<T, 3>>().forEach(
      toplid, FlagFM, BBMovingWallFlag, [&](auto& f, std::size_t id) { f.SetField(id, uw); });
  using NSTask = TaskSelector<std::uint8_t, CELL, tmp::Key_TypePair<AABBFlag, Bulk>,
                              tmp::Key_TypePair<BouncebackFlag, collision::BounceBack<CELL>>,
                              tmp::Key_TypePair<BBMovingWallFlag, collision::BounceBackMovingWall<CELL>>>;
  using HWTask = TaskSelector<std::uint8_t, CELL,
                              tmp::Key_TypePair<AABBFlag | BouncebackFlag | BBMovingWallFlag, Bulk>>;
  using RhoU = TaskSelector<std::uint8_t, CELL, tmp::Key_TypePair<AABBFlag, moment::rhoU<CELL, true>>>;
  using LM = BlockLatticeManager<T, LatSet, FIELDS>;
  using FM = BlockFieldManager<FLAG, T, 3>;
  Timer timer;
  if constexpr (Halfway) {
    BBLikeFixedBlockBdManager<bounceback::normal<CELL>, LM, FM> NS_BB("NS_BB", NS, FlagFM,
                                                                      BouncebackFlag, VoidFlag);
    BBLikeFixedBlockBdManager<bounceback::movingwall<CELL>, LM, FM> NS_BBMW(
        "NS_BBMW", NS, FlagFM, BBMovingWallFlag, VoidFlag);
    BlockBoundaryManager BM(&NS_BB, &NS_BBMW);
    while (timer() < steps) {
      NS.template ApplyCellDynamics<HWTask>(FlagFM);
      NS.Stream();
      BM.Apply();
      ++timer;
    }
  } else {
    while (timer() < steps) {
      NS.template ApplyCellDynamics<NSTask>(FlagFM);
      NS.Stream();
      ++timer;
    }
  }
  timer.Print_MainLoopPerformance(Geo.getTotalCellNum());
  NS.template ApplyCellDynamics<RhoU>(FlagFM);
  if (out) {
    std::ofstream f(out, std::ios::binary);
    const auto& rho = NS.template getField<RHO<T>>().field().data;
    const auto& u = NS.template getField<VELOCITY<T, 3>>().field().data;
    for (T v : rho) {
      const double d = v;
      f.write(reinterpret_cast<const char*>(&d), sizeof d);
    }
    for (const auto& v : u)
      for (int c = 0; c < 3; ++c) {
        const double d = v[c];
        f.write(reinterpret_cast<const char*>(&d), sizeof d);
      }
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s <Ni> <tau> <u_lid> <steps> [bgk|mrt|les] [out.bin]\n", argv[0]);
    return 2;
  }
  const int Ni = std::atoi(argv[1]);
  const double tau = std::atof(argv[2]), ulid = std::atof(argv[3]);
  const int steps = std::atoi(argv[4]);
  const std::string model = argc > 5 ? argv[5] : "bgk";
  const char* out = argc > 6 ? argv[6] : nullptr;
  using T = float;
  using FIELDS = TypePack<RHO<T>, VELOCITY<T, 3>, POP<T, 19>, SMAGORINSKY<T>>;
  using CELL = Cell<T, D3Q19<T>, FIELDS>;
  try {
    if (model == "mrt") return run<collision::MRT_Feq_RhoU<CELL>, CELL, FIELDS>(Ni, tau, ulid, steps, out);
    if (model == "halfway")
      return run<collision::BGK<moment::rhoU<CELL>, equilibrium::SecondOrder<CELL>>, CELL, FIELDS,
                 true>(Ni, tau, ulid, steps, out);
    if (model == "les")
      return run<collision::SmagorinskyBGK<moment::rhoU<CELL, true>, equilibrium::SecondOrder<CELL>>,
                 CELL, FIELDS>(Ni, tau, ulid, steps, out);
    return run<collision::BGK<moment::rhoU<CELL>, equilibrium::SecondOrder<CELL>>, CELL, FIELDS>(
        Ni, tau, ulid, steps, out);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
