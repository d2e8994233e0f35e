// periodic3d_b200.cpp -- the lid-driven cavity made periodic in x through the
// C++17 host classes' FixedPeriodicBoundaryManager.
//
//   periodic3d_b200 <Ni> <tau> <u_lid> <steps> [out.bin]
//
// The wall cells of the x = 0 and x = Ni-1 interior columns take flag 16, which
// no task matches, and a FixedPeriodicBoundaryManager on the two columns,
// Setup(left, XN, right, XP), runs Apply() between ApplyCellDynamics and Stream
// (examples/couette2d/couette2d.cpp:171-214 in the reference).  With an output
// path it writes the populations (19 x N, reference cell order, float64).
#include <cstdlib>
#include <fstream>
#include <vector>

#include "../freelb.h"

int Thread_Num = 1;

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s <Ni> <tau> <u_lid> <steps> [out.bin]\n", argv[0]);
    return 2;
  }
  const int Ni = std::atoi(argv[1]);
  const double tau = std::atof(argv[2]), ulid = std::atof(argv[3]);
  const int steps = std::atoi(argv[4]);
  using T = float;
  using LatSet = D3Q19<T>;
  using FIELDS = TypePack<RHO<T>, VELOCITY<T, 3>, POP<T, 19>>;
  using CELL = Cell<T, LatSet, FIELDS>;
  constexpr std::uint8_t VoidFlag = 1, AABBFlag = 2, BouncebackFlag = 4, BBMovingWallFlag = 8,
                         PeriodicFlag = 16;
  BaseConverter<T> conv(LatSet::cs2);
  conv.SimplifiedConverterFromRT(Ni, T(ulid), T(tau));
  AABB<T, 3> cavity(Vector<T, 3>{}, Vector<T, 3>(T(Ni), T(Ni), T(Ni)));
  AABB<T, 3> toplid(Vector<T, 3>(T(1), T(1), T(Ni - 1)), Vector<T, 3>(T(Ni - 1), T(Ni - 1), T(Ni)));
  AABB<T, 3> left(Vector<T, 3>(T(0), T(1), T(1)), Vector<T, 3>(T(1), T(Ni - 1), T(Ni - 1)));
  AABB<T, 3> right(Vector<T, 3>(T(Ni - 1), T(1), T(1)), Vector<T, 3>(T(Ni), T(Ni - 1), T(Ni - 1)));
  BlockGeometry3D<T> Geo(Ni, Ni, Ni, 1, cavity, T(1));
  BlockFieldManager<FLAG, T, 3> FlagFM(Geo, VoidFlag);
  FlagFM.forEach(cavity, [&](FLAG& f, std::size_t id) { f.SetField(id, AABBFlag); });
  FlagFM.template SetupBoundary<LatSet>(cavity, BouncebackFlag);
  FlagFM.forEach(toplid, [&](FLAG& f, std::size_t id) {
    if (util::isFlag(f.get(id), BouncebackFlag)) f.SetField(id, BBMovingWallFlag);
  });
  FlagFM.forEach(left, [&](FLAG& f, std::size_t id) {
    if (util::isFlag(f.get(id), BouncebackFlag)) f.SetField(id, PeriodicFlag);
  });
  FlagFM.forEach(right, [&](FLAG& f, std::size_t id) {
    if (util::isFlag(f.get(id), BouncebackFlag)) f.SetField(id, PeriodicFlag);
  });
  ValuePack Init(conv.getLatRhoInit(), Vector<T, 3>{}, T{});
  BlockLatticeManager<T, LatSet, FIELDS> NS(Geo, Init, conv);
  const Vector<T, 3> uw = conv.getLatticeU(Vector<T, 3>(T(ulid), T(0), T(0)));
  NS.template getField<VELOCITY<T, 3>>().forEach(
      toplid, FlagFM, BBMovingWallFlag, [&](auto& f, std::size_t id) { f.SetField(id, uw); });
  using Bulk = collision::BGK<moment::rhoU<CELL>, equilibrium::SecondOrder<CELL>>;
  using NSTask = TaskSelector<std::uint8_t, CELL, tmp::Key_TypePair<AABBFlag, Bulk>,
                              tmp::Key_TypePair<BouncebackFlag, collision::BounceBack<CELL>>,
                              tmp::Key_TypePair<BBMovingWallFlag, collision::BounceBackMovingWall<CELL>>>;
  using LM = BlockLatticeManager<T, LatSet, FIELDS>;
  using FM = BlockFieldManager<FLAG, T, 3>;
  FixedPeriodicBoundaryManager<LM, FM> NS_Peri("NS_Peri", NS, FlagFM, PeriodicFlag, VoidFlag);
  NS_Peri.Setup(left, NbrDirection::XN, right, NbrDirection::XP);
  NS_Peri.getinfo();
  Timer timer;
  while (timer() < steps) {
    NS.template ApplyCellDynamics<NSTask>(FlagFM);
    NS_Peri.Apply();
    NS.Stream();
    ++timer;
  }
  timer.Print_MainLoopPerformance(Geo.getTotalCellNum());
  if (argc > 5) {
    const std::size_t N = Geo.getTotalCellNum();
    std::vector<T> pops(19 * N);
    flbcpp::check(flb_download_pops(NS.handle(), pops.data(), FLB_DTYPE_F32, nullptr),
                  "flb_download_pops");
    std::ofstream f(argv[5], std::ios::binary);
    for (T v : pops) {
      const double d = v;
      f.write(reinterpret_cast<const char*>(&d), sizeof d);
    }
  }
  return 0;
}
