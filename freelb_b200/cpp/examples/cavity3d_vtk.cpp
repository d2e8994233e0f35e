// cavity3d_vtk.cpp -- VTK output of the lid-driven cavity through the C++17
// host classes, with the writer calls of examples/cavity3d/cavity3d.cpp.
//
//   cavity3d_vtk <Ni> <tau> <u_lid> <steps> <overlapth> <name> [fields.bin] [fp64]
//
// Sets up the cavity, optionally replaces the RHO and VELOCITY fields from
// fields.bin (N values of rho then 3N of u, float64, the stored-mesh order),
// runs <steps> steps and writes flag, rho, velocity, physRho and physVelocity
// with vtmo::vtmWriter into ./vtkoutput/vtidata/ (step number in the names).
// With Ni <= 0 only the flag field is written and no GPU is used.
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "../freelb.h"

int Thread_Num = 1;

template <typename T>
int run(int Ni, T tau, T ulid, int steps, int overlapth, const std::string& name,
        const char* fields) {
  using LatSet = D3Q19<T>;
  constexpr std::uint8_t VoidFlag = 1, AABBFlag = 2, BouncebackFlag = 4, BBMovingWallFlag = 8;
  const bool flags_only = Ni <= 0;
  if (flags_only) Ni = -Ni;
  BaseConverter<T> conv(LatSet::cs2);
  conv.SimplifiedConverterFromRT(Ni, ulid, tau);
  AABB<T, 3> cavity(Vector<T, 3>{}, Vector<T, 3>(T(Ni), T(Ni), T(Ni)));
  AABB<T, 3> toplid(Vector<T, 3>(T(1), T(1), T(Ni - 1)), Vector<T, 3>(T(Ni - 1), T(Ni - 1), T(Ni)));
  BlockGeometry3D<T> Geo(Ni, Ni, Ni, 1, cavity, T(1));
  BlockFieldManager<FLAG, T, 3> FlagFM(Geo, VoidFlag);
  FlagFM.forEach(cavity, [&](FLAG& f, std::size_t id) { f.SetField(id, AABBFlag); });
  FlagFM.template SetupBoundary<LatSet>(cavity, BouncebackFlag);
  FlagFM.forEach(toplid, [&](FLAG& f, std::size_t id) {
    if (util::isFlag(f.get(id), BouncebackFlag)) f.SetField(id, BBMovingWallFlag);
  });
  vtmo::ScalarWriter FlagWriter("flag", FlagFM);
  if (flags_only) {
    vtmo::vtmWriter<T, LatSet::d> Writer(name, Geo, overlapth);
    Writer.addWriterSet(FlagWriter);
    Writer.WriteBinary(steps);
    return 0;
  }
  using FIELDS = TypePack<RHO<T>, VELOCITY<T, 3>, POP<T, 19>>;
  using CELL = Cell<T, LatSet, FIELDS>;
  ValuePack Init(conv.getLatRhoInit(), Vector<T, 3>{}, T{});
  BlockLatticeManager<T, LatSet, FIELDS> NS(Geo, Init, conv);
  const Vector<T, 3> uw = conv.getLatticeU(Vector<T, 3>(ulid, T(0), T(0)));
  NS.template getField<VELOCITY<T, 3>>().forEach(
      toplid, FlagFM, BBMovingWallFlag, [&](auto& f, std::size_t id) { f.SetField(id, uw); });
  if (fields) {
    const std::size_t N = Geo.getTotalCellNum();
    std::vector<double> buf(4 * N);
    std::ifstream in(fields, std::ios::binary);
    in.read(reinterpret_cast<char*>(buf.data()), std::streamsize(buf.size() * sizeof(double)));
    if (!in) {
      std::fprintf(stderr, "short fields file\n");
      return 2;
    }
    auto& rho = NS.template getField<RHO<T>>().field();
    auto& vel = NS.template getField<VELOCITY<T, 3>>().field();
    for (std::size_t id = 0; id < N; ++id) {
      rho.SetField(id, T(buf[id]));
      vel.SetField(id, Vector<T, 3>(T(buf[N + 3 * id]), T(buf[N + 3 * id + 1]),
                                    T(buf[N + 3 * id + 2])));
    }
  }
  using NSTask = TaskSelector<std::uint8_t, CELL,
                              tmp::Key_TypePair<AABBFlag, collision::BGK<moment::rhoU<CELL>,
                                                                        equilibrium::SecondOrder<CELL>>>,
                              tmp::Key_TypePair<BouncebackFlag, collision::BounceBack<CELL>>,
                              tmp::Key_TypePair<BBMovingWallFlag, collision::BounceBackMovingWall<CELL>>>;
  vtmo::ScalarWriter RhoWriter("rho", NS.template getField<RHO<T>>());
  vtmo::VectorWriter VecWriter("velocity", NS.template getField<VELOCITY<T, 3>>());
  vtmo::PhysScalarWriter PhysRhoWriter("physRho", NS.template getField<RHO<T>>(),
      [&conv](T x) { return conv.getPhysRho(x); });
  vtmo::PhysVectorWriter PhysVecWriter("physVelocity", NS.template getField<VELOCITY<T, 3>>(),
      [&conv](Vector<T, 3> v) { return conv.getPhysU(v); });
  vtmo::vtmWriter<T, LatSet::d> Writer(name, Geo, overlapth);
  Writer.addWriterSet(FlagWriter, RhoWriter, VecWriter, PhysRhoWriter, PhysVecWriter);
  for (int t = 0; t < steps; ++t) {
    NS.template ApplyCellDynamics<NSTask>(FlagFM);
    NS.Stream();
  }
  // the fields as the run left them on the device (or as uploaded)
  NS.sync(FlagFM);
  Writer.WriteBinary(steps);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr,
                 "usage: %s <Ni> <tau> <u_lid> <steps> <overlapth> <name> [fields.bin] [fp64]\n",
                 argv[0]);
    return 2;
  }
  const int Ni = std::atoi(argv[1]);
  const double tau = std::atof(argv[2]), ulid = std::atof(argv[3]);
  const int steps = std::atoi(argv[4]), overlapth = std::atoi(argv[5]);
  const std::string name = argv[6];
  const char* fields = argc > 7 && std::string(argv[7]) != "-" ? argv[7] : nullptr;
  const bool fp64 = argc > 8 && std::string(argv[8]) == "fp64";
  try {
    if (fp64) return run<double>(Ni, tau, ulid, steps, overlapth, name, fields);
    return run<float>(Ni, float(tau), float(ulid), steps, overlapth, name, fields);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
