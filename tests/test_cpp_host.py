"""The C++17 host classes (freelb_b200/cpp/freelb.h): reference programs compile
against them unchanged, and the example program runs the cavity on the GPU."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, rel_maxnorm

INC = os.path.join(ROOT, "freelb_b200", "cpp")
LIBDIR = os.path.join(ROOT, "freelb_b200")
# The reference project's root for the compile tests (FLB_REFERENCE_ROOT); the
# build step compiles the same programs where the sources are, and the GPU
# tests run whichever of them exist.
REF_ROOT = os.environ.get("FLB_REFERENCE_ROOT")
needs_ref = pytest.mark.skipif(
    not (REF_ROOT and os.path.exists(os.path.join(REF_ROOT, "src", "freelb.h"))),
    reason="FLB_REFERENCE_ROOT does not point at the reference sources")


def _gxx(args):
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    return subprocess.run(["g++", "-std=c++17", "-O1"] + args, capture_output=True, text=True,
                          env=env)


@needs_ref
def test_reference_benchmark_compiles_unchanged_against_host_classes():
    """benchmarks/cavity3d/cavity3d.cpp, untouched, with only the include path
    changed, compiles and links against libflb_b200.so."""
    from freelb_b200 import build as B
    assert os.path.exists(B.build_reference_program("cpu", REF_ROOT, force=True))


@needs_ref
def test_reference_cuda_benchmark_compiles_unchanged_against_host_classes():
    """benchmarks/cavity3d_cu/cavity3d.cu (CuDevApplyCellDynamics / CuDevStream,
    cudev::Cell, copyToDevice), untouched, compiles with nvcc and links against
    libflb_b200.so with only the include path changed."""
    from freelb_b200 import build as B
    assert os.path.exists(B.build_reference_program("cu", REF_ROOT, force=True))


@needs_ref
@pytest.mark.parametrize("kind", ["example", "example_f32"])
def test_reference_cavity3d_example_compiles_unchanged_against_host_classes(kind):
    """examples/cavity3d/cavity3d.cpp (post-stream bounce-back managers, vtmo
    writers, getToleranceU, NormalCommunicate, the MPI rank guards), untouched,
    compiles and links against the host classes for FLOAT_TYPE double and float."""
    from freelb_b200 import build as B
    assert os.path.exists(B.build_reference_program(kind, REF_ROOT, force=True))


CAVITY_INI = """[parallel]
thread_num = 1
block_num = 1
[Mesh]
Ni = 24
Nj = 24
Nk = 24
Cell_Len = 1
BlockCellLen = 8
[Physical_Property]
rho_ref = 1
Kine_Visc = 0.01
[Init_Conditions]
U_Ini0 = 0
U_Ini1 = 0
U_Ini2 = 0
U_Max = 0.1
[Boundary_Conditions]
Velo_Wall0 = 0.1
Velo_Wall1 = 0
Velo_Wall2 = 0
[LB]
RT = 0.53
[Simulation_Settings]
TotalStep = 30
OutputStep = 10
[tolerance]
tol = 1e-9
"""


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["cpu", "cu"])
def test_reference_benchmark_programs_run_on_gpu(gpu_ok, kind):
    """The reference's two cavity3d benchmark programs (CPU and CUDA), built
    unchanged against the host classes, run their main loop on the GPU (they
    print only their timing; the example program's output is compared with the
    reference's own build below)."""
    from freelb_b200 import build as B
    exe = B.ref_program_path(kind)
    if not os.path.exists(exe):
        pytest.skip("reference benchmark programs not built (no reference sources at build)")
    with tempfile.TemporaryDirectory() as d:
        open(os.path.join(d, "cavity3d.ini"), "w").write(CAVITY_INI)
        r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "MLUPs" in r.stdout


def test_host_example_compiles():
    src = os.path.join(INC, "examples", "cavity3d_b200.cpp")
    with tempfile.TemporaryDirectory() as d:
        r = _gxx(["-fsyntax-only", src])
        assert r.returncode == 0, r.stderr[-3000:]


def test_unknown_policy_is_a_compile_error():
    """A policy without a device op must not compile (no CPU fallback)."""
    code = '''#include "freelb.h"
int Thread_Num = 1;
struct MyPolicy {};
using T = float;
using CELL = Cell<T, D3Q19<T>, TypePack<RHO<T>>>;
int main() { auto t = flbcpp::task_list<TaskSelector<std::uint8_t, CELL,
             tmp::Key_TypePair<2, MyPolicy>>>(); return t.n; }
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "bad.cpp")
        open(src, "w").write(code)
        r = _gxx(["-fsyntax-only", "-I" + INC, src])
        assert r.returncode != 0 and "no CPU fallback" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
def test_host_example_runs_on_gpu_and_matches_oracle(gpu_ok, model):
    from freelb_b200 import build as B
    from oracle import oracle as O
    exe = B.build_examples()
    ni, tau, steps = 20, 0.55, 80
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        r = subprocess.run([exe, str(ni), str(tau), "0.1", str(steps), model, out],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert "Average_MLUPs" in r.stdout
        data = np.fromfile(out, dtype=np.float64)
    N = (ni + 2) ** 3
    rho, u = data[:N], data[N:]
    ref = O.cavity(ni, model=model, tau=tau, ulid=0.1, cs=0.1)
    ref.step(steps)
    rrho, ru = ref.rhou_fields()
    assert rel_maxnorm(rho, rrho) < 1e-5
    assert rel_maxnorm(u, ru) < 1e-5


@pytest.mark.gpu
def test_host_example_halfway_bounce_back_managers(gpu_ok):
    """BBLikeFixedBlockBdManager<bounceback::normal / movingwall> through the host
    classes against the oracle's post-stream restatement."""
    from freelb_b200 import build as B
    from oracle import oracle as O
    exe = B.build_examples()
    ni, tau, steps = 16, 0.6, 60
    n = ni + 2
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        r = subprocess.run([exe, str(ni), str(tau), "0.1", str(steps), "halfway", out],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        data = np.fromfile(out, dtype=np.float64)
    N = n ** 3
    fl = O.cavity_flags(ni)
    ref = O.Lattice(n, n, n, fl, tau=tau, dtype=np.float32, keys=(2 | 4 | 8,), ops=(O.OP_BULK,))
    ref.u.reshape(-1, 3)[fl == 8, 0] = np.float32(0.1)
    for _ in range(steps):
        ref.step(1)
        O.poststream_bb(ref, 4, 1, "normal")
        O.poststream_bb(ref, 8, 1, "movingwall")
    rrho, ru = ref.rhou_fields()
    assert rel_maxnorm(data[:N], rrho) < 1e-5
    assert rel_maxnorm(data[N:], ru) < 1e-5


@pytest.mark.gpu
def test_host_periodic_manager_matches_reference(gpu_ok):
    """FixedPeriodicBoundaryManager through the host classes (AABB boxes,
    Setup(left, XN, right, XP), Apply() between ApplyCellDynamics and Stream)
    against the reference's own periodic run (tests/golden/periodic_*)."""
    from freelb_b200 import build as B
    from conftest import golden
    from test_periodic import fluid_compare
    B.build_examples()
    exe = os.path.join(ROOT, "freelb_b200", "cpp", "_build", "periodic3d_b200")
    g = golden("periodic_bgk_f32_n12_s30")
    ni, tau, ulid, steps = (float(v) for v in g["params"])
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        r = subprocess.run([exe, str(int(ni)), str(tau), str(ulid), str(int(steps)), out],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        pops = np.fromfile(out, dtype=np.float64).astype(np.float32)
    assert fluid_compare(g, pops, int(ni), np.float32) < 1e-5


EXAMPLE_INI = """[parallel]
thread_num = {threads}
[Mesh]
Ni = 20
Nj = 18
Nk = 16
Cell_Len = 1
BlockCellLen = 10
[Physical_Property]
rho_ref = 0.001
Kine_Visc = 0.01
[Init_Conditions]
U_Ini0 = 0
U_Ini1 = 0
U_Ini2 = 0
U_Max = 0.1
[Boundary_Conditions]
Velo_Wall0 = 0.1
Velo_Wall1 = 0
Velo_Wall2 = 0
[LB]
RT = 0.56
[Simulation_Settings]
TotalStep = 120
OutputStep = 40
[tolerance]
tol = 1e-12
"""


def _run_in(exe, d, env=None):
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = os.path.join(d, "vtkoutput", "vtidata")
    return {f: os.path.join(out, f) for f in sorted(os.listdir(out))}


def _assemble(files, prefix, dtypes):
    """The DataArrays of the block files `prefix`_B<k>.vti placed into the
    global stored mesh by each file's Origin (unit spacing): {name: array of
    shape (nz, ny, nx, ncomp)}.  Cells two blocks share (their overlap layers)
    must carry the same value in both."""
    import re
    from oracle import oracle as O
    pieces = []
    for name, path in files.items():
        if not re.fullmatch(re.escape(prefix) + r"_B\d+\.vti", name):
            continue
        head = open(path).read(400)
        ext = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', head).group(1).split()]
        org = [float(v) for v in re.search(r'Origin="([^"]+)"', head).group(1).split()]
        arrays = {k: O.vtk_decode(v[2], dtypes[k]).reshape(ext[5] + 1, ext[3] + 1, ext[1] + 1, v[1])
                  for k, v in O.vtk_arrays(path).items()}
        pieces.append((org, arrays))
    assert pieces, prefix
    lo = [min(p[0][a] for p in pieces) for a in range(3)]
    shape = {}
    for org, arrays in pieces:
        off = [int(round(org[a] - lo[a])) for a in range(3)]
        for k, v in arrays.items():
            end = (off[2] + v.shape[0], off[1] + v.shape[1], off[0] + v.shape[2], v.shape[3])
            shape[k] = tuple(max(x, y) for x, y in zip(shape.get(k, end), end))
    out = {k: np.full(sh, np.nan) for k, sh in shape.items()}
    for org, arrays in pieces:
        off = [int(round(org[a] - lo[a])) for a in range(3)]
        for k, v in arrays.items():
            dst = out[k][off[2]:off[2] + v.shape[0], off[1]:off[1] + v.shape[1],
                         off[0]:off[0] + v.shape[2]]
            seen = ~np.isnan(dst)
            assert np.array_equal(dst[seen], v[seen].astype(np.float64)), (prefix, k)
            dst[...] = v
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32", 1e-5)])
@pytest.mark.parametrize("threads", [1, 2])
def test_reference_example_output_equals_reference_build(gpu_ok, precision, tol, threads):
    """examples/cavity3d/cavity3d.cpp built twice from the same untouched source,
    against the reference's own headers (CPU, oracle/_ref) and against the host
    classes (GPU), run on the same ini: ConvertFromRT and the unit conversion,
    the ini reader, geometry and flags, the moving-lid field, the step loop with
    NormalCommunicate, rhoU, getToleranceU and the vtmo writers all meet in the
    .vtm / .vti files of steps 0, 40, 80 and 120.  The flag field must be
    identical and the physRho and physVelocity arrays agree to 1e-12 (FLOAT
    double) / 1e-5 (FLOAT float) relative max-norm on every stored cell.  With
    thread_num = 1 both runs write one block and the flag and .vtm files are
    identical byte for byte; with thread_num = 2 the reference splits the
    domain into two OpenMP blocks and the device run keeps one, so the
    reference's block files are assembled into the global mesh first."""
    from freelb_b200 import build as B
    ours = B.ref_program_path("example" if precision == "f64" else "example_f32")
    ref = os.path.join(ROOT, "oracle", "_ref", f"ref_example_cavity3d_{precision}")
    if not (os.path.exists(ours) and os.path.exists(ref)):
        pytest.skip("reference example not built (no reference sources at build)")
    dt = np.float64 if precision == "f64" else np.float32
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        for d in (d1, d2):
            open(os.path.join(d, "cavity3d.ini"), "w").write(EXAMPLE_INI.format(threads=threads))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        a = _run_in(ours, d1)
        b = _run_in(ref, d2, env)
        if threads == 1:
            assert sorted(a) == sorted(b)
            for name in a:
                if name.startswith("GeoFlag") or name.endswith(".vtm"):
                    assert open(a[name], "rb").read() == open(b[name], "rb").read(), name
        fa = _assemble(a, "GeoFlag", {"flag": np.uint8})
        fb = _assemble(b, "GeoFlag", {"flag": np.uint8})
        assert np.array_equal(fa["flag"], fb["flag"])
        dts = {"physRho": dt, "physVelocity": dt}
        for step in (0, 40, 80, 120):
            A = _assemble(a, f"cavity3d_T{step}", dts)
            R = _assemble(b, f"cavity3d_T{step}", dts)
            assert sorted(A) == sorted(R) == ["physRho", "physVelocity"], step
            for k in A:
                assert A[k].shape == R[k].shape and not np.isnan(R[k]).any(), (step, k)
                err = rel_maxnorm(A[k], R[k])
                assert err < tol, (step, k, err)
