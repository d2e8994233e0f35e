"""The C++17 host classes (freelb_b200/cpp/freelb.h): reference programs compile
against them unchanged, and the example program runs the cavity on the GPU."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, rel_maxnorm

REF_BENCH = "/root/reference/benchmarks/cavity3d/cavity3d.cpp"
REF_BENCH_CU = "/root/reference/benchmarks/cavity3d_cu/cavity3d.cu"
REF_EXAMPLE = "/root/reference/examples/cavity3d/cavity3d.cpp"
INC = os.path.join(ROOT, "freelb_b200", "cpp")
LIBDIR = os.path.join(ROOT, "freelb_b200")
# the reference's own benchmark programs built against the host classes (here,
# where their sources are); the GPU tests run whichever of them exist
REF_PROGRAMS = {"cpu": os.path.join(INC, "_build", "ref_cavity3d"),
                "cu": os.path.join(INC, "_build", "ref_cavity3d_cu"),
                "example": os.path.join(INC, "_build", "ref_example_cavity3d")}


def _gxx(args):
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    return subprocess.run(["g++", "-std=c++17", "-O1"] + args, capture_output=True, text=True,
                          env=env)


@pytest.mark.skipif(not os.path.exists(REF_BENCH), reason="reference sources not present")
def test_reference_benchmark_compiles_unchanged_against_host_classes():
    """benchmarks/cavity3d/cavity3d.cpp, untouched, with only the include path
    changed, compiles and links against libflb_b200.so."""
    exe = REF_PROGRAMS["cpu"]
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    r = _gxx(["-I" + INC, REF_BENCH, "-L" + LIBDIR, "-lflb_b200", "-Wl,-rpath,$ORIGIN/../..",
              "-o", exe])
    assert r.returncode == 0, r.stderr[-3000:]
    assert os.path.exists(exe)


@pytest.mark.skipif(not os.path.exists(REF_BENCH_CU), reason="reference sources not present")
def test_reference_cuda_benchmark_compiles_unchanged_against_host_classes():
    """benchmarks/cavity3d_cu/cavity3d.cu (CuDevApplyCellDynamics / CuDevStream,
    cudev::Cell, copyToDevice), untouched, compiles with nvcc and links against
    libflb_b200.so with only the include path changed."""
    exe = REF_PROGRAMS["cu"]
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I" + INC, REF_BENCH_CU, "-L" + LIBDIR, "-lflb_b200",
                        "-Xlinker", "-rpath,$ORIGIN/../..", "-o", exe],
                       capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    assert os.path.exists(exe)


@pytest.mark.skipif(not os.path.exists(REF_EXAMPLE), reason="reference sources not present")
def test_reference_cavity3d_example_compiles_unchanged_against_host_classes():
    """examples/cavity3d/cavity3d.cpp (post-stream bounce-back managers, vtmo
    writers, getToleranceU, NormalCommunicate, the MPI rank guards), untouched,
    compiles and links against the host classes."""
    exe = REF_PROGRAMS["example"]
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    r = _gxx(["-I" + INC, REF_EXAMPLE, "-L" + LIBDIR, "-lflb_b200", "-Wl,-rpath,$ORIGIN/../..",
              "-o", exe])
    assert r.returncode == 0, r.stderr[-3000:]


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
@pytest.mark.parametrize("kind", ["cpu", "cu", "example"])
def test_reference_benchmark_programs_run_on_gpu(gpu_ok, kind):
    """The reference's cavity3d programs (the CPU and CUDA benchmarks and the
    cavity3d example), built unchanged against the host classes, run their main
    loop on the GPU."""
    exe = REF_PROGRAMS[kind]
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
