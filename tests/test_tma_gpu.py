"""The FP16S bulk-copy kernel (k_pull_tma, launch ctas_per_sm = -2 / -3): the
sources of each tile are staged in shared memory by bulk asynchronous copies
and collided there.  It must give the direct kernel's bits on every cell, for
every model, on lattices whose tiles fall across row ends, padding and the
unstaged tiles near the first and last planes; its bounded waits must report a
wait that gave up through flb_device_status, and leave the handle usable."""
import numpy as np
import pytest

import freelb_b200 as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def pair(make, steps, mode, rounding="default"):
    """The same lattice stepped by the direct kernel and by the bulk-copy kernel."""
    a, b = make(), make()
    a.set_rounding(rounding)
    b.set_rounding(rounding)
    a.set_launch(1, 0, 4)
    b.set_launch(4, mode, 4)
    a.step(steps)
    b.step(steps)
    b.device_status()
    return a, b


@pytest.mark.parametrize("rounding", ["nearest", "stochastic"])
@pytest.mark.parametrize("mode", [-2, -3])
@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
@pytest.mark.parametrize("ni", [22, 30, 62])
def test_tma_equals_direct_kernel_on_cavity(gpu_ok, model, ni, mode, rounding):
    a, b = pair(lambda: F.cavity(ni, tau=0.55, storage="fp16s", model=model), 25, mode,
                rounding)
    assert np.array_equal(a.download_pops(), b.download_pops())


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
@pytest.mark.parametrize("dims", [(23, 11, 40), (24, 30, 19), (40, 9, 30), (31, 17, 25)])
def test_tma_equals_direct_kernel_on_random_flags(gpu_ok, model, dims):
    """Every op and flag value (random first-match task list), perturbed
    populations and fields; pitch - nx from 0 to 1 (rows ending right before
    the next row or one half short of it)."""
    nx, ny, nz = dims
    N = nx * ny * nz
    rng = np.random.default_rng(nx + 7 * ny + 31 * nz)
    flags = rng.choice(np.array([1, 2, 4, 8, 16, 2 | 16, 32], dtype=np.uint8), size=N,
                       p=[.1, .5, .1, .1, .1, .05, .05])
    tasks = ((2, "bulk"), (4, "bounceback"), (8, "movingwall"), (16, "field_bgk"))
    w = np.repeat(O.W, N)
    pops = (w * (1 + 0.05 * rng.standard_normal(19 * N))).astype(np.float32)
    rho = (1 + 0.01 * rng.standard_normal(N)).astype(np.float32)
    u = (0.03 * rng.standard_normal(3 * N)).astype(np.float32)

    def make():
        lat = F.Lattice(nx, ny, nz, 0.57, storage="fp16s", model=model, smagorinsky=0.15,
                        mrt_rate=1.1, tasks=tasks)
        lat.upload_flags(flags)
        lat.upload_pops(pops)
        lat.upload_field("rho", rho)
        lat.upload_field("u", u)
        return lat

    for rounding in ("nearest", "stochastic"):
        a, b = pair(make, 9, -2, rounding)
        assert np.array_equal(a.download_pops(), b.download_pops())


@pytest.mark.parametrize("rounding", ["nearest", "stochastic"])
def test_tma_equals_direct_kernel_general_mrt(gpu_ok, rounding):
    """MRT whose non-shear rates differ runs the general moment form (the
    two-rate form needs one rate for all of them): the same bits in both
    kernels, from perturbed populations with bounce-back cells."""
    nx, ny, nz = 32, 24, 30
    N = nx * ny * nz
    rng = np.random.default_rng(11)
    flags = np.full(N, 2, dtype=np.uint8)
    flags[::7] = 4
    pops = (np.repeat(O.W, N) * (1 + 0.05 * rng.standard_normal(19 * N))).astype(np.float32)
    rates = [0, 1.1, 1.3, 0, 1.25, 0, 1.25, 0, 1.25, 1, 1.4, 1, 1.4, 1, 1, 1, 1.5, 1.5, 1.5]

    def make():
        lat = F.Lattice(nx, ny, nz, 0.55, storage="fp16s", model="mrt", mrt_rate=rates)
        lat.upload_flags(flags)
        lat.upload_pops(pops)
        return lat

    a, b = pair(make, 20, -2, rounding)
    assert np.array_equal(a.download_pops(), b.download_pops())


def test_tma_graph_and_autotune(gpu_ok):
    """CUDA-graph replay of the bulk-copy kernel equals plain launches; the
    autotuner times it among the candidates."""
    a = F.cavity(62, storage="fp16s")
    b = F.cavity(62, storage="fp16s")
    a.set_launch(4, -3, 4)
    b.set_launch(4, -3, 4)
    a.step(8, graph=True)
    b.step(8)
    assert np.array_equal(a.download_pops(), b.download_pops())
    c = F.cavity(62, storage="fp16s")
    (ty, ctas, v), ms, taken = c.autotune(trial_steps=1)
    assert ms > 0 and taken > 0
    c.device_status()


def test_tma_launch_rules(gpu_ok):
    with pytest.raises(F.FlbError):   # FP32 storage: not built
        F.cavity(30).set_launch(4, -2, 4)
    with pytest.raises(F.FlbError):   # rows not 16-byte aligned (pitch 52 halves)
        F.cavity(48, storage="fp16s").set_launch(4, -2, 4)
    with pytest.raises(F.FlbError):   # 2 cells per thread
        F.cavity(30, storage="fp16s").set_launch(4, -2, 2)
    with pytest.raises(F.FlbError):
        F.cavity(30, storage="fp16s").set_wait_limit(-1.0)


def test_tma_wait_that_gives_up_is_reported_and_the_handle_recovers(gpu_ok):
    """A tile whose stage is never signalled (the test hook withholds it): its
    consumers' waits run out after the 50 ms limit, the producer's wait for
    that stage too, the kernel ends early (the step is incomplete) and the
    status reads FLB_ERR_TIMEOUT once.  With the hook off and the state
    re-uploaded, the handle steps exactly like the direct kernel."""
    ni, steps = 62, 6
    ref = F.cavity(ni, tau=0.55, storage="fp16s")
    ref.set_launch(1, 0, 4)
    ref.step(steps)
    lat = F.cavity(ni, tau=0.55, storage="fp16s")
    start = lat.download_pops(np.float64)
    lat.set_launch(4, -2, 4)
    lat.set_wait_limit(0.05)
    lat.device_status()
    F._capi.call("flb_test_withhold_tile", lat._h, 150)   # a staged tile of CTA 2
    lat.step(1)
    with pytest.raises(F.FlbError) as e:
        lat.device_status()
    assert e.value.code == -4          # FLB_ERR_TIMEOUT
    lat.device_status()                # cleared
    F._capi.call("flb_test_withhold_tile", lat._h, -1)
    lat.set_wait_limit(2.0)
    lat.upload_pops(start)
    lat.step(steps)
    lat.device_status()
    assert np.array_equal(lat.download_pops(), ref.download_pops())
