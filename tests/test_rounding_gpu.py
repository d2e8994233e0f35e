"""Rounding of FP16S stores: round to nearest and stochastic rounding (the
sm_100a cvt.rs conversion), checked against one FP64 step of the oracle from
the same binary16 state.  Round to nearest stays within half a unit in the last
place (ulp) of every stored deviation; stochastic rounding stays within one ulp,
rounds away from the nearest value for about a quarter of them, and is
unbiased (mean error far below the ulp).  The mode is per handle, defaults to
stochastic for MRT only, and both modes are
deterministic (the random bits come from the cell's own inputs)."""
import numpy as np
import pytest

import freelb_b200 as F
from freelb_b200 import _capi as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu

W32 = O.W.astype(np.float32).astype(np.float64)
# MRT rates per moment (rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww,
# piww, pxy, pyz, pxz, mx, my, mz; shear entries are replaced by 1/tau): one
# rate for every other moment runs the two-rate form, these the general form
GENERAL_RATES = [0, 1.1, 1.3, 0, 1.25, 0, 1.25, 0, 1.25, 1, 1.4, 1, 1.4, 1, 1, 1, 1.5, 1.5, 1.5]


def ulp16(x):
    """Unit in the last place of binary16 at |x| (subnormal spacing below 2^-14)."""
    ax = np.abs(x)
    e = np.floor(np.log2(np.maximum(ax, 2.0 ** -14)))
    return 2.0 ** (e - 10)


def one_step_errors(model, mode, shape=(32, 12, 12), seed=5, rates=1.2):
    """Stored deviations H = (f - w) 2^10 after one FP16S step from a random
    binary16 state, in ulps of the FP64 oracle's H from the same state."""
    nx, ny, nz = shape
    N = nx * ny * nz
    rng = np.random.default_rng(seed)
    h0 = (2.0 * rng.standard_normal((19, N))).astype(np.float16).astype(np.float64)
    # |H| >= 1/16 or 0: w + H / 2^10 is then exact in FP32 (w = 1/3 included)
    h0[np.abs(h0) < 1.0 / 16] = 0.0
    f0 = (W32[:, None] + h0 / 1024.0).reshape(-1)
    flags = np.full(N, 2, dtype=np.uint8)
    lat = F.Lattice(nx, ny, nz, 0.56, storage="fp16s", model=model, smagorinsky=0.12,
                    mrt_rate=rates)
    lat.set_rounding(mode)
    lat.upload_flags(flags)
    lat.upload_pops(f0.astype(np.float32))
    lat.step(1)
    fd = lat.download_pops(np.float32).astype(np.float64).reshape(19, N)
    lat.close()
    ref = O.Lattice(nx, ny, nz, flags, model=model, tau=0.56, cs=0.12, mrt_rate=rates,
                    dtype=np.float64)
    ref.pops[:] = f0
    ref.step(1)
    hd = (fd - W32[:, None]) * 1024.0
    hx = (ref.pops.reshape(19, N) - W32[:, None]) * 1024.0
    sel = np.abs(hx) >= 1.0  # FP32 arithmetic error << 1 ulp here
    return ((hd - hx) / ulp16(hx))[sel]


@pytest.mark.parametrize("model", ["bgk", "mrt", "mrt_general", "les"])
def test_nearest_is_within_half_an_ulp(gpu_ok, model):
    """Also pins both FP16S MRT forms (two-rate and general) to the FP64
    oracle: their FP32 arithmetic stays far inside half an ulp."""
    if model == "mrt_general":
        e = one_step_errors("mrt", "nearest", rates=GENERAL_RATES)
    else:
        e = one_step_errors(model, "nearest")
    assert e.size > 20000
    assert np.max(np.abs(e)) < 0.51, np.max(np.abs(e))


@pytest.mark.parametrize("model", ["bgk", "mrt", "mrt_general", "les"])
def test_stochastic_is_within_one_ulp_and_unbiased(gpu_ok, model):
    if model == "mrt_general":
        e = one_step_errors("mrt", "stochastic", rates=GENERAL_RATES)
    else:
        e = one_step_errors(model, "stochastic")
    assert e.size > 20000
    assert np.max(np.abs(e)) < 1.01, np.max(np.abs(e))
    away = np.mean(np.abs(e) > 0.51)  # rounded away from the nearest value
    assert 0.18 < away < 0.32, away
    assert abs(np.mean(e)) < 4 * 0.41 / np.sqrt(e.size), np.mean(e)


def test_modes_and_defaults(gpu_ok):
    assert F.cavity(10, storage="fp16s", model="mrt").rounding() == "stochastic"
    assert F.cavity(10, storage="fp16s", model="bgk").rounding() == "nearest"
    assert F.cavity(10, storage="fp16s", model="les").rounding() == "nearest"
    assert F.cavity(10, storage="fp32", model="mrt").rounding() == "nearest"  # FP16S only
    lat = F.cavity(10, storage="fp16s", model="bgk")
    lat.set_rounding("stochastic")
    assert lat.rounding() == "stochastic"
    lat.set_rounding("default")
    assert lat.rounding() == "nearest"
    with pytest.raises(F.FlbError):
        C.call("flb_set_rounding", lat._h, 7)
    les = F.cavity(10, storage="fp16s", model="les")
    les.set_rounding("stochastic")
    assert les.rounding() == "stochastic"


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
def test_stochastic_runs_are_reproducible_and_differ_from_nearest(gpu_ok, model):
    """The random bits are a function of the state: two runs give the same
    bits, CUDA-graph replay gives the plain launches' bits, and the two modes
    give different states."""
    runs = []
    for mode, graph in (("stochastic", False), ("stochastic", True), ("nearest", False)):
        lat = F.cavity(30, tau=0.55, storage="fp16s", model=model)
        lat.set_rounding(mode)
        lat.step(40, graph=graph)
        runs.append(lat.download_pops())
        assert lat.nonfinite() == 0
    assert np.array_equal(runs[0], runs[1])
    assert not np.array_equal(runs[0], runs[2])
