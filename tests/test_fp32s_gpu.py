"""FP32S storage on the GPU: populations kept as FP32 deviations d_i = f_i -
rho0 w_i and collided as stored (the FP16S deviation form at FP32 width).

FP32S has no reference counterpart to match bit for bit: its bar is the FP64
run of the same step (the reference's own FP64 path through the golden
fixtures, or the FP64 oracle), where it must beat FP32 storage of f.  Inside
the library it must behave like every other storage: multi-block handles equal
the single-block run bit for bit on fluid cells and the transfers convert the
deviations (the post-stream bounce-back managers are covered in
test_boundary_gpu.py, the adjoint in test_adjoint_gpu.py).
"""
import numpy as np
import pytest

import freelb_b200 as F
from conftest import golden, rel_l2, rel_maxnorm
from freelb_b200 import geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
def test_fp32s_against_reference_fp64_golden(gpu_ok, model):
    """10^3 cavity, 40 steps: FP32S is closer to the reference's FP64 run than
    FP32 storage is, and within 1e-6 (relative max-norm) on every cell."""
    g = golden(f"cavity_{model}_f64_n10_s40")
    ni, tau, ulid, steps, cs = g["params"]
    err = {}
    for storage in ("fp32s", "fp32"):
        lat = F.cavity(int(ni), tau=tau, ulid=ulid, storage=storage, model=model, smagorinsky=cs)
        lat.step(int(steps))
        rho, u = lat.rhou(key=2, dtype=np.float64)
        assert np.array_equal(lat.download_flags(), g["flags"])
        err[storage] = (rel_maxnorm(lat.download_pops(np.float64), g["pops"]),
                        rel_maxnorm(rho, g["rho"]), rel_maxnorm(u, g["u"]))
    assert max(err["fp32s"]) < 1e-6, err
    assert err["fp32s"][2] < err["fp32"][2], err


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
def test_fp32s_velocity_error_vs_fp64(gpu_ok, model):
    """48^3 cavity, 600 steps: relative L2 velocity error against the FP64 run
    of the same kernel, FP32S against FP32 storage of f."""
    tau = 0.53 if model != "les" else 0.51
    us = {}
    for storage in ("fp64", "fp32s", "fp32"):
        lat = F.cavity(48, tau=tau, ulid=0.1, storage=storage, model=model)
        lat.step(600)
        _, u = lat.rhou(key=2, dtype=np.float64)
        us[storage] = u
        assert lat.nonfinite() == 0
    e32s = rel_l2(us["fp32s"], us["fp64"])
    e32 = rel_l2(us["fp32"], us["fp64"])
    assert e32s < 1e-5, (e32s, e32)
    assert e32s < 0.25 * e32, (e32s, e32)


@pytest.mark.parametrize("model", ["bgk", "mrt", "les", "brinkman"])
def test_fp32s_random_flags_against_fp64_oracle(gpu_ok, model):
    """Every op (bulk, bounce-back, moving wall, field-velocity BGK, none) on a
    non-cubic mesh with a random first-match task list, against the FP64
    oracle from the same perturbed state."""
    nx, ny, nz = 37, 9, 11
    N = nx * ny * nz
    rng = np.random.default_rng(17)
    flags = rng.choice(np.array([1, 2, 4, 8, 16, 2 | 16, 32], dtype=np.uint8), size=N,
                       p=[.1, .5, .1, .1, .1, .05, .05])
    keys, ops = (2, 4, 8, 16), ("bulk", "bounceback", "movingwall", "field_bgk")
    tasks = tuple(zip(keys, ops))
    lat = F.Lattice(nx, ny, nz, 0.57, storage="fp32s", model=model, smagorinsky=0.15,
                    mrt_rate=1.1, tasks=tasks)
    ref = O.Lattice(nx, ny, nz, flags, model=model, tau=0.57, cs=0.15, mrt_rate=1.1,
                    dtype=np.float64, keys=keys,
                    ops=(O.OP_BULK, O.OP_BB, O.OP_MBB, O.OP_FIELD_BGK))
    pops0 = (ref.pops.reshape(19, N) * (1 + 0.02 * rng.standard_normal((19, N)))).reshape(-1)
    ref.pops[:] = pops0
    ref.rho[:] = 1 + 0.01 * rng.standard_normal(N)
    ref.u[:] = 0.03 * rng.standard_normal(3 * N)
    lat.upload_flags(flags)
    lat.upload_pops(pops0)
    lat.upload_field("rho", ref.rho)
    lat.upload_field("u", ref.u)
    if model == "brinkman":
        a = rng.uniform(0.0, 0.05, size=N)
        ref.set_alpha(a)
        lat.upload_field("alpha", a)
    lat.step(7)
    ref.step(7)
    assert rel_maxnorm(lat.download_pops(np.float64), ref.pops) < 1e-6


def test_fp32s_pops_roundtrip_and_conservation(gpu_ok):
    """Uploads store f - rho0 w and downloads add it back: FP32 host values in
    [w/2, 2w] come back bit for bit (both subtractions are exact there); the
    FP64 mass and momentum sums add the shift in FP64."""
    nx, ny, nz = 45, 7, 6
    N = nx * ny * nz
    rng = np.random.default_rng(3)
    w = np.repeat(O.W, N)
    p = (w * (1 + np.clip(0.1 * rng.standard_normal(19 * N), -0.45, 0.45))).astype(np.float32)
    lat = F.Lattice(nx, ny, nz, 0.6, storage="fp32s")
    lat.upload_pops(p)
    assert np.array_equal(lat.download_pops(np.float32), p)
    p64 = w * (1 + 0.05 * rng.standard_normal(19 * N))
    lat.upload_pops(p64)
    back = lat.download_pops(np.float64)
    # the deviation is rounded once, to FP32
    assert np.max(np.abs(back - p64)) <= np.max(np.abs(p64 - w)) * 2.0 ** -24 * 1.01
    lat.upload_flags(np.full(N, 2, dtype=np.uint8))
    s = lat.conservation(key=2)
    # the sums over the reference's post-stream state (download order)
    P = back.reshape(19, N)
    assert abs(s[0] - P.sum()) < 1e-9
    assert abs(s[1] - (O.C[:, 0:1] * P).sum()) < 1e-9


@pytest.mark.parametrize("tile_y,ctas,vec", [(8, 0, 4), (2, 8, 2), (4, 16, 4)])
def test_fp32s_blocks_vs_single_block_bitwise_on_fluid(gpu_ok, tile_y, ctas, vec):
    """Uneven blocks with device halos give the single-block run's bits on
    fluid cells (the halo copies move deviations as stored)."""
    ni = 40
    blocks = G.uneven_blocks(ni, edges=(8, 12, 16), seed=11)
    n = ni + 2
    flags = F.cavity_flags(ni)
    lat = F.Lattice.blocks(G.block_tuples(blocks), 0.55, mode="halo", storage="fp32s")
    u = np.zeros((n ** 3, 3), dtype=np.float32)
    u[flags == 8, 0] = np.float32(0.1)
    for k, b in enumerate(blocks):
        lat.upload_flags(G.slice_block(flags, n, b), block=k)
        lat.upload_field("u", G.slice_block(u, n, b, comps=3), block=k)
    lat.set_launch(tile_y, ctas, vec)
    lat.step(30)
    one = F.cavity(ni, tau=0.55, storage="fp32s")
    one.step(30)
    P = one.download_pops().reshape(19, n, n, n)
    for k, b in enumerate(blocks):
        pb = lat.download_pops(block=k).reshape(19, b["nz"], b["ny"], b["nx"])
        fb = G.slice_block(flags, n, b).reshape(b["nz"], b["ny"], b["nx"])
        ps = P[:, b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"], b["ox"]:b["ox"] + b["nx"]]
        assert np.array_equal(pb[:, fb == 2], ps[:, fb == 2]), k


def test_fp32s_graph_and_autotune(gpu_ok):
    """CUDA-graph stepping and the autotuner cover FP32S like FP32."""
    a = F.cavity(30, storage="fp32s")
    b = F.cavity(30, storage="fp32s")
    (ty, c, v), ms, taken = a.autotune(trial_steps=1)
    assert v in (2, 4) and ms > 0
    b.set_launch(ty, c, v)
    b.step(taken)
    a.step(6, graph=True)
    b.step(6)
    assert np.array_equal(a.download_pops(), b.download_pops())
