"""GPU tests of multi-block lattices: device halo exchange (uneven blocks of
one cavity), the batched ensemble of independent cavities, launch-shape
control, the autotuner and CUDA-graph stepping."""
import numpy as np
import pytest

import freelb_b200 as F
from conftest import golden, rel_maxnorm
from freelb_b200 import geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gpu_blocks(ni, blocks, storage="fp32", tau=0.53, ulid=0.1, model="bgk"):
    n = ni + 2
    flags = F.cavity_flags(ni)
    lat = F.Lattice.blocks(G.block_tuples(blocks), tau, mode="halo", storage=storage,
                           model=model)
    real = lat.real
    u = np.zeros((n ** 3, 3), dtype=real)
    u[flags == 8, 0] = real(ulid)
    for k, b in enumerate(blocks):
        lat.upload_flags(G.slice_block(flags, n, b), block=k)
        lat.upload_field("u", G.slice_block(u, n, b, comps=3), block=k)
    return lat


@pytest.mark.parametrize("name", ["blocks_bgk_f64_n12_s30", "blocks_bgk_f32_n12_s30"])
def test_blocks_match_reference_multiblock_golden(gpu_ok, name):
    g = golden(name)
    ni, _, _, steps, seed = g["params"]
    blocks = G.uneven_blocks(int(ni), edges=tuple(int(e) for e in g["edges"]), seed=int(seed))
    storage = "fp64" if "f64" in name else "fp32"
    lat = gpu_blocks(int(ni), blocks, storage)
    assert lat.halo_count() > 0
    lat.step(int(steps))
    lat.compute_rhou(2)
    tol = 1e-12 if storage == "fp64" else 1e-5
    pops = np.concatenate([lat.download_pops(block=k) for k in range(len(blocks))])
    ref = np.concatenate([g[f"pops_b{k}"] for k in range(len(blocks))])
    assert rel_maxnorm(pops, ref) < tol
    u = np.concatenate([lat.download_field("u", block=k) for k in range(len(blocks))])
    uref = np.concatenate([g[f"u_b{k}"] for k in range(len(blocks))])
    assert rel_maxnorm(u, uref) < tol
    for k in range(len(blocks)):
        assert np.array_equal(lat.download_flags(block=k), g[f"flags_b{k}"])


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
@pytest.mark.parametrize("tile_y,ctas,vec", [(8, 0, 4), (2, 8, 2), (1, 0, 2), (4, 16, 4)])
def test_blocks_vs_single_block_bitwise_on_fluid(gpu_ok, tile_y, ctas, vec, model):
    """Uneven blocks with device halos reproduce the single-block run exactly on
    fluid cells, for every launch shape and model (MRT in its two-rate form)."""
    ni = 40
    blocks = G.uneven_blocks(ni, edges=(8, 12, 16), seed=5)
    lat = gpu_blocks(ni, blocks, "fp32", model=model)
    lat.set_launch(tile_y, ctas, vec)
    lat.step(40)
    one = F.cavity(ni, model=model)
    one.step(40)
    n = ni + 2
    P = one.download_pops().reshape(19, n, n, n)
    for k, b in enumerate(blocks):
        pb = lat.download_pops(block=k).reshape(19, b["nz"], b["ny"], b["nx"])
        fb = G.slice_block(F.cavity_flags(ni), n, b).reshape(b["nz"], b["ny"], b["nx"])
        ps = P[:, b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"], b["ox"]:b["ox"] + b["nx"]]
        assert np.array_equal(pb[:, fb == 2], ps[:, fb == 2])


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
@pytest.mark.parametrize("tile_y,ctas,vec", [(8, 0, 4), (2, 8, 2), (4, 16, 4)])
def test_fp16s_blocks_vs_single_block_bitwise_on_fluid(gpu_ok, model, tile_y, ctas, vec):
    """FP16S storage: the multi-block tile kernel (32-bit offsets) and the
    single-block kernel give the same bits on fluid cells."""
    ni = 40
    blocks = G.uneven_blocks(ni, edges=(8, 12, 16), seed=7)
    lat = gpu_blocks(ni, blocks, "fp16s", tau=0.55, model=model)
    lat.set_launch(tile_y, ctas, vec)
    lat.step(30)
    one = F.cavity(ni, tau=0.55, storage="fp16s", model=model)
    one.step(30)
    n = ni + 2
    P = one.download_pops().reshape(19, n, n, n)
    for k, b in enumerate(blocks):
        pb = lat.download_pops(block=k).reshape(19, b["nz"], b["ny"], b["nx"])
        fb = G.slice_block(F.cavity_flags(ni), n, b).reshape(b["nz"], b["ny"], b["nx"])
        ps = P[:, b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"], b["ox"]:b["ox"] + b["nx"]]
        assert np.array_equal(pb[:, fb == 2], ps[:, fb == 2]), (model, k)


def test_blocks_vs_oracle_multiblock_fp64(gpu_ok):
    ni = 18
    blocks = G.uneven_blocks(ni, edges=(4, 6, 8), seed=9)
    lat = gpu_blocks(ni, blocks, "fp64", tau=0.56, ulid=0.08)
    mb = O.MultiBlock(blocks, O.cavity_flags(ni), ni + 2, tau=0.56, ulid=0.08, dtype=np.float64)
    lat.step(33)
    mb.step(33)
    ours = np.concatenate([lat.download_pops(block=k) for k in range(len(blocks))])
    ref = np.concatenate([m.pops for m in mb.lats])
    assert rel_maxnorm(ours, ref) < 1e-12


def ensemble(sizes, taus, storage="fp32", ulid=0.1):
    lat = F.Lattice.blocks([(n + 2, n + 2, n + 2, 0, 0, 0, 1.0 / t) for n, t in zip(sizes, taus)],
                           0.6, mode="independent", storage=storage)
    for k, n in enumerate(sizes):
        fl = F.cavity_flags(n)
        u = np.zeros(((n + 2) ** 3, 3), dtype=lat.real)
        u[fl == 8, 0] = lat.real(ulid)
        lat.upload_flags(fl, block=k)
        lat.upload_field("u", u, block=k)
    return lat


@pytest.mark.parametrize("graph", [False, True])
def test_ensemble_each_cavity_matches_single(gpu_ok, graph):
    """Batched independent cavities, each with its own tau, match one-at-a-time runs."""
    rng = np.random.default_rng(1)
    sizes = [int(v) for v in rng.integers(6, 20, size=9)]
    taus = [0.5 + 3 * 0.1 * n / float(np.exp(rng.uniform(np.log(100), np.log(3000))))
            for n in sizes]
    lat = ensemble(sizes, taus)
    lat.step(25, graph=graph)
    for k, (n, t) in enumerate(zip(sizes, taus)):
        ref = O.cavity(n, tau=t, ulid=0.1)
        ref.step(25)
        assert rel_maxnorm(lat.download_pops(block=k), ref.pops) < 1e-5, (k, n, t)


@pytest.mark.parametrize("graph", [False, True])
def test_fp16s_ensemble_each_cavity_equals_single(gpu_ok, graph):
    """FP16S storage: the batched cavities, each with its own tau, give the bits
    of one FP16S handle per cavity (the 32-bit tile kernel against the
    single-block kernel)."""
    rng = np.random.default_rng(2)
    sizes = [int(v) for v in rng.integers(6, 24, size=7)]
    taus = [0.5 + 3 * 0.1 * n / float(np.exp(rng.uniform(np.log(100), np.log(3000))))
            for n in sizes]
    lat = ensemble(sizes, taus, storage="fp16s")
    lat.step(25, graph=graph)
    for k, (n, t) in enumerate(zip(sizes, taus)):
        one = F.cavity(n, tau=t, ulid=0.1, storage="fp16s")
        one.step(25)
        assert np.array_equal(lat.download_pops(block=k), one.download_pops()), (k, n, t)
        one.close()


def test_graph_step_equals_plain_step(gpu_ok):
    a = F.cavity(30)
    b = F.cavity(30)
    a.step(17)
    b.step(17, graph=True)
    assert np.array_equal(a.download_pops(), b.download_pops())
    a.step(4, graph=True)
    b.step(4)
    assert np.array_equal(a.download_pops(), b.download_pops())


@pytest.mark.parametrize("storage", ["fp32", "fp16s", "fp64"])
def test_autotune_keeps_results_exact(gpu_ok, storage):
    a = F.cavity(36, storage=storage)
    b = F.cavity(36, storage=storage)
    (ty, c, v), ms, taken = a.autotune(trial_steps=2)
    assert ty in (1, 2, 4, 8) and c in (-3, -2, -1, 0, 8, 16, 32) and ms > 0 and taken > 0
    assert c >= 0 or storage == "fp16s"
    assert v in ((1, 2) if storage == "fp64" else (2, 4))
    assert a.get_launch() == (ty, c, v)
    b.step(taken)
    a.step(5)
    b.step(5)
    assert np.array_equal(a.download_pops(), b.download_pops())


def test_set_launch_rejects_bad_shapes(gpu_ok):
    a = F.cavity(8)
    with pytest.raises(F.FlbError):
        a.set_launch(3, 0)
    with pytest.raises(F.FlbError):
        a.set_launch(8, -1)
    with pytest.raises(F.FlbError):
        a.set_launch(8, 0, 1)     # FP32 builds 2 or 4 cells per thread


@pytest.mark.parametrize("storage,vec", [("fp32", 2), ("fp32", 4), ("fp16s", 2), ("fp16s", 4),
                                         ("fp64", 1), ("fp64", 2)])
def test_every_vector_width_matches_oracle(gpu_ok, storage, vec):
    lat = F.cavity(21, tau=0.55, storage=storage)
    lat.set_launch(4, 0, vec)
    lat.step(30)
    ref = O.cavity(21, tau=0.55, dtype=np.float64 if storage == "fp64" else np.float32)
    ref.step(30)
    tol = {"fp32": 1e-5, "fp64": 1e-12, "fp16s": 2e-3}[storage]
    assert rel_maxnorm(lat.download_pops(), ref.pops) < tol


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
@pytest.mark.parametrize("storage,widths", [("fp32", (2, 4)), ("fp16s", (2, 4)), ("fp64", (1, 2)),
                                            ("fp32s", (2, 4))])
@pytest.mark.parametrize("ni", [21, 30])
def test_vector_widths_are_bitwise_equal(gpu_ok, storage, widths, ni, model):
    """Every cell's update is the same function of its 19 sources whatever the
    cells per thread or launch shape (direct, persistent tile kernel), so they
    agree bit for bit (ragged rows and row ends included): the autotuner's pick
    never changes a result."""
    out = []
    for v in widths:
        for shape in ((2, 0, v), (8, 16, v)):
            lat = F.cavity(ni, tau=0.55, storage=storage, model=model)
            lat.set_launch(*shape)
            lat.step(25)
            out.append(lat.download_pops())
    for o in out[1:]:
        assert np.array_equal(out[0], o)


@pytest.mark.parametrize("storage,tol", [("fp64", 1e-12), ("fp32", 1e-5), ("fp16s", 2e-3)])
def test_full_halo_matches_oracle(gpu_ok, storage, tol):
    """flb_set_halo_mode(FULL): all 19 populations of every overlap cell from its
    owner (NormalFullCommunicate / NormalAllCommunicate), against the oracle's
    restatement (itself pinned to the reference's run)."""
    ni, steps = 16, 20
    blocks = G.uneven_blocks(ni, edges=(4, 6, 8), seed=3)
    lat = gpu_blocks(ni, blocks, storage)
    normal = lat.halo_count()
    lat.set_halo_mode("full")
    assert lat.halo_count() > normal
    lat.step(steps)
    dt = np.float32 if storage == "fp32" else np.float64  # FP16S against FP64
    mb = O.MultiBlock(blocks, O.cavity_flags(ni), ni + 2, dtype=dt, full=True)
    mb.step(steps)
    pops = np.concatenate([lat.download_pops(block=k) for k in range(len(blocks))])
    want = np.concatenate([mb.lats[k].pops for k in range(len(blocks))])
    assert rel_maxnorm(pops, want) < tol
    lat.set_halo_mode("normal")
    assert lat.halo_count() == normal
