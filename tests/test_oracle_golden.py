"""CPU tests: pin the oracle restatement (oracle/flb_oracle.c) to the reference.

The golden fixtures are outputs of the reference's own CPU path
(tests/golden/make_golden.py).  When the reference harness is built
(oracle/_ref, only where the reference sources exist) the restatement is also
checked against live reference runs.
"""
import numpy as np
import pytest

from conftest import golden, rel_maxnorm
from oracle import oracle as O

SMALL = ["cavity_bgk_f32_n10_s40", "cavity_bgk_f64_n10_s40", "cavity_les_f32_n10_s40",
         "cavity_les_f64_n10_s40", "cavity_mrt_f32_n10_s40", "cavity_mrt_f64_n10_s40",
         "cavity_bgk_f32_n7_s200"]


def run_oracle(model, ni, tau, ulid, steps, cs, dtype):
    lat = O.cavity(int(ni), model=model, tau=tau, ulid=ulid, cs=cs, dtype=dtype)
    lat.step(int(steps))
    rho, u = lat.rhou_fields()
    return lat, rho, u


@pytest.mark.parametrize("name", SMALL)
def test_restatement_matches_reference_golden(name):
    g = golden(name)
    ni, tau, ulid, steps, cs = g["params"]
    model = str(g["model"])
    dtype = np.float64 if "f64" in name else np.float32
    lat, rho, u = run_oracle(model, ni, tau, ulid, steps, cs, dtype)
    assert np.array_equal(lat.flags, g["flags"]), "flags must be bit-exact"
    tol = 1e-12 if dtype == np.float64 else 1e-5
    assert rel_maxnorm(lat.pops, g["pops"]) < tol
    assert rel_maxnorm(rho, g["rho"]) < tol
    assert rel_maxnorm(u, g["u"]) < tol


def test_restatement_c1_benchmark_shape():
    """100^3 cavity, tau=0.53, u_lid=0.1, 1000 steps (reference cavity3d shape)."""
    g = golden("c1_bgk_f32_n100_s1000")
    lat, rho, u = run_oracle("bgk", 100, 0.53, 0.1, 1000, 0.1, np.float32)
    n = 102
    assert np.array_equal(lat.flags, g["flags"])
    pops = lat.pops.reshape(19, n, n, n)
    sums = pops.astype(np.float64).sum(axis=(1, 2, 3))
    assert np.max(np.abs(sums - g["pop_sums"]) / np.abs(g["pop_sums"])) < 1e-6
    assert rel_maxnorm(pops[:, :, n // 2, :], g["pops_plane"]) < 1e-5
    assert rel_maxnorm(u.reshape(n, n, n, 3)[:, n // 2], g["u_plane"]) < 1e-5
    assert rel_maxnorm(rho.reshape(n, n, n)[:, n // 2], g["rho_plane"]) < 1e-5


@pytest.mark.parametrize("ni", [4, 9, 16])
def test_cavity_flags_restatement(ni):
    """oracle_cavity_flags against the analytic layout, and the product helper."""
    import freelb_b200
    f = O.cavity_flags(ni)
    assert np.array_equal(f, freelb_b200.cavity_flags(ni))
    n = ni + 2
    v = f.reshape(n, n, n)
    assert (v[0] == 1).all() and (v[-1] == 1).all()
    assert (v[n - 2, 2:n - 2, 2:n - 2] == 8).all()
    assert int((f == 2).sum()) == (ni - 2) ** 3


def test_task_lut_first_match():
    lut = O.task_lut([2, 4 | 8, 8], [O.OP_BULK, O.OP_BB, O.OP_MBB])
    assert lut[2] == O.OP_BULK and lut[4] == O.OP_BB
    assert lut[8] == O.OP_BB          # first key sharing a bit wins (tmp.h:283-309)
    assert lut[1] == O.OP_NONE and lut[6] == O.OP_BULK


def test_ps_streaming_is_linear_periodic_shift():
    """With no collision, one step shifts every direction array by Delta_i mod N."""
    nx, ny, nz = 5, 4, 3
    N = nx * ny * nz
    flags = np.ones(N, dtype=np.uint8)
    lat = O.Lattice(nx, ny, nz, flags, dtype=np.float64)
    rng = np.random.default_rng(0)
    lat.pops[:] = rng.random(19 * N)
    before = lat.pops.reshape(19, N).copy()
    lat.step(1)
    after = lat.pops.reshape(19, N)
    for i in range(19):
        d = O.C[i, 0] + O.C[i, 1] * nx + O.C[i, 2] * nx * ny
        assert np.array_equal(after[i], np.roll(before[i], d))


@pytest.mark.skipif(O.ref_binary() is None, reason="reference harness not built here")
@pytest.mark.parametrize("model", ["bgk", "les", "mrt"])
def test_restatement_matches_live_reference(model):
    r = O.run_reference(model, 14, 0.52, 0.08, 60, 0, cs=0.12, dtype=np.float64, threads=2)
    lat, rho, u = run_oracle(model, 14, 0.52, 0.08, 60, 0.12, np.float64)
    assert np.array_equal(lat.flags, r["flags"])
    assert rel_maxnorm(lat.pops, r["pops"]) < 1e-12
    assert rel_maxnorm(u, r["u"]) < 1e-12


def _blocks_from_golden(g):
    from freelb_b200 import geometry as G
    ni, _, _, _, seed = g["params"]
    return G.uneven_blocks(int(ni), edges=tuple(int(e) for e in g["edges"]), seed=int(seed))


@pytest.mark.parametrize("name", ["blocks_bgk_f64_n12_s30", "blocks_bgk_f32_n12_s30"])
def test_multiblock_restatement_matches_reference(name):
    """BlockReader blocks + NormalCommunicate, restated, against the reference run."""
    g = golden(name)
    blocks = _blocks_from_golden(g)
    assert len(blocks) == int(g["nblocks"])
    dtype = np.float64 if "f64" in name else np.float32
    ni = int(g["params"][0])
    mb = O.MultiBlock(blocks, O.cavity_flags(ni), ni + 2, dtype=dtype)
    mb.step(int(g["params"][3]))
    fields = mb.rhou_fields()
    tol = 1e-12 if dtype == np.float64 else 1e-5
    ours = np.concatenate([mb.lats[k].pops for k in range(len(blocks))])
    ref = np.concatenate([g[f"pops_b{k}"] for k in range(len(blocks))])
    assert rel_maxnorm(ours, ref) < tol
    u = np.concatenate([fields[k][1] for k in range(len(blocks))])
    uref = np.concatenate([g[f"u_b{k}"] for k in range(len(blocks))])
    assert rel_maxnorm(u, uref) < tol
    for k in range(len(blocks)):
        assert np.array_equal(mb.lats[k].flags, g[f"flags_b{k}"])


@pytest.mark.skipif(O.ref_binary(np.float64) is None, reason="reference harness not built here")
@pytest.mark.parametrize("comm", ["full", "all"])
def test_full_halo_restatement_matches_reference(comm, tmp_path):
    """NormalFullCommunicate / NormalAllCommunicate (all populations of the
    overlap cells), restated, against the reference's multi-block run."""
    from freelb_b200 import geometry as G
    ni, steps = 16, 20
    blocks = G.uneven_blocks(ni, edges=(4, 6, 8), seed=3)
    bf = str(tmp_path / "blocks.txt")
    G.write_block_file(bf, blocks)
    for dt, tol in ((np.float64, 1e-12), (np.float32, 1e-5)):
        ref = O.run_reference("bgk", ni, 0.53, 0.1, steps, 0, dtype=dt, blockfile=bf, threads=2,
                              comm=comm)
        mb = O.MultiBlock(blocks, O.cavity_flags(ni), ni + 2, dtype=dt, full=True)
        mb.step(steps)
        ours = np.concatenate([mb.lats[k].pops for k in range(len(blocks))])
        want = np.concatenate([ref[f"pops_b{k}"] for k in range(len(blocks))])
        assert rel_maxnorm(ours, want) < tol
    normal = O.MultiBlock(blocks, O.cavity_flags(ni), ni + 2, dtype=np.float32)
    normal.step(steps)
    assert not np.array_equal(np.concatenate([l.pops for l in normal.lats]), ours)


def test_multiblock_equals_single_block_on_fluid_cells():
    from freelb_b200 import geometry as G
    blocks = G.uneven_blocks(16, edges=(4, 6, 8), seed=11)
    mb = O.MultiBlock(blocks, O.cavity_flags(16), 18, dtype=np.float64)
    mb.step(25)
    sb = O.cavity(16, dtype=np.float64)
    sb.step(25)
    P = sb.pops.reshape(19, 18, 18, 18)
    for k, b in enumerate(blocks):
        pb = mb.lats[k].pops.reshape(19, b["nz"], b["ny"], b["nx"])
        fb = mb.lats[k].flags.reshape(b["nz"], b["ny"], b["nx"])
        ps = P[:, b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"], b["ox"]:b["ox"] + b["nx"]]
        assert np.array_equal(pb[:, fb == 2], ps[:, fb == 2])


def test_partition_axis_tiles_exactly():
    import random
    from freelb_b200 import geometry as G
    for seed in range(20):
        p = G.partition_axis(256, (32, 48, 64, 96), random.Random(seed))
        assert sum(p) == 256 and set(p) <= {32, 48, 64, 96}


def test_brinkman_restatement_matches_reference_policy():
    """The Brinkman-forced BGK restated in C against the reference-built policy
    (reference ForcePop + SecondOrder + BGKForce update) in the harness."""
    ni = 10
    a = O.porosity(ni, 7)
    for dt, tol in ((np.float64, 1e-13), (np.float32, 1e-5)):
        if O.ref_binary(dt) is None:
            pytest.skip("reference harness not built here")
        ref = O.run_reference("brinkman", ni, 0.55, 0.1, 40, 0, dtype=dt, alpha=a, threads=2)
        lat = O.cavity(ni, model="brinkman", tau=0.55, ulid=0.1, dtype=dt, alpha=a)
        lat.step(40)
        assert rel_maxnorm(lat.pops, ref["pops"]) < tol


@pytest.mark.skipif(O.ref_binary(np.float64) is None, reason="reference harness not built here")
def test_finite_difference_gradient_of_reference_solver():
    """Central-difference dJ/dalpha of the reference CPU solver (Brinkman policy in
    the harness) equals that of the restatement: the adjoint's FD oracle is pinned."""
    ni, tau, steps, h = 6, 0.6, 25, 1e-4
    a = O.porosity(ni, 2)
    fl = O.cavity_flags(ni)
    c = int(np.flatnonzero(fl == 2)[5])

    def j_ref(al):
        r = O.run_reference("brinkman", ni, tau, 0.1, steps, 0, dtype=np.float64, alpha=al,
                            threads=1)
        lat = O.cavity(ni, model="brinkman", tau=tau, dtype=np.float64, alpha=al)
        lat.pops[:] = r["pops"]
        return lat.objective_u2()

    def j_orc(al):
        lat = O.cavity(ni, model="brinkman", tau=tau, dtype=np.float64, alpha=al)
        lat.step(steps)
        return lat.objective_u2()

    ap, am = a.copy(), a.copy()
    ap[c] += h
    am[c] -= h
    g_ref = (j_ref(ap) - j_ref(am)) / (2 * h)
    g_orc = (j_orc(ap) - j_orc(am)) / (2 * h)
    assert abs(g_ref - g_orc) <= 1e-7 * abs(g_ref)


WALL_KINDS = {1: "normal", 2: "anti_simple", 3: "anti_o1", 4: "anti_o2", 5: "anti_pressure"}


def seeded_fields(n, seed=7):
    """RHO near 1 and small VELOCITY on every cell, so that each kind's
    dependence on the fields is exercised."""
    rng = np.random.default_rng(seed)
    return 1.0 + rng.uniform(-0.02, 0.02, n ** 3), rng.uniform(-0.03, 0.03, (n ** 3, 3))


@pytest.mark.skipif(O.ref_binary(np.float64) is None, reason="reference harness not built here")
@pytest.mark.parametrize("wallkind", sorted(WALL_KINDS))
def test_poststream_bb_restatement_matches_reference_managers(wallkind):
    """oracle.poststream_bb against the reference's own BBLikeFixedBlockBdManager
    applied after Stream(): bounceback::movingwall on the lid and, on the walls,
    bounceback::normal / anti_simple / anti_O1 / anti_O2 / anti_pressure, with
    seeded RHO and VELOCITY fields.  The anti kinds feed the fields back into
    the walls every step and amplify the last-bit differences of the reference
    build's FMA contraction, so the run is kept short."""
    ni, steps = 8, 8
    n = ni + 2
    rho, u = seeded_fields(n)
    for dt, tol in ((np.float64, 1e-12), (np.float32, 1e-5)):
        ref = O.run_reference("bgk", ni, 0.6, 0.1, steps, 0, dtype=dt, threads=2,
                              fields=(rho, u), poststream=wallkind)
        fl = O.cavity_flags(ni)
        lat = O.Lattice(n, n, n, fl, tau=0.6, dtype=dt, keys=(2 | 4 | 8,), ops=(O.OP_BULK,))
        lat.rho[:] = rho.astype(dt)
        lat.u.reshape(-1, 3)[:] = u.astype(dt)
        for _ in range(steps):
            lat.step(1)
            O.poststream_bb(lat, 4, 1, WALL_KINDS[wallkind])
            O.poststream_bb(lat, 8, 1, "movingwall")
        assert rel_maxnorm(lat.pops, ref["pops"]) < tol, (wallkind, dt)
