"""Post-stream halfway bounce-back managers on the GPU against the reference's
BBLikeFixedBlockBdManager (run in the reference harness with FLB_POSTSTREAM_BB
and restated in oracle.poststream_bb)."""
import numpy as np
import pytest

import freelb_b200 as F
from conftest import rel_maxnorm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def seeded_fields(n, seed=7):
    rng = np.random.default_rng(seed)
    return 1.0 + rng.uniform(-0.02, 0.02, n ** 3), rng.uniform(-0.03, 0.03, (n ** 3, 3))


def hw_cavity(ni, tau, storage, wall_kind, fields):
    """Cavity whose wall (4) and lid (8) cells collide like fluid and get the
    post-stream managers, as examples/couette2d/couette2d.cpp:212-216 does."""
    n = ni + 2
    lat = F.Lattice(n, n, n, tau, storage=storage, tasks=((2 | 4 | 8, "bulk"),))
    lat.upload_flags(F.cavity_flags(ni))
    lat.upload_field("rho", fields[0].astype(lat.real))
    lat.upload_field("u", fields[1].astype(lat.real))
    wall = F.BounceBackManager(lat, 4, 1, kind=wall_kind)
    lid = F.BounceBackManager(lat, 8, 1, kind="movingwall")
    return lat, wall, lid


@pytest.mark.parametrize("kind", ["normal", "anti_simple", "anti_o1", "anti_o2",
                                  "anti_pressure"])
@pytest.mark.parametrize("storage,tol", [("fp64", 1e-12), ("fp32", 1e-5), ("fp32s", 1e-6)])
def test_poststream_bb_matches_oracle(gpu_ok, storage, tol, kind):
    """FP32S (FP32 deviations f - rho0 w) is held against the FP64 oracle."""
    ni, tau, steps = 16, 0.6, 8
    n = ni + 2
    dt = np.float32 if storage == "fp32" else np.float64
    fields = seeded_fields(n)
    lat, wall, lid = hw_cavity(ni, tau, storage, kind, fields)
    ncells, nlinks = wall.counts()
    assert ncells > 0 and nlinks > ncells
    fl = O.cavity_flags(ni)
    ref = O.Lattice(n, n, n, fl, tau=tau, dtype=dt, keys=(2 | 4 | 8,), ops=(O.OP_BULK,))
    ref.rho[:] = fields[0].astype(dt)
    ref.u.reshape(-1, 3)[:] = fields[1].astype(dt)
    for _ in range(steps):
        lat.step(1)
        wall.apply()
        lid.apply()
        ref.step(1)
        O.poststream_bb(ref, 4, 1, kind)
        O.poststream_bb(ref, 8, 1, "movingwall")
    assert rel_maxnorm(lat.download_pops(), ref.pops) < tol


def test_poststream_bb_cavity_40_steps(gpu_ok):
    """The couette-style cavity (normal walls, moving lid, fields as set up by
    the cavity) over 40 steps in FP64."""
    ni, tau, steps = 16, 0.6, 40
    n = ni + 2
    fl = O.cavity_flags(ni)
    u = np.zeros((n ** 3, 3))
    u[fl == 8, 0] = 0.1
    lat, wall, lid = hw_cavity(ni, tau, "fp64", "normal", (np.ones(n ** 3), u))
    ref = O.Lattice(n, n, n, fl, tau=tau, dtype=np.float64, keys=(2 | 4 | 8,), ops=(O.OP_BULK,))
    ref.u.reshape(-1, 3)[fl == 8, 0] = 0.1
    for _ in range(steps):
        lat.step(1)
        wall.apply()
        lid.apply()
        ref.step(1)
        O.poststream_bb(ref, 4, 1, "normal")
        O.poststream_bb(ref, 8, 1, "movingwall")
    assert rel_maxnorm(lat.download_pops(), ref.pops) < 1e-12


def test_poststream_bb_fp16s_close_to_fp32(gpu_ok):
    ni, steps = 16, 40
    n = ni + 2
    fl = O.cavity_flags(ni)
    u = np.zeros((n ** 3, 3))
    u[fl == 8, 0] = 0.1
    out = {}
    for storage in ("fp32", "fp16s"):
        lat, wall, lid = hw_cavity(ni, 0.6, storage, "normal", (np.ones(n ** 3), u))
        for _ in range(steps):
            lat.step(1)
            wall.apply()
            lid.apply()
        out[storage] = lat.download_pops(np.float32)
    assert rel_maxnorm(out["fp16s"], out["fp32"]) < 2e-3


def test_bb_manager_rejects_unknown_kind(gpu_ok):
    lat = F.cavity(8)
    with pytest.raises(ValueError):
        F.BounceBackManager(lat, 4, 1, kind="sideways")
