"""FixedPeriodicBoundaryManager (src/boundary/periodic_boundary.h:136-321).

The fixtures are the reference's own run (oracle/ref_cavity FLB_PERIODIC=1):
the lid-driven cavity with its x = 0 and x = Ni-1 wall columns flagged 16 (no
task matches them, so they only carry populations), a periodic manager
Setup(left, XN, right, XP) applied between ApplyCellDynamics and Stream, and
two blocks split along x so that the manager takes its cross-block pairing.
Fluid cells do not depend on the block split, so a single-block run with the
two-way exchange must reproduce them."""
import numpy as np
import pytest

import freelb_b200 as F
from conftest import golden, rel_maxnorm
from oracle import oracle as O
from freelb_b200.geometry import x_blocks

NAMES = ["periodic_bgk_f64_n12_s30", "periodic_bgk_f32_n12_s30"]


def periodic_flags(ni):
    n = ni + 2
    f = O.cavity_flags(ni).reshape(n, n, n)
    f[2:n - 2, 2:n - 2, 1] = 16
    f[2:n - 2, 2:n - 2, n - 2] = 16
    return f.reshape(-1)


def boxes(ni):
    n = ni + 2
    return (1, 1, 2, n - 3, 2, n - 3), (n - 2, n - 2, 2, n - 3, 2, n - 3)


def fluid_compare(g, pops, ni, dtype):
    """Relative max-norm over the fluid cells of every reference block, after
    checking the flags bit for bit."""
    n = ni + 2
    blocks = x_blocks(ni, tuple(int(c) for c in g["cuts"]))
    flags = periodic_flags(ni).reshape(n, n, n)
    P = np.asarray(pops).reshape(19, n, n, n)
    got, ref = [], []
    for k, b in enumerate(blocks):
        fb = g[f"flags_b{k}"].reshape(b["nz"], b["ny"], b["nx"])
        assert np.array_equal(fb, flags[:, :, b["ox"]:b["ox"] + b["nx"]])
        pb = g[f"pops_b{k}"].reshape(19, b["nz"], b["ny"], b["nx"])
        ps = P[:, :, :, b["ox"]:b["ox"] + b["nx"]]
        m = fb == 2
        got.append(ps[:, m].ravel())
        ref.append(pb[:, m].ravel())
    return rel_maxnorm(np.concatenate(got).astype(dtype), np.concatenate(ref))


def test_comm_pop_dirs():
    # getCommPopDir: XN -> c_x > 0; XP -> c_x < 0; union over the set bits
    assert O.comm_pop_dirs(1) == [i for i in range(19) if O.C[i][0] > 0]
    assert O.comm_pop_dirs(2) == [i for i in range(19) if O.C[i][0] < 0]
    assert O.comm_pop_dirs(1 | 8) == sorted(
        i for i in range(19) if O.C[i][0] > 0 or O.C[i][1] < 0)
    assert O.comm_pop_dirs(0) == []


@pytest.mark.parametrize("name", NAMES)
def test_oracle_periodic_matches_reference(name):
    """The restated exchange (oracle.periodic_copy) against the reference."""
    g = golden(name)
    ni, tau, ulid, steps = (float(v) for v in g["params"])
    ni, steps = int(ni), int(steps)
    dtype = np.float64 if "f64" in name else np.float32
    lat = O.cavity(ni, tau=tau, ulid=ulid, dtype=dtype)
    lat.flags[:] = periodic_flags(ni)
    b0, b1 = boxes(ni)
    for _ in range(steps):
        lat.step(1)
        O.periodic_copy(lat, b0, 1, b1, 2)
    tol = 1e-13 if dtype == np.float64 else 1e-5
    assert fluid_compare(g, lat.pops, ni, dtype) < tol


def device_periodic(ni, storage, tau, ulid):
    n = ni + 2
    lat = F.Lattice(n, n, n, tau, storage=storage)
    flags = periodic_flags(ni)
    lat.upload_flags(flags)
    u = np.zeros((lat.N, 3), dtype=lat.real)
    u[flags == 8, 0] = lat.real(ulid)
    lat.upload_field("u", u)
    b0, b1 = boxes(ni)
    per = F.PeriodicBoundaryManager(lat, b0, "XN", b1, "XP", cell_flag=16)
    return lat, per


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_periodic_matches_reference(gpu_ok, name):
    g = golden(name)
    ni, tau, ulid, steps = (float(v) for v in g["params"])
    ni, steps = int(ni), int(steps)
    storage = "fp64" if "f64" in name else "fp32"
    lat, per = device_periodic(ni, storage, tau, ulid)
    n2 = (ni + 2 - 4) ** 2  # cells per box
    assert per.counts() == (n2, n2 * 10)  # five directions each way
    for _ in range(steps):
        lat.step(1)
        per.apply()
    tol = 1e-12 if storage == "fp64" else 1e-5
    assert fluid_compare(g, lat.download_pops(), ni, np.float64 if storage == "fp64" else
                         np.float32) < tol


@pytest.mark.gpu
def test_device_periodic_fp16s_against_fp64(gpu_ok):
    g = golden("periodic_bgk_f64_n12_s30")
    ni, tau, ulid, steps = (float(v) for v in g["params"])
    ni, steps = int(ni), int(steps)
    lat, per = device_periodic(ni, "fp16s", tau, ulid)
    for _ in range(steps):
        lat.step(1)
        per.apply()
    assert fluid_compare(g, lat.download_pops(), ni, np.float64) < 2e-3


@pytest.mark.gpu
def test_device_periodic_rules(gpu_ok):
    ni = 8
    n = ni + 2
    lat = F.Lattice(n, n, n, 0.6)
    lat.upload_flags(periodic_flags(ni))
    b0, b1 = boxes(ni)
    with pytest.raises(F.FlbError):  # different cell counts
        F.PeriodicBoundaryManager(lat, b0, "XN", (n - 2, n - 2, 2, n - 4, 2, n - 3), "XP", 16)
    # no cell carries the flag: an empty manager, as in the reference
    empty = F.PeriodicBoundaryManager(lat, b0, "XN", b1, "XP", 32)
    assert empty.counts() == (0, 0)
    empty.apply()
    # a box outside the interior: empty
    out = F.PeriodicBoundaryManager(lat, (0, 0, 0, 0, 0, 0), "XN", b1, "XP", 16)
    assert out.counts() == (0, 0)


@pytest.mark.gpu
def test_periodic_rejects_multiblock_handles(gpu_ok):
    from freelb_b200 import geometry as G
    blocks = x_blocks(8, (4,))
    lat = F.Lattice.blocks(G.block_tuples(blocks), 0.6, mode="halo")
    b0, b1 = boxes(8)
    with pytest.raises(F.FlbError):
        F.PeriodicBoundaryManager(lat, b0, "XN", b1, "XP", 16)
