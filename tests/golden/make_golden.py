"""Generate the golden fixtures in tests/golden/ by running the reference itself.

    make -C oracle && python tests/golden/make_golden.py
    python tests/golden/make_golden.py --periodic   (the periodic-manager fixtures only)

Each fixture is the output of the reference FreeLB CPU path (the harness
oracle/ref_cavity.cpp compiled from the reference's own headers into
oracle/_ref/), on the lid-driven cavity of benchmarks/cavity3d/cavity3d.cpp.
Small cases keep every array; the 100^3 x 1000-step case (the reference's
cavity3d benchmark shape) keeps per-direction population sums, the flags and
the y = 51 mid-plane of rho and u.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

SMALL = [
    # name, model, Ni, tau, u_lid, steps, Cs, dtype
    ("cavity_bgk_f32_n10_s40", "bgk", 10, 0.53, 0.1, 40, 0.1, np.float32),
    ("cavity_bgk_f64_n10_s40", "bgk", 10, 0.53, 0.1, 40, 0.1, np.float64),
    ("cavity_les_f32_n10_s40", "les", 10, 0.51, 0.1, 40, 0.1, np.float32),
    ("cavity_les_f64_n10_s40", "les", 10, 0.51, 0.1, 40, 0.1, np.float64),
    ("cavity_mrt_f32_n10_s40", "mrt", 10, 0.53, 0.1, 40, 0.1, np.float32),
    ("cavity_mrt_f64_n10_s40", "mrt", 10, 0.53, 0.1, 40, 0.1, np.float64),
    ("cavity_bgk_f32_n7_s200", "bgk", 7, 0.6, 0.05, 200, 0.1, np.float32),
]


def small(name, model, ni, tau, ulid, steps, cs, dtype):
    r = O.run_reference(model, ni, tau, ulid, steps, 0, cs=cs, dtype=dtype, threads=4)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), flags=r["flags"], pops=r["pops"],
                        rho=r["rho"], u=r["u"],
                        params=np.array([ni, tau, ulid, steps, cs], dtype=np.float64),
                        model=np.array(model))
    print(name, "written")


def multiblock(name, ni, edges, seed, steps, dtype):
    """Reference multi-block run (BlockReader blocks + NormalCommunicate)."""
    import tempfile
    from freelb_b200 import geometry as G
    blocks = G.uneven_blocks(ni, edges=edges, seed=seed)
    with tempfile.TemporaryDirectory() as d:
        bf = os.path.join(d, "blocks.txt")
        G.write_block_file(bf, blocks)
        r = O.run_reference("bgk", ni, 0.53, 0.1, steps, 0, dtype=dtype, blockfile=bf,
                            threads=4)
    out = {"params": np.array([ni, 0.53, 0.1, steps, seed], dtype=np.float64),
           "edges": np.array(edges), "nblocks": np.array(len(blocks))}
    for k in range(len(blocks)):
        for f in ("flags", "pops", "rho", "u"):
            out[f"{f}_b{k}"] = r[f"{f}_b{k}"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "written,", len(blocks), "blocks")


def periodic(name, ni, cuts, steps, dtype):
    """Reference run with FixedPeriodicBoundaryManager on the x = 0 / x = ni-1
    wall columns (ref_cavity FLB_PERIODIC=1) over x-split blocks."""
    import tempfile
    from freelb_b200 import geometry as G
    blocks = G.x_blocks(ni, cuts)  # the manager pairs a box in an earlier block with a later one
    with tempfile.TemporaryDirectory() as d:
        bf = os.path.join(d, "blocks.txt")
        G.write_block_file(bf, blocks)
        r = O.run_reference("bgk", ni, 0.6, 0.1, steps, 0, dtype=dtype, blockfile=bf,
                            threads=4, periodic=True)
    out = {"params": np.array([ni, 0.6, 0.1, steps], dtype=np.float64),
           "cuts": np.array(cuts), "nblocks": np.array(len(blocks))}
    for k in range(len(blocks)):
        for f in ("flags", "pops"):
            out[f"{f}_b{k}"] = r[f"{f}_b{k}"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "written,", len(blocks), "blocks")


def c1():
    ni, steps = 100, 1000
    r = O.run_reference("bgk", ni, 0.53, 0.1, steps, 0, dtype=np.float32)
    n = ni + 2
    pops = r["pops"].reshape(19, n, n, n)
    u = r["u"].reshape(n, n, n, 3)
    rho = r["rho"].reshape(n, n, n)
    np.savez_compressed(os.path.join(HERE, "c1_bgk_f32_n100_s1000.npz"),
                        flags=r["flags"],
                        pop_sums=pops.astype(np.float64).sum(axis=(1, 2, 3)),
                        u_plane=u[:, n // 2, :, :].copy(), rho_plane=rho[:, n // 2, :].copy(),
                        pops_plane=pops[:, :, n // 2, :].copy(),
                        params=np.array([ni, 0.53, 0.1, steps, 0.1], dtype=np.float64))
    print("c1 written, reference MLUPs", r["mlups"])


if __name__ == "__main__":
    if "--periodic" in sys.argv:
        periodic("periodic_bgk_f64_n12_s30", 12, (5,), 30, np.float64)
        periodic("periodic_bgk_f32_n12_s30", 12, (5,), 30, np.float32)
        sys.exit(0)
    for case in SMALL:
        small(*case)
    multiblock("blocks_bgk_f64_n12_s30", 12, (4, 8), 3, 30, np.float64)
    multiblock("blocks_bgk_f32_n12_s30", 12, (4, 8), 3, 30, np.float32)
    if "--no-c1" not in sys.argv:
        c1()
