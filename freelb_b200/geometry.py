"""Block decomposition of the cavity domain (host side).

Mirrors what the reference builds with BlockReader (src/io/block_reader.h)
and BlockGeometry3D(BlockReader&, true) (src/geometry/block_geometry3d.hh:199-219):
each block is an axis-aligned box of interior cells plus a one-cell overlap
layer.  Global stored indices put the domain's void layer at 0 and Ni+1 and
the interior at 1..Ni, so a block whose interior starts at physical
coordinate X0 (cell centres X0 + 0.5, ...) has its stored origin at X0.
"""
from __future__ import annotations

import random


def partition_axis(total: int, edges=(32, 48, 64, 96), rng: random.Random | None = None):
    """Split `total` cells into a seeded sequence of edge lengths drawn from `edges`."""
    rng = rng or random.Random(0)
    edges = sorted(set(int(e) for e in edges))
    for _ in range(10000):
        out, left = [], total
        while left > 0:
            cand = [e for e in edges if e <= left and (left - e == 0 or left - e >= edges[0])]
            if not cand:
                break
            e = rng.choice(cand)
            out.append(e)
            left -= e
        if left == 0:
            return out
    raise ValueError(f"cannot tile {total} with edges {edges}")


def uneven_blocks(ni: int, edges=(32, 48, 64, 96), seed: int = 0):
    """Blocks tiling an ni^3 interior with per-axis edge sequences drawn by seed.

    Returns a list of dicts with the interior box (x0, y0, z0, ex, ey, ez) and
    the stored block (nx, ny, nz, ox, oy, oz) including the overlap layer,
    ordered x fastest, then y, then z.
    """
    rng = random.Random(seed)
    px = partition_axis(ni, edges, rng)
    py = partition_axis(ni, edges, rng)
    pz = partition_axis(ni, edges, rng)

    def starts(p):
        s, acc = [], 0
        for e in p:
            s.append(acc)
            acc += e
        return s

    blocks = []
    for z0, ez in zip(starts(pz), pz):
        for y0, ey in zip(starts(py), py):
            for x0, ex in zip(starts(px), px):
                blocks.append({"x0": x0, "y0": y0, "z0": z0, "ex": ex, "ey": ey, "ez": ez,
                               "nx": ex + 2, "ny": ey + 2, "nz": ez + 2,
                               "ox": x0, "oy": y0, "oz": z0})
    return blocks


def x_blocks(ni: int, cuts):
    """Blocks tiling an ni^3 interior split along x only at the given cuts (full
    y and z), in x order, in the form uneven_blocks returns."""
    n = ni + 2
    edges = [0] + list(cuts) + [ni]
    return [{"x0": a, "y0": 0, "z0": 0, "ex": b - a, "ey": ni, "ez": ni,
             "nx": b - a + 2, "ny": n, "nz": n, "ox": a, "oy": 0, "oz": 0}
            for a, b in zip(edges[:-1], edges[1:])]


def block_tuples(blocks):
    """(nx, ny, nz, ox, oy, oz) per block, the form the C ABI takes."""
    return [(b["nx"], b["ny"], b["nz"], b["ox"], b["oy"], b["oz"]) for b in blocks]


def write_block_file(path: str, blocks) -> None:
    """Write blocks in the reference's BlockReader text format (block_reader.h:30-40)."""
    lines = ["Refine: 0", "VoxelSize: 1.", ""]
    for b in blocks:
        lines += ["[Block]", "Overlap: 1", "Level: 0",
                  f"AABB: {{{{{b['x0']}, {b['y0']}, {b['z0']}}}, "
                  f"{{{b['x0'] + b['ex']}, {b['y0'] + b['ey']}, {b['z0'] + b['ez']}}}}}",
                  f"Mesh: {{{b['ex']}, {b['ey']}, {b['ez']}}}", ""]
    with open(path, "w") as f:
        f.write("\n".join(lines))


def slice_block(global_field, n: int, b, comps: int = 1):
    """The part of a global (n^3 stored cells) field that block b stores."""
    import numpy as np
    g = np.asarray(global_field).reshape(n, n, n, comps) if comps > 1 else \
        np.asarray(global_field).reshape(n, n, n)
    s = g[b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"], b["ox"]:b["ox"] + b["nx"]]
    return np.ascontiguousarray(s).reshape(-1)
