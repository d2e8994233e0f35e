"""Python access to the oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (the C restatement in flb_oracle.c) and, where
built, runs the reference harness binaries in ``oracle/_ref/`` (compiled from
the reference's own sources by oracle/Makefile).  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs use
this module; the product (freelb_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

OP_NONE, OP_BULK, OP_BB, OP_MBB, OP_FIELD_BGK = 0, 1, 2, 3, 4
MODEL_BGK, MODEL_MRT, MODEL_LES = 0, 1, 2
MODEL_BRINKMAN = 3
MODELS = {"bgk": MODEL_BGK, "mrt": MODEL_MRT, "les": MODEL_LES, "brinkman": MODEL_BRINKMAN}

# D3Q19, reference ordering (src/lbm/lattice_set.h:263-266)
C = np.array([(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
              (1, 1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, -1), (0, 1, 1), (0, -1, -1),
              (1, -1, 0), (-1, 1, 0), (1, 0, -1), (-1, 0, 1), (0, 1, -1), (0, -1, 1)],
             dtype=np.int64)
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


class _Desc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("model", ctypes.c_int), ("omega", ctypes.c_double),
                ("cs_smag", ctypes.c_double), ("mrt_s", ctypes.c_double * 19),
                ("op_lut", ctypes.c_uint8 * 256), ("alpha", ctypes.c_void_p)]


_lib = None


def build():
    """Compile the restatement (and the reference harness when its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        _lib.oracle_cavity_flags.argtypes = [ctypes.c_int, P]
        _lib.oracle_build_lut.argtypes = [ctypes.c_int, P, P, P]
        for s in ("f32", "f64"):
            getattr(_lib, f"oracle_step_{s}").argtypes = [P, P, P, P, P, P, ctypes.c_int]
            getattr(_lib, f"oracle_rhou_fields_{s}").argtypes = [ctypes.c_long, P, ctypes.c_uint8,
                                                                  P, P, P]
            getattr(_lib, f"oracle_init_pops_{s}").argtypes = [ctypes.c_long, ctypes.c_double, P]
        _lib.oracle_mrt_basis.argtypes = [P, P]
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def cavity_flags(ni: int) -> np.ndarray:
    n = ni + 2
    f = np.empty(n * n * n, dtype=np.uint8)
    lib().oracle_cavity_flags(ni, _ptr(f))
    return f


def task_lut(keys, ops) -> np.ndarray:
    keys = np.asarray(keys, dtype=np.uint8)
    ops = np.asarray(ops, dtype=np.uint8)
    lut = np.empty(256, dtype=np.uint8)
    lib().oracle_build_lut(len(keys), _ptr(keys), _ptr(ops), _ptr(lut))
    return lut


CAVITY_KEYS = (2, 4, 8)
CAVITY_OPS = (OP_BULK, OP_BB, OP_MBB)


def mrt_basis():
    M = np.empty(361)
    inv = np.empty(361)
    lib().oracle_mrt_basis(_ptr(M), _ptr(inv))
    return M.reshape(19, 19), inv.reshape(19, 19)


class Lattice:
    """One block of the restated reference lattice (populations in logical order)."""

    def __init__(self, nx, ny, nz, flags, model="bgk", tau=0.53, cs=0.1, mrt_rate=1.2,
                 dtype=np.float32, keys=CAVITY_KEYS, ops=CAVITY_OPS):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.N = nx * ny * nz
        self.dtype = np.dtype(dtype)
        self.suffix = "f32" if self.dtype == np.float32 else "f64"
        self.flags = np.ascontiguousarray(flags, dtype=np.uint8).reshape(-1)
        assert self.flags.size == self.N
        d = _Desc()
        d.nx, d.ny, d.nz = nx, ny, nz
        d.model = MODELS[model]
        tau_t = self.dtype.type(tau)
        # omega = T(1)/T(RT) as in unit_converter.h:209
        d.omega = float(self.dtype.type(1) / tau_t)
        d.cs_smag = float(cs)
        rates = [float(mrt_rate)] * 19 if np.isscalar(mrt_rate) else [float(r) for r in mrt_rate]
        for i in range(19):
            d.mrt_s[i] = 0.0 if i in (0, 3, 5, 7) else rates[i]
        lut = task_lut(keys, ops)
        for v in range(256):
            d.op_lut[v] = int(lut[v])
        self.desc = d
        self.pops = np.empty(19 * self.N, dtype=self.dtype)
        getattr(lib(), f"oracle_init_pops_{self.suffix}")(self.N, 1.0, _ptr(self.pops))
        self.tmp = np.empty_like(self.pops)
        self.rho = np.ones(self.N, dtype=self.dtype)
        self.u = np.zeros(3 * self.N, dtype=self.dtype)
        self.alpha = None

    def set_alpha(self, alpha):
        """Per-cell Brinkman porosity for the brinkman model."""
        self.alpha = np.ascontiguousarray(alpha, dtype=self.dtype).reshape(-1)
        assert self.alpha.size == self.N
        self.desc.alpha = self.alpha.ctypes.data

    def objective_u2(self, key=2):
        """J = sum over cells matching key of |u|^2, u = sum c f / (rho + alpha/2)."""
        f = self.pops.reshape(19, self.N).astype(np.float64)
        m = (self.flags & key) != 0
        rho = f[:, m].sum(axis=0)
        mom = C.T.astype(np.float64) @ f[:, m]
        a = self.alpha[m].astype(np.float64) if self.alpha is not None else 0.0
        u = mom / (rho + 0.5 * a)
        return float((u * u).sum())

    def step(self, n=1):
        getattr(lib(), f"oracle_step_{self.suffix}")(ctypes.byref(self.desc), _ptr(self.flags),
                                                     _ptr(self.pops), _ptr(self.tmp),
                                                     _ptr(self.rho), _ptr(self.u), int(n))

    def rhou_fields(self, key=2):
        getattr(lib(), f"oracle_rhou_fields_{self.suffix}")(self.N, _ptr(self.flags), key,
                                                            _ptr(self.pops), _ptr(self.rho),
                                                            _ptr(self.u))
        return self.rho, self.u


def cavity(ni, model="bgk", tau=0.53, ulid=0.1, cs=0.1, mrt_rate=1.2, dtype=np.float32,
           alpha=None):
    """The reference lid-driven cavity (benchmarks/cavity3d/cavity3d.cpp:111-161)."""
    n = ni + 2
    flags = cavity_flags(ni)
    lat = Lattice(n, n, n, flags, model=model, tau=tau, cs=cs, mrt_rate=mrt_rate, dtype=dtype)
    lat.u.reshape(-1, 3)[flags == 8, 0] = lat.dtype.type(ulid)
    if alpha is not None:
        lat.set_alpha(alpha)
    return lat


def porosity(ni, seed, amax=0.05):
    """Seeded i.i.d. U[0, amax] porosity on the (ni+2)^3 stored mesh (float64)."""
    n = ni + 2
    return np.random.default_rng(seed).uniform(0.0, amax, size=n ** 3)


# --------------------------------------------------------------------------- reference harness

def ref_binary(dtype=np.float32):
    """Path of the reference harness for this host's ISA, or None when not built."""
    s = "f32" if np.dtype(dtype) == np.float32 else "f64"
    isa = "v3"
    try:
        with open("/proc/cpuinfo") as f:
            if " avx512f" in f.read():
                isa = "v4"
    except OSError:
        pass
    for cand in (isa, "v3"):
        p = os.path.join(REF_DIR, f"ref_cavity_{s}_{cand}")
        if os.path.exists(p):
            return p
    return None


def run_reference(model, ni, tau, ulid, steps, warmup=0, cs=0.1, dtype=np.float32,
                  blockfile=None, threads=None, outdir=None, alpha=None, fields=None,
                  poststream=None, comm=None, periodic=False):
    """Run the reference's own CPU path; returns (dict of arrays, mlups)."""
    exe = ref_binary(dtype)
    if exe is None:
        raise FileNotFoundError("reference harness not built (oracle/_ref)")
    own = outdir is None
    if own:
        tmpd = tempfile.TemporaryDirectory()
        outdir = tmpd.name
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    if alpha is not None:
        afile = os.path.join(tempfile.mkdtemp(), "alpha.bin")
        np.ascontiguousarray(alpha, dtype=dtype).tofile(afile)
        env["FLB_ALPHA_FILE"] = afile
    if fields is not None:  # (rho[N], u[N, 3]) replacing the RHO and VELOCITY fields
        ffile = os.path.join(tempfile.mkdtemp(), "fields.bin")
        np.concatenate([np.ravel(fields[0]), np.ravel(fields[1])]).astype(dtype).tofile(ffile)
        env["FLB_FIELDS_FILE"] = ffile
    if poststream is not None:  # wall kind 1..5 of the post-stream managers
        env["FLB_POSTSTREAM_BB"] = str(int(poststream))
    if comm is not None:  # "full" / "all": NormalFullCommunicate / NormalAllCommunicate
        env["FLB_COMM"] = comm
    if periodic:  # FixedPeriodicBoundaryManager on the x = 0 / x = Ni-1 wall columns
        env["FLB_PERIODIC"] = "1"
    args = [exe, model, str(ni), repr(float(tau)), repr(float(ulid)), str(steps), str(warmup),
            outdir, repr(float(cs))]
    if blockfile:
        args.append(blockfile)
    out = subprocess.run(args, check=True, capture_output=True, text=True, env=env).stdout
    line = [ln for ln in out.splitlines() if ln.startswith("MLUPS")][-1].split()
    mlups = float(line[1])
    res = {"mlups": mlups, "seconds": float(line[7]), "threads": int(line[9])}
    if outdir != "-":
        res.update(load_dump(outdir, dtype))
    if own:
        tmpd.cleanup()
    return res


def load_dump(outdir, dtype=np.float32):
    dt = np.dtype(dtype)
    meta = {}
    blocks = []
    with open(os.path.join(outdir, "meta.txt")) as f:
        for ln in f:
            parts = ln.split()
            if parts[0] == "block":
                blocks.append({"mesh": tuple(int(v) for v in parts[3:6]),
                               "min": tuple(float(v) for v in parts[7:10]),
                               "overlap": int(parts[11])})
            else:
                meta[parts[0]] = parts[1]
    res = {"meta": meta, "blocks": blocks}
    nb = len(blocks)
    for k, b in enumerate(blocks):
        sfx = f"_b{k}" if nb > 1 else ""
        N = b["mesh"][0] * b["mesh"][1] * b["mesh"][2]
        res[f"flags{sfx}"] = np.fromfile(os.path.join(outdir, f"flags{sfx}.u8"), dtype=np.uint8)
        res[f"pops{sfx}"] = np.fromfile(os.path.join(outdir, f"pops{sfx}.bin"), dtype=dt)
        res[f"rho{sfx}"] = np.fromfile(os.path.join(outdir, f"rho{sfx}.bin"), dtype=dt)
        res[f"u{sfx}"] = np.fromfile(os.path.join(outdir, f"u{sfx}.bin"), dtype=dt)
        assert res[f"pops{sfx}"].size == 19 * N
    return res


def rel_maxnorm(a, b):
    """max|a-b| / max|b| (the parity norm used by the tests)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


# --------------------------------------------------------------------------- multi-block

class MultiBlock:
    """Blocks of one cavity domain, each a restated BlockLattice with its own
    periodic-shift streaming, followed after every step by the halo copy of
    BlockLatticeManager::normalCommunicate (src/data_struct/block_lattice.hh:
    1668-1685): each overlap cell owned by a neighbour's interior receives that
    neighbour cell's populations in the directions that cross into the block
    (getCommPopDir, src/parallel/communicator.h:76-150: union over the faces
    the cell lies beyond)."""

    def __init__(self, blocks, global_flags, n, model="bgk", tau=0.53, ulid=0.1, cs=0.1,
                 mrt_rate=1.2, dtype=np.float32, full=False):
        """full=True: normalFullCommunicate / normalAllCommunicate
        (block_lattice.hh:1687-1720): all 19 populations of every overlap cell
        owned by a neighbour (one overlap layer: the first layer is all)."""
        self.blocks = blocks
        self.lats = []
        gf = np.asarray(global_flags).reshape(n, n, n)
        for b in blocks:
            fl = np.ascontiguousarray(gf[b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"],
                                      b["ox"]:b["ox"] + b["nx"]]).reshape(-1)
            lat = Lattice(b["nx"], b["ny"], b["nz"], fl, model=model, tau=tau, cs=cs,
                          mrt_rate=mrt_rate, dtype=dtype)
            lat.u.reshape(-1, 3)[fl == 8, 0] = lat.dtype.type(ulid)
            self.lats.append(lat)
        owner = -np.ones((n, n, n), dtype=np.int64)
        for k, b in enumerate(blocks):
            owner[b["oz"] + 1:b["oz"] + b["nz"] - 1, b["oy"] + 1:b["oy"] + b["ny"] - 1,
                  b["ox"] + 1:b["ox"] + b["nx"] - 1] = k
        # records grouped per (block, neighbour, direction): (dst idx array, src idx array)
        self.copies = []
        for k, b in enumerate(blocks):
            nx, ny, nz = b["nx"], b["ny"], b["nz"]
            lz, ly, lx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
            lx, ly, lz = lx.ravel(), ly.ravel(), lz.ravel()
            outer = (lx == 0) | (ly == 0) | (lz == 0) | (lx == nx - 1) | (ly == ny - 1) | \
                    (lz == nz - 1)
            lx, ly, lz = lx[outer], ly[outer], lz[outer]
            gx, gy, gz = lx + b["ox"], ly + b["oy"], lz + b["oz"]
            own = owner[gz, gy, gx]
            keep = own >= 0
            lx, ly, lz, gx, gy, gz, own = (a[keep] for a in (lx, ly, lz, gx, gy, gz, own))
            dst = lx + nx * (ly + ny * lz)
            for i in range(0 if full else 1, 19):
                cxi, cyi, czi = C[i]
                cross = np.zeros(lx.size, dtype=bool)
                for l, m, c in ((lx, nx, cxi), (ly, ny, cyi), (lz, nz, czi)):
                    cross |= ((l == 0) & (c > 0)) | ((l == m - 1) & (c < 0))
                if full:
                    cross[:] = True
                for o in np.unique(own[cross]):
                    sel = cross & (own == o)
                    nb = blocks[o]
                    src = (gx[sel] - nb["ox"]) + nb["nx"] * ((gy[sel] - nb["oy"]) +
                                                            nb["ny"] * (gz[sel] - nb["oz"]))
                    self.copies.append((k, int(o), i, dst[sel], src))

    def step(self, n=1):
        for _ in range(n):
            for lat in self.lats:
                lat.step(1)
            for k, o, i, dst, src in self.copies:
                a, b = self.lats[k], self.lats[o]
                a.pops[i * a.N + dst] = b.pops[i * b.N + src]

    def rhou_fields(self, key=2):
        return [lat.rhou_fields(key) for lat in self.lats]


BB_KINDS = ("normal", "movingwall", "anti_simple", "anti_o1", "anti_o2", "anti_pressure")


def poststream_bb(lat, cell_flag, void_flag, kind="normal"):
    """Post-stream halfway bounce-back of one BBLikeFixedBlockBdManager
    (src/boundary/boundary.h:86-140) on a restated lattice.  For every inner
    cell with `cell_flag` and every direction k whose neighbour x + c_k has
    `void_flag` (basic_boundary.h:196-211), the outflow j = opp(k) is set from
    prev = getPrevious(k)(x) = R_k(x + Delta_k mod N) (field.h:645-656) and the
    cell's RHO and VELOCITY fields (bounce_back_boundary.h:167-256):
        normal         R_j = prev
        movingwall     R_j = prev + 2 InvCs2 w_j rho (u . c_j)
        anti_simple    R_j = 2 rho w_j - prev
        anti_o1        R_j = 2 feq1_j(rho, u) - prev
        anti_o2        R_j = 2 feq2_j(rho, u, |u|^2) - prev
        anti_pressure  R_j = 2 rho w_j (1 + (uw . c_j)^2 InvCs4 / 2
                                        - |uw|^2 InvCs2 / 2) - prev,
                       uw = u + (u - u(x + c_k)) / 2.
    The arithmetic follows the reference expressions term by term."""
    if kind is True or kind is False:  # moving flag of the two-kind form
        kind = "movingwall" if kind else "normal"
    if kind not in BB_KINDS:
        raise ValueError(f"unknown bounce-back kind {kind!r}")
    nx, ny, nz, N = lat.nx, lat.ny, lat.nz, lat.N
    R = lat.pops.reshape(19, N)
    f = lat.flags.reshape(nz, ny, nx)
    inner = np.zeros_like(f, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    cells = np.flatnonzero((inner & ((f & cell_flag) != 0)).reshape(-1))
    x = cells % nx
    y = (cells // nx) % ny
    z = cells // (nx * ny)
    T = lat.dtype.type
    U = lat.u.reshape(-1, 3)
    opp = [0] + [i + 1 if i % 2 else i - 1 for i in range(1, 19)]

    def dot(u, c):
        return (u[:, 0] * T(c[0]) + u[:, 1] * T(c[1])) + u[:, 2] * T(c[2])

    def norm2(u):
        return (u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1]) + u[:, 2] * u[:, 2]

    for k in range(1, 19):
        cxk, cyk, czk = (int(v) for v in C[k])
        nb = (x + cxk) + nx * ((y + cyk) + ny * (z + czk))
        sel = (lat.flags[nb] & void_flag) != 0
        if not sel.any():
            continue
        xs = cells[sel]
        d = cxk + cyk * nx + czk * nx * ny
        prev = R[k, (xs + d) % N].copy()
        j = opp[k]
        w = T(1) / T(3) if j == 0 else (T(1) / T(18) if j < 7 else T(1) / T(36))
        rho = lat.rho[xs]
        u = U[xs]
        if kind == "normal":
            val = prev
        elif kind == "movingwall":
            val = prev + T(2) * T(3) * w * rho * dot(u, C[j])
        elif kind == "anti_simple":
            val = T(2) * rho * w - prev
        elif kind == "anti_o1":
            val = T(2) * (w * rho * (T(1) + T(3) * dot(u, C[j]))) - prev
        elif kind == "anti_o2":
            uc = dot(u, C[j])
            val = T(2) * (w * rho * (T(1) + T(3) * uc + uc * uc * T(0.5) * T(9)
                                     - T(3) * norm2(u) * T(0.5))) - prev
        else:
            # std::pow(T, int) is evaluated in double, which carries the rest
            # of the expression in double until the store into the T array.
            uw = u + T(0.5) * (u - U[nb[sel]])
            sq = np.float64(dot(uw, C[j])) ** 2
            bracket = (1.0 + sq * 0.5 * 9.0) - np.float64(norm2(uw) * T(0.5) * T(3))
            val = (np.float64(T(2) * rho * w) * bracket - np.float64(prev)).astype(lat.dtype)
        R[j, xs] = val


def comm_pop_dirs(direction):
    """getCommPopDir (src/parallel/communicator.h:74-150): the directions that
    enter a cell across the faces named by the NbrDirection bits (XN=1, XP=2,
    YN=4, YP=8, ZN=16, ZP=32), sorted."""
    out = []
    for i in range(19):
        c = C[i]
        sel = ((direction & 1 and c[0] > 0) or (direction & 2 and not direction & 1 and c[0] < 0)
               or (direction & 4 and c[1] > 0) or (direction & 8 and not direction & 4 and c[1] < 0)
               or (direction & 16 and c[2] > 0)
               or (direction & 32 and not direction & 16 and c[2] < 0))
        if sel:
            out.append(i)
    return out


def box_cells(nx, ny, nz, box):
    """Stored cells of an inclusive box (x0, x1, y0, y1, z0, z1), clamped to the
    mesh, in z, y, x order (BasicBlock::getCellIdx, basic_geometry.hh:593-619)."""
    x0, x1, y0, y1, z0, z1 = box
    x0, y0, z0 = max(x0, 0), max(y0, 0), max(z0, 0)
    x1, y1, z1 = min(x1, nx - 1), min(y1, ny - 1), min(z1, nz - 1)
    z, y, x = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1),
                          indexing="ij")
    return (x + nx * (y + ny * z)).reshape(-1)


def periodic_copy(lat, box0, dir0, box1, dir1):
    """FixedPeriodicBoundaryManager::Apply (src/boundary/periodic_boundary.h:
    302-321) on a restated single-block lattice, as the two-way exchange the
    reference performs between boxes in different blocks: box0 cell[k] =
    box1 cell[k] for k in getCommPopDir(dir0) and box1 cell[k] = box0 cell[k]
    for k in getCommPopDir(dir1), on the post-collision populations.  The
    restated step fuses collide and stream, so the copy is applied to the
    post-stream state: a pre-stream P_k(x) sits at R_k((x + Delta_k) mod N)
    (CyclicArray::rotate, field.h:676-697).  Sources are read before any write."""
    nx, ny, nz, N = lat.nx, lat.ny, lat.nz, lat.N
    R = lat.pops.reshape(19, N)
    c0 = box_cells(nx, ny, nz, box0)
    c1 = box_cells(nx, ny, nz, box1)
    assert c0.size == c1.size
    moves = []
    for k in comm_pop_dirs(dir0):
        d = int(C[k][0]) + nx * (int(C[k][1]) + ny * int(C[k][2]))
        moves.append((k, (c0 + d) % N, R[k, (c1 + d) % N].copy()))
    for k in comm_pop_dirs(dir1):
        d = int(C[k][0]) + nx * (int(C[k][1]) + ny * int(C[k][2]))
        moves.append((k, (c1 + d) % N, R[k, (c0 + d) % N].copy()))
    for k, dst, val in moves:
        R[k, dst] = val


# ---------------------------------------------------------------------------
# VTK DataArray bodies (test infrastructure for the device encoder).

def vtk_crop(values, mesh, overlap, ncomp=1):
    """Cells [overlap, n - overlap) per axis, x fastest, components interleaved
    (util::CopyFromFieldArray, src/utils/util.h:439-540)."""
    nx, ny, nz = mesh
    v = np.asarray(values).reshape(nz, ny, nx, ncomp) if ncomp > 1 else \
        np.asarray(values).reshape(nz, ny, nx)
    o = overlap
    return np.ascontiguousarray(v[o:nz - o, o:ny - o, o:nx - o]).reshape(-1)


def vtk_body(data):
    """Body of a binary base64 DataArray as Base64Encoder writes it
    (src/io/base64.h; vti_writer.h:552-611): the data size in bytes as a
    little-endian unsigned int, encoded on its own, then the data."""
    import base64
    raw = np.ascontiguousarray(data).tobytes()
    size = np.array([len(raw) & 0xFFFFFFFF], dtype="<u4").tobytes()
    return base64.b64encode(size).decode() + base64.b64encode(raw).decode()


def vtk_arrays(path):
    """{name: (type, ncomp, body)} of the DataArrays of a .vti file."""
    import re
    text = open(path, "rb").read().decode()
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)" Name="(\w+)" format="binary" '
                         r'encoding="base64" NumberOfComponents="(\d+)">\n(.*?)\n</DataArray>',
                         text, re.S):
        out[m.group(2)] = (m.group(1), int(m.group(3)), m.group(4))
    return out


def vtk_decode(body, dtype):
    """Values of a DataArray body (inverse of vtk_body)."""
    import base64
    size = np.frombuffer(base64.b64decode(body[:8]), dtype="<u4")[0]
    data = base64.b64decode(body[8:])
    assert len(data) == size
    return np.frombuffer(data, dtype=dtype)
