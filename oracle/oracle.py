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
MODELS = {"bgk": MODEL_BGK, "mrt": MODEL_MRT, "les": MODEL_LES}

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
                ("op_lut", ctypes.c_uint8 * 256)]


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
        for i in range(19):
            d.mrt_s[i] = 0.0 if i in (0, 3, 5, 7) else float(mrt_rate)
        lut = task_lut(keys, ops)
        for v in range(256):
            d.op_lut[v] = int(lut[v])
        self.desc = d
        self.pops = np.empty(19 * self.N, dtype=self.dtype)
        getattr(lib(), f"oracle_init_pops_{self.suffix}")(self.N, 1.0, _ptr(self.pops))
        self.tmp = np.empty_like(self.pops)
        self.rho = np.ones(self.N, dtype=self.dtype)
        self.u = np.zeros(3 * self.N, dtype=self.dtype)

    def step(self, n=1):
        getattr(lib(), f"oracle_step_{self.suffix}")(ctypes.byref(self.desc), _ptr(self.flags),
                                                     _ptr(self.pops), _ptr(self.tmp),
                                                     _ptr(self.rho), _ptr(self.u), int(n))

    def rhou_fields(self, key=2):
        getattr(lib(), f"oracle_rhou_fields_{self.suffix}")(self.N, _ptr(self.flags), key,
                                                            _ptr(self.pops), _ptr(self.rho),
                                                            _ptr(self.u))
        return self.rho, self.u


def cavity(ni, model="bgk", tau=0.53, ulid=0.1, cs=0.1, mrt_rate=1.2, dtype=np.float32):
    """The reference lid-driven cavity (benchmarks/cavity3d/cavity3d.cpp:111-161)."""
    n = ni + 2
    flags = cavity_flags(ni)
    lat = Lattice(n, n, n, flags, model=model, tau=tau, cs=cs, mrt_rate=mrt_rate, dtype=dtype)
    lat.u.reshape(-1, 3)[flags == 8, 0] = lat.dtype.type(ulid)
    return lat


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
                  blockfile=None, threads=None, outdir=None):
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
