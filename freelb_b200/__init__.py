"""freelb_b200 -- B200 (sm_100a) D3Q19 stream-and-collide for FreeLB's hot path.

Python access to the C ABI in include/flb.h.  The compute path is the CUDA
library ``libflb_b200.so`` built in this directory; nothing here computes on
the CPU.  ``Lattice`` mirrors one ``BlockLattice`` of the reference
(src/data_struct/block_lattice.h): construct, upload flags and fields, step
(= ApplyCellDynamics<NSTask> + Stream), read populations / RHO / VELOCITY.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from ._capi import FlbError  # noqa: F401

STORAGES = {"fp32": C.STORAGE_FP32, "fp16s": C.STORAGE_FP16S, "fp64": C.STORAGE_FP64}
MODELS = {"bgk": C.MODEL_BGK, "mrt": C.MODEL_MRT, "les": C.MODEL_LES}
OPS = {"none": C.OP_NONE, "bulk": C.OP_BULK, "bounceback": C.OP_BOUNCEBACK,
       "movingwall": C.OP_MOVINGWALL, "field_bgk": C.OP_FIELD_BGK}

# the cavity benchmark's task list: {2: bulk, 4: BounceBack, 8: BounceBackMovingWall}
CAVITY_TASKS = ((2, "bulk"), (4, "bounceback"), (8, "movingwall"))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(int(stream.cuda_stream))  # torch.cuda.Stream


def version():
    a, s = ctypes.c_int(), ctypes.c_int()
    C.call("flb_version", ctypes.byref(a), ctypes.byref(s))
    return a.value, s.value


def make_desc(nx, ny, nz, tau, storage="fp32", model="bgk", smagorinsky=0.1, mrt_rate=1.2,
              rho0=1.0, tasks=CAVITY_TASKS, omega=None):
    d = C.LatticeDesc()
    C.call("flb_desc_default", ctypes.byref(d), nx, ny, nz, float(tau))
    d.storage = STORAGES[storage]
    d.model = MODELS[model]
    if omega is not None:
        d.omega = float(omega)
    d.smagorinsky = float(smagorinsky)
    for k in range(19):
        d.mrt_rates[k] = float(mrt_rate)
    d.rho0 = float(rho0)
    d.ntasks = len(tasks)
    for t, (key, op) in enumerate(tasks):
        d.task_keys[t] = int(key)
        d.task_ops[t] = OPS[op] if isinstance(op, str) else int(op)
    return d


class Lattice:
    """One device-resident D3Q19 block lattice (BlockLattice on the GPU)."""

    def __init__(self, nx, ny, nz, tau, storage="fp32", model="bgk", smagorinsky=0.1,
                 mrt_rate=1.2, rho0=1.0, tasks=CAVITY_TASKS, omega=None):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.N = self.nx * self.ny * self.nz
        self.storage = storage
        self.desc = make_desc(nx, ny, nz, tau, storage, model, smagorinsky, mrt_rate, rho0,
                              tasks, omega)
        h = ctypes.c_void_p()
        C.call("flb_create", ctypes.byref(self.desc), ctypes.byref(h))
        self._h = h
        self.real = np.float64 if storage == "fp64" else np.float32

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            C.load().flb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- transfers
    def upload_flags(self, flags, stream=None):
        f = np.ascontiguousarray(flags, dtype=np.uint8).reshape(-1)
        assert f.size == self.N
        C.call("flb_upload_flags", self._h, _ptr(f), _stream(stream))

    def download_flags(self, stream=None):
        f = np.empty(self.N, dtype=np.uint8)
        C.call("flb_download_flags", self._h, _ptr(f), _stream(stream))
        return f

    def upload_pops(self, pops, stream=None):
        p = np.ascontiguousarray(pops).reshape(-1)
        assert p.size == 19 * self.N
        dt = C.DTYPE_F64 if p.dtype == np.float64 else C.DTYPE_F32
        p = p.astype(np.float64 if dt == C.DTYPE_F64 else np.float32, copy=False)
        C.call("flb_upload_pops", self._h, _ptr(p), dt, _stream(stream))

    def download_pops(self, dtype=None, stream=None):
        dtype = np.dtype(dtype or self.real)
        p = np.empty(19 * self.N, dtype=dtype)
        dt = C.DTYPE_F64 if dtype == np.float64 else C.DTYPE_F32
        C.call("flb_download_pops", self._h, _ptr(p), dt, _stream(stream))
        return p

    def upload_field(self, name, values, stream=None):
        fid = C.FIELD_RHO if name == "rho" else C.FIELD_VELOCITY
        v = np.ascontiguousarray(values).reshape(-1)
        assert v.size == (self.N if fid == C.FIELD_RHO else 3 * self.N)
        dt = C.DTYPE_F64 if v.dtype == np.float64 else C.DTYPE_F32
        v = v.astype(np.float64 if dt == C.DTYPE_F64 else np.float32, copy=False)
        C.call("flb_upload_field", self._h, fid, _ptr(v), dt, _stream(stream))

    def download_field(self, name, dtype=None, stream=None):
        fid = C.FIELD_RHO if name == "rho" else C.FIELD_VELOCITY
        dtype = np.dtype(dtype or self.real)
        v = np.empty(self.N if fid == C.FIELD_RHO else 3 * self.N, dtype=dtype)
        dt = C.DTYPE_F64 if dtype == np.float64 else C.DTYPE_F32
        C.call("flb_download_field", self._h, fid, _ptr(v), dt, _stream(stream))
        return v

    # -- compute
    def init_equilibrium(self, rho0=1.0, stream=None):
        C.call("flb_init_equilibrium", self._h, float(rho0), _stream(stream))

    def step(self, n=1, stream=None):
        C.call("flb_step", self._h, int(n), _stream(stream))

    def compute_rhou(self, key=2, stream=None):
        C.call("flb_compute_rhou", self._h, int(key), _stream(stream))

    def rhou(self, key=2, dtype=None, stream=None):
        self.compute_rhou(key, stream)
        return self.download_field("rho", dtype, stream), self.download_field("u", dtype, stream)

    def conservation(self, key=0xFF, stream=None):
        out = (ctypes.c_double * 4)()
        C.call("flb_reduce_conservation", self._h, int(key), out, _stream(stream))
        return np.array(out[:])

    def tolerance_u(self, key=2, stream=None):
        v = ctypes.c_double()
        C.call("flb_tolerance_u", self._h, int(key), ctypes.byref(v), _stream(stream))
        return v.value

    def nonfinite(self, stream=None):
        v = ctypes.c_uint64()
        C.call("flb_check_finite", self._h, ctypes.byref(v), _stream(stream))
        return int(v.value)

    def layout(self):
        L = C.Layout()
        C.call("flb_get_layout", self._h, ctypes.byref(L))
        return L

    def memory_bytes(self):
        v = ctypes.c_size_t()
        C.call("flb_memory_bytes", self._h, ctypes.byref(v))
        return int(v.value)


def cavity_flags(ni: int) -> np.ndarray:
    """Flags of the reference lid-driven cavity on the stored (ni+2)^3 mesh.

    benchmarks/cavity3d/cavity3d.cpp:136-142 with cell centres at idx - 0.5
    (Cell_Len = 1): 2 inside [1, ni]^3, 4 on that region's outer layer, 8 on its
    top layer for 2 <= x, y <= ni-1, 1 elsewhere.
    """
    n = ni + 2
    f = np.ones((n, n, n), dtype=np.uint8)
    f[1:n - 1, 1:n - 1, 1:n - 1] = 4
    f[2:n - 2, 2:n - 2, 2:n - 2] = 2
    f[n - 2, 2:n - 2, 2:n - 2] = 8
    return f.reshape(-1)


def cavity(ni, tau=0.53, ulid=0.1, storage="fp32", model="bgk", smagorinsky=0.1, mrt_rate=1.2):
    """Set up the reference lid-driven cavity (cavity3d.cpp:111-161) on the device."""
    n = ni + 2
    lat = Lattice(n, n, n, tau, storage=storage, model=model, smagorinsky=smagorinsky,
                  mrt_rate=mrt_rate)
    flags = cavity_flags(ni)
    lat.upload_flags(flags)
    real = lat.real
    u = np.zeros((lat.N, 3), dtype=real)
    u[flags == 8, 0] = real(ulid)
    lat.upload_field("u", u)
    return lat
