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

STORAGES = {"fp32": C.STORAGE_FP32, "fp16s": C.STORAGE_FP16S, "fp64": C.STORAGE_FP64,
            "fp32s": C.STORAGE_FP32S}
MODELS = {"bgk": C.MODEL_BGK, "mrt": C.MODEL_MRT, "les": C.MODEL_LES,
          "brinkman": C.MODEL_BRINKMAN}
FIELDS = {"rho": C.FIELD_RHO, "u": C.FIELD_VELOCITY, "alpha": C.FIELD_ALPHA}
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
    rates = [float(mrt_rate)] * 19 if np.isscalar(mrt_rate) else [float(r) for r in mrt_rate]
    assert len(rates) == 19, "mrt_rate: one rate or 19 (moment order of the D3Q19 basis)"
    for k in range(19):
        d.mrt_rates[k] = rates[k]
    d.rho0 = float(rho0)
    d.ntasks = len(tasks)
    for t, (key, op) in enumerate(tasks):
        d.task_keys[t] = int(key)
        d.task_ops[t] = OPS[op] if isinstance(op, str) else int(op)
    return d


class Lattice:
    """Device-resident D3Q19 lattice: one block (BlockLattice) or several blocks
    (BlockLatticeManager) advanced together.

    Single block:  Lattice(nx, ny, nz, tau, ...)
    Blocks:        Lattice.blocks([(nx, ny, nz, ox, oy, oz[, omega]), ...], tau, mode=...)
    Transfer methods take ``block=`` (default 0).
    """

    def __init__(self, nx, ny, nz, tau, storage="fp32", model="bgk", smagorinsky=0.1,
                 mrt_rate=1.2, rho0=1.0, tasks=CAVITY_TASKS, omega=None, _blocks=None,
                 _mode=None):
        self.storage = storage
        self.real = np.float64 if storage == "fp64" else np.float32
        self.desc = make_desc(nx, ny, nz, tau, storage, model, smagorinsky, mrt_rate, rho0,
                              tasks, omega)
        h = ctypes.c_void_p()
        if _blocks is None:
            C.call("flb_create", ctypes.byref(self.desc), ctypes.byref(h))
            self.shapes = [(int(nx), int(ny), int(nz))]
        else:
            arr = (C.BlockDesc * len(_blocks))()
            for k, b in enumerate(_blocks):
                arr[k].nx, arr[k].ny, arr[k].nz = int(b[0]), int(b[1]), int(b[2])
                arr[k].ox, arr[k].oy, arr[k].oz = int(b[3]), int(b[4]), int(b[5])
                arr[k].omega = float(b[6]) if len(b) > 6 else 0.0
            C.call("flb_create_blocks", ctypes.byref(self.desc), len(_blocks), arr,
                   int(_mode), ctypes.byref(h))
            self.shapes = [(int(b[0]), int(b[1]), int(b[2])) for b in _blocks]
        self._h = h
        self.nx, self.ny, self.nz = self.shapes[0]
        self.N = self.nx * self.ny * self.nz

    @classmethod
    def blocks(cls, blocks, tau, mode="halo", **kw):
        m = C.BLOCKS_HALO if mode == "halo" else C.BLOCKS_INDEPENDENT
        return cls(3, 3, 3, tau, _blocks=blocks, _mode=m, **kw)

    @property
    def nblocks(self):
        return len(self.shapes)

    def ncells(self, block=0):
        nx, ny, nz = self.shapes[block]
        return nx * ny * nz

    def halo_count(self):
        v = ctypes.c_longlong()
        C.call("flb_halo_count", self._h, ctypes.byref(v))
        return int(v.value)

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
    def upload_flags(self, flags, stream=None, block=0):
        f = np.ascontiguousarray(flags, dtype=np.uint8).reshape(-1)
        assert f.size == self.ncells(block)
        C.call("flb_upload_flags_block", self._h, block, _ptr(f), _stream(stream))

    def download_flags(self, stream=None, block=0):
        f = np.empty(self.ncells(block), dtype=np.uint8)
        C.call("flb_download_flags_block", self._h, block, _ptr(f), _stream(stream))
        return f

    def upload_pops(self, pops, stream=None, block=0):
        p = np.ascontiguousarray(pops).reshape(-1)
        assert p.size == 19 * self.ncells(block)
        dt = C.DTYPE_F64 if p.dtype == np.float64 else C.DTYPE_F32
        p = p.astype(np.float64 if dt == C.DTYPE_F64 else np.float32, copy=False)
        C.call("flb_upload_pops_block", self._h, block, _ptr(p), dt, _stream(stream))

    def download_pops(self, dtype=None, stream=None, block=0):
        dtype = np.dtype(dtype or self.real)
        p = np.empty(19 * self.ncells(block), dtype=dtype)
        dt = C.DTYPE_F64 if dtype == np.float64 else C.DTYPE_F32
        C.call("flb_download_pops_block", self._h, block, _ptr(p), dt, _stream(stream))
        return p

    def upload_field(self, name, values, stream=None, block=0):
        fid = FIELDS[name]
        n = self.ncells(block)
        v = np.ascontiguousarray(values).reshape(-1)
        assert v.size == (3 * n if fid == C.FIELD_VELOCITY else n)
        dt = C.DTYPE_F64 if v.dtype == np.float64 else C.DTYPE_F32
        v = v.astype(np.float64 if dt == C.DTYPE_F64 else np.float32, copy=False)
        C.call("flb_upload_field_block", self._h, block, fid, _ptr(v), dt, _stream(stream))

    def download_field(self, name, dtype=None, stream=None, block=0):
        fid = FIELDS[name]
        dtype = np.dtype(dtype or self.real)
        n = self.ncells(block)
        v = np.empty(3 * n if fid == C.FIELD_VELOCITY else n, dtype=dtype)
        dt = C.DTYPE_F64 if dtype == np.float64 else C.DTYPE_F32
        C.call("flb_download_field_block", self._h, block, fid, _ptr(v), dt, _stream(stream))
        return v

    # -- compute
    def init_equilibrium(self, rho0=1.0, stream=None):
        C.call("flb_init_equilibrium", self._h, float(rho0), _stream(stream))

    def step(self, n=1, stream=None, graph=False):
        C.call("flb_step_graph" if graph else "flb_step", self._h, int(n), _stream(stream))

    def set_launch(self, tile_y=8, ctas_per_sm=0, cells_per_thread=0):
        C.call("flb_set_launch", self._h, int(tile_y), int(ctas_per_sm), int(cells_per_thread))

    def set_wait_limit(self, seconds):
        """Bound of one device-side wait of the bulk-copy kernel (seconds)."""
        C.call("flb_set_wait_limit", self._h, float(seconds))

    def snapshot_bytes(self):
        n = ctypes.c_size_t()
        C.call("flb_snapshot_bytes", self._h, ctypes.byref(n))
        return int(n.value)

    def snapshot_save(self, ptr, cap, stream=None):
        """Copy the state (header + populations) to the buffer at address
        `ptr` (device or host) of `cap` bytes."""
        C.call("flb_snapshot_save", self._h, ctypes.c_void_p(ptr), ctypes.c_size_t(cap),
               _stream(stream))

    def snapshot_restore(self, ptr, nbytes, stream=None):
        C.call("flb_snapshot_restore", self._h, ctypes.c_void_p(ptr), ctypes.c_size_t(nbytes),
               _stream(stream))

    def set_rounding(self, mode):
        """Rounding of FP16S stores: "nearest", "stochastic" or "default"
        (stochastic for MRT, nearest otherwise)."""
        m = {"default": C.ROUND_DEFAULT, "nearest": C.ROUND_NEAREST,
             "stochastic": C.ROUND_STOCHASTIC}[mode]
        C.call("flb_set_rounding", self._h, m)

    def rounding(self):
        """The FP16S rounding in effect: "nearest" or "stochastic"."""
        v = ctypes.c_int()
        C.call("flb_get_rounding", self._h, ctypes.byref(v))
        return "stochastic" if v.value == C.ROUND_STOCHASTIC else "nearest"

    def device_status(self, stream=None):
        """Raise FlbError(FLB_ERR_TIMEOUT) if a device-side wait gave up since
        the last check (and clear it)."""
        C.call("flb_device_status", self._h, _stream(stream))

    def get_launch(self):
        """(tile_y, ctas_per_sm, cells_per_thread)."""
        a, b, v = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        C.call("flb_get_launch", self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(v))
        return a.value, b.value, v.value

    def autotune(self, trial_steps=4, stream=None):
        """Pick the fastest launch shape; returns
        ((tile_y, ctas_per_sm, cells_per_thread), ms per step, steps run)."""
        ty, c, v, steps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_double()
        C.call("flb_autotune", self._h, int(trial_steps), _stream(stream), ctypes.byref(ty),
               ctypes.byref(c), ctypes.byref(v), ctypes.byref(ms), ctypes.byref(steps))
        return (ty.value, c.value, v.value), ms.value, steps.value

    def compute_rhou(self, key=2, stream=None):
        C.call("flb_compute_rhou", self._h, int(key), _stream(stream))

    def rhou(self, key=2, dtype=None, stream=None, block=0):
        self.compute_rhou(key, stream)
        return (self.download_field("rho", dtype, stream, block),
                self.download_field("u", dtype, stream, block))

    def conservation(self, key=0xFF, stream=None):
        out = (ctypes.c_double * 4)()
        C.call("flb_reduce_conservation", self._h, int(key), out, _stream(stream))
        return np.array(out[:])

    def tolerance_u(self, key=2, stream=None):
        v = ctypes.c_double()
        C.call("flb_tolerance_u", self._h, int(key), ctypes.byref(v), _stream(stream))
        return v.value

    def nonfinite(self, stream=None):
        """Number of non-finite populations (the C call returns FLB_ERR_NUMERIC
        when it is not zero)."""
        v = ctypes.c_uint64()
        rc = C.load().flb_check_finite(self._h, ctypes.byref(v), _stream(stream))
        if rc not in (C.FLB_OK, C.ERR_NUMERIC):
            raise C.FlbError(rc, "flb_check_finite", C.load().flb_last_error().decode())
        return int(v.value)

    def set_halo_mode(self, mode):
        """"normal" (NormalCommunicate) or "full" (NormalFullCommunicate /
        NormalAllCommunicate) halo exchange of a halo-mode block handle."""
        C.call("flb_set_halo_mode", self._h, {"normal": C.HALO_NORMAL, "full": C.HALO_FULL}[mode])

    # -- VTK output
    def vtk_body(self, field, overlap=0, dtype=None, scale=None, offset=0.0, block=0,
                 stream=None):
        """Base64 body of the VTK DataArray of `field` ("rho", "u", "alpha" or
        "flag") on `block` without `overlap` layers per side, converted to
        `dtype` (float32 / float64; default: the lattice's arithmetic type) and,
        with `scale`, mapped v -> v * scale + offset in that type first: the
        characters the reference's vtmo writers put between the DataArray tags."""
        fid = C.VTK_FLAG if field == "flag" else FIELDS[field]
        dt = np.dtype(dtype or self.real)
        odt = C.DTYPE_F64 if dt == np.float64 else C.DTYPE_F32
        mp = 0 if scale is None else 1
        sc = 1.0 if scale is None else float(scale)
        n = ctypes.c_size_t()
        C.call("flb_vtk_field_base64", self._h, int(block), fid, int(overlap), odt, mp, sc,
               float(offset), None, 0, ctypes.byref(n), _stream(stream))
        buf = ctypes.create_string_buffer(n.value)
        C.call("flb_vtk_field_base64", self._h, int(block), fid, int(overlap), odt, mp, sc,
               float(offset), buf, n.value, ctypes.byref(n), _stream(stream))
        return buf.raw[:n.value].decode()

    # -- objective and discrete adjoint
    def objective_u2(self, stream=None):
        """J = sum over bulk cells of |u|^2 (forced moment with the alpha field)."""
        v = ctypes.c_double()
        C.call("flb_objective_u2", self._h, ctypes.byref(v), _stream(stream))
        return v.value

    def adjoint_forward(self, nsteps, checkpoint_every=100, stream=None):
        """Advance nsteps keeping checkpoints; returns J at the end."""
        v = ctypes.c_double()
        C.call("flb_adjoint_forward", self._h, int(nsteps), int(checkpoint_every),
               ctypes.byref(v), _stream(stream))
        return v.value

    def adjoint_backward(self, alpha_grad=True, stream=None):
        """Gradients of the last adjoint_forward objective:
        (dJ/dalpha per cell or None, dJ/dtau, dJ/du_lid)."""
        g = np.empty(self.N, dtype=np.float64) if alpha_grad else None
        t, u = ctypes.c_double(), ctypes.c_double()
        C.call("flb_adjoint_backward", self._h, _ptr(g) if g is not None else None,
               ctypes.byref(t), ctypes.byref(u), _stream(stream))
        return g, t.value, u.value

    def adjoint_release(self):
        C.call("flb_adjoint_release", self._h)

    def layout(self):
        L = C.Layout()
        C.call("flb_get_layout", self._h, ctypes.byref(L))
        return L

    def memory_bytes(self):
        v = ctypes.c_size_t()
        C.call("flb_memory_bytes", self._h, ctypes.byref(v))
        return int(v.value)


BB_KINDS = {"normal": C.BB_NORMAL, "movingwall": C.BB_MOVINGWALL,
            "anti_simple": C.BB_ANTI_SIMPLE, "anti_o1": C.BB_ANTI_O1, "anti_o2": C.BB_ANTI_O2,
            "anti_pressure": C.BB_ANTI_PRESSURE}


# NbrDirection bits (src/parallel/communicator.h:37-52)
NBR = {"XN": 1, "XP": 2, "YN": 4, "YP": 8, "ZN": 16, "ZP": 32}


class PeriodicBoundaryManager:
    """FixedPeriodicBoundaryManager on a single-block lattice
    (src/boundary/periodic_boundary.h:136-321): Setup(box0, dir0, box1, dir1)
    at construction, apply() after each step (the reference calls Apply()
    between ApplyCellDynamics and Stream; the collision is part of the step
    here).  Boxes are inclusive stored-cell ranges (x0, x1, y0, y1, z0, z1);
    directions are NbrDirection names ("XN", ...) or FLB_NBR_* bit masks."""

    def __init__(self, lattice, box0, dir0, box1, dir1, cell_flag):
        def bits(d):
            return d if isinstance(d, int) else NBR[d]
        self.lattice = lattice
        b0 = (ctypes.c_int * 6)(*[int(v) for v in box0])
        b1 = (ctypes.c_int * 6)(*[int(v) for v in box1])
        h = ctypes.c_void_p()
        C.call("flb_periodic_create", lattice._h, b0, bits(dir0), b1, bits(dir1), int(cell_flag),
               ctypes.byref(h))
        self._h = h

    def counts(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        C.call("flb_periodic_count", self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def apply(self, stream=None):
        C.call("flb_periodic_apply", self._h, self.lattice._h, _stream(stream))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            C.load().flb_periodic_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BounceBackManager:
    """Post-stream halfway bounce-back on a single-block lattice:
    BBLikeFixedBlockBdManager<bounceback::KIND<CELL>, ...> with KIND one of
    normal, movingwall, anti_simple, anti_O1, anti_O2, anti_pressure
    (src/boundary/bounce_back_boundary.h:167-256).  apply() after each step, as
    BlockBoundaryManager::Apply() after Stream()."""

    def __init__(self, lattice, cell_flag, void_flag=1, kind="normal", rho0=1.0):
        if kind not in BB_KINDS:
            raise ValueError(f"unknown bounce-back kind {kind!r}; one of {sorted(BB_KINDS)}")
        self.lattice = lattice
        self.kind = kind
        h = ctypes.c_void_p()
        C.call("flb_bb_create", lattice._h, int(cell_flag), int(void_flag), BB_KINDS[kind],
               float(rho0), ctypes.byref(h))
        self._h = h

    def counts(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        C.call("flb_bb_count", self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def apply(self, stream=None):
        C.call("flb_bb_apply", self._h, self.lattice._h, _stream(stream))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            C.load().flb_bb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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
