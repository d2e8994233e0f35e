"""Benchmark: D3Q19 lid-driven cavity stream-and-collide on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--ni 512]

Workload (per GPU): the reference's lid-driven cavity (benchmarks/cavity3d)
scaled to 512^3 interior cells (514^3 = 135.8 M stored cells incl. the void
layer), D3Q19 BGK, tau = 0.53, u_lid = 0.1, FP32 populations.  One step = one
fused stream+collide launch over the whole lattice (ApplyCellDynamics<NSTask>
+ Stream in the reference).  GLUPs = stored cells x steps / s / 1e9, counting
cells like the reference (Geo.getTotalCellNum(), void layer included).

The working set (2 x 19 x 4 B x 143.7 M padded cells = 21.8 GB) is far larger
than L2 (126 MB), so no L2 flush is needed between timed steps.

Multi-GPU (torchrun): every rank runs its own independent cavity (replicas,
weak scaling; no collective on the data path).  Time = max over ranks.

--impl reference runs the reference FreeLB CPU path itself (oracle/_ref,
compiled from the reference sources) on this host's cores, on the same
cavity; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

Q = 19
BYTES_PER_POP = {"fp32": 4, "fp16s": 2, "fp64": 8, "fp32s": 4}
CPU_BASELINE_STEPS = 20   # ~8 s of the reference's OpenMP path at 512^3 on 16 host cores
MRT_PARITY_STEPS = 20     # the reference's generic MRT runs ~3 s per 256^3 step on 14 cores


def algo_bytes_per_cell(storage: str) -> int:
    """2*Q*s + 1: read and write every population once, read the flag byte."""
    return 2 * Q * BYTES_PER_POP[storage] + 1


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(key: str):
    """DRAM bytes per cell from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(key)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"flb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        # nvidia-smi takes a moment to start: begin the timed region only once
        # it is sampling (at most 10 s)
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for ln in f:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "samples": len(sm), "reasons": sorted(reasons)}


# --------------------------------------------------------------------------- reference arm

def reference_cpu(ni: int, steps: int, warmup: int, threads=None):
    """Run the reference CPU path (oracle/_ref) on the cavity; returns dict or None."""
    from oracle import oracle as O
    exe = O.ref_binary(np.float32)
    if exe is None:
        return None
    r = O.run_reference("bgk", ni, 0.53, 0.1, steps, warmup, threads=threads, outdir="-")
    return {"mlups": r["mlups"], "seconds": r["seconds"], "threads": r["threads"],
            "binary": os.path.basename(exe)}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    ni = args.ni
    cells = (ni + 2) ** 3
    steps = max(1, min(args.steps, 20))
    warm = args.warmup
    r = reference_cpu(ni, steps, warm)
    base = {"impl": "reference", "metric": "D3Q19 cavity GLUPs (stored cells)", "unit": "GLUPs",
            "n_gpus": args.gpus, "higher_is_better": True}
    if r is None:
        base["unavailable"] = "reference harness oracle/_ref not built on this machine"
        print(json.dumps(base))
        return
    v = r["mlups"] / 1000.0
    base.update({
        "value": v, "steps": steps, "warmup": warm, "steps_requested": args.steps,
        "ms_per_step": 1000.0 * r["seconds"] / steps, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"lid-driven cavity {ni}^3 D3Q19 BGK tau=0.53 u_lid=0.1",
                   "stored_cells": cells, "storage": "fp32"},
        "cpu_baseline": {"value": v, "unit": "GLUPs", "cores": r["threads"], "kind": "reference",
                         "sample": f"{steps} timed steps (+{warm} warm-up) of the {ni}^3 cavity, "
                                   f"reference FreeLB OpenMP path ({r['binary']})"},
        "e2e": {"value": v, "unit": "GLUPs", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(base))


# --------------------------------------------------------------------------- our arm

def compact(v, digits=4):
    """Floats rounded to `digits` significant digits, recursively (keeps the
    JSON line short enough to be read whole from a log tail)."""
    if isinstance(v, float):
        return float(f"{v:.{digits}g}") if np.isfinite(v) else v
    if isinstance(v, dict):
        return {k: compact(x, digits) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [compact(x, digits) for x in v]
    return v


def max_over_ranks(torch, dist, value, device):
    """Largest value over all ranks (the job time of independent replicas)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class DeviceTimer:
    """CUDA events on the launching stream, synchronised on both sides."""

    def __init__(self, torch, stream):
        self.torch, self.stream = torch, stream

    def __enter__(self):
        self.torch.cuda.synchronize()
        self.e0 = self.torch.cuda.Event(enable_timing=True)
        self.e1 = self.torch.cuda.Event(enable_timing=True)
        self.e0.record(self.stream)
        return self

    def __exit__(self, *exc):
        self.e1.record(self.stream)
        self.torch.cuda.synchronize()
        self.ms = self.e0.elapsed_time(self.e1)


def timed_cavity(F, torch, stream, ni, steps, warmup, storage="fp32", model="bgk", tune=True,
                 tau=0.53, smagorinsky=0.1, rounding="default"):
    """Cavity of ni^3 interior cells: autotune the launch shape (the tuning steps
    are real warm-up steps), then time `steps` steps.  Returns (ms, launch, lat)."""
    lat = F.cavity(ni, tau=tau, ulid=0.1, storage=storage, model=model, smagorinsky=smagorinsky)
    lat.set_rounding(rounding)
    launch = None
    if tune:
        launch, _, _ = lat.autotune(trial_steps=2, stream=stream)
    for _ in range(warmup):
        lat.step(1, stream)
    with DeviceTimer(torch, stream) as t:
        lat.step(steps, stream)
    return t.ms, launch, lat


W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def round_once_fp16s(pops):
    """Every population's deviation from its lattice weight rounded once, in
    place, to FP16S precision: binary16 of (f - w) * 2^10, read back in FP64
    (direction by direction, in 16M-cell pieces, so a 512^3 lattice needs no
    second full-size host array)."""
    p = pops.reshape(19, -1)
    out_of_range = 0  # |f - w| * 2^10 beyond binary16 (FP16S storage would hold inf there)
    for i, wi in enumerate(W19):
        for s in range(0, p.shape[1], 1 << 24):
            seg = p[i, s:s + (1 << 24)]
            d = (seg - wi) * 1024.0
            out_of_range += int(np.count_nonzero(~(np.abs(d) <= 65504.0)))
            with np.errstate(over="ignore", invalid="ignore"):
                seg[:] = d.astype(np.float16).astype(np.float64) / 1024.0 + wi
    return out_of_range


def accuracy_block(F, ni, steps, keep_bgk_fp32=False, models=("bgk", "mrt", "les")):
    """Relative L2 error of u after `steps` steps against an FP64 run of the same
    kernel, per model and storage (C2 accuracy report).  Beside it, the flow's
    own sensitivity: an FP64 run whose populations are rounded once to FP16S
    precision at step steps/2 (FP16S storage rounds at that precision every
    step), and for LES two FP64 runs whose initial populations differ by 1e-7
    and 2^-12 (relative, seeded).  With keep_bgk_fp32 the FP32 BGK populations
    (reference order) are returned for the parity check against the
    reference's own FP32 run."""
    out, kept = {}, None
    taus = {"bgk": 0.53, "mrt": 0.53, "les": 3 * 0.1 * ni / 10000 + 0.5}
    for model, tau in ((m, taus[m]) for m in models):
        us = {}
        other = "nearest" if model == "mrt" else "stochastic"
        for storage in ("fp64", "fp32", "fp32s", "fp16s") + (("fp16s_" + other,) if other else ()):
            lat = F.cavity(ni, tau=tau, ulid=0.1, storage=storage.split("_")[0], model=model)
            lat.set_rounding(other if "_" in storage else "default")
            lat.step(steps)
            _, u = lat.rhou(key=2, dtype=np.float64)
            us[storage] = u
            if keep_bgk_fp32 and model == "bgk" and storage == "fp32":
                kept = (lat.download_pops(), lat.download_field("rho"), u.astype(np.float32))
            lat.close()
        ref = np.linalg.norm(us["fp64"])
        out[model] = {"tau": tau, **{f"{s}_rel_l2_u": float(np.linalg.norm(us[s] - us["fp64"]) / ref)
                                     for s in us if s != "fp64"}}
        out[model]["fp16s_rounding"] = "stochastic" if model == "mrt" else "nearest"
        if keep_bgk_fp32 and model == "bgk":
            kept = kept + (us["fp64"],)
        lat = F.cavity(ni, tau=tau, ulid=0.1, storage="fp64", model=model)
        lat.step(steps // 2)
        pops = lat.download_pops(np.float64)
        beyond = round_once_fp16s(pops)
        lat.upload_pops(pops)
        del pops
        lat.step(steps - steps // 2)
        _, u = lat.rhou(key=2, dtype=np.float64)
        lat.close()
        out[model]["fp64_one_fp16s_rounding_rel_l2_u"] = float(np.linalg.norm(u - us["fp64"]) / ref)
        if beyond:
            out[model]["fp64_values_beyond_fp16s"] = beyond
        del u
        if model == "les":
            # FP64 runs from initial populations perturbed by eps (relative,
            # seeded): 1e-7, and 2^-12, the rounding of one FP16 store
            n = ni + 2
            w = np.repeat(W19, n ** 3)
            xi = np.random.default_rng(123).standard_normal(19 * n ** 3)
            for name, eps in (("1e-7", 1e-7), ("2^-12", 2.0 ** -12)):
                lat = F.cavity(ni, tau=tau, ulid=0.1, storage="fp64", model=model)
                lat.upload_pops(w * (1.0 + eps * xi))
                lat.step(steps)
                _, u = lat.rhou(key=2, dtype=np.float64)
                lat.close()
                out[model][f"fp64_perturbed_{name}_rel_l2_u"] = float(
                    np.linalg.norm(u - us["fp64"]) / ref)
        del us
    res = {"config": f"{ni}^3 cavity, {steps} steps, u_lid=0.1 (LES: Cs=0.1, Re=10000)",
           "models": out}
    return (res, kept) if keep_bgk_fp32 else res


class ReferenceParity:
    """The reference's own FP32 CPU path (oracle/_ref) on the 256^3 cavity, run in
    a background process while the GPU sections run: BGK for the full 2000 steps
    of the accuracy run, MRT (26x slower per cell in the reference's generic
    MRT_Feq_RhoU) for a bounded number of steps.  compare() checks the GPU's FP32
    results against its dumps (relative max-norm over every cell)."""

    def __init__(self, ni, bgk_steps, mrt_steps):
        import tempfile
        import threading
        from oracle import oracle as O
        self.O = O
        self.ni, self.bgk_steps, self.mrt_steps = ni, bgk_steps, mrt_steps
        self.dir = tempfile.TemporaryDirectory(prefix="flb_refpar_")
        self.res, self.err = {}, None
        self.threads = max(1, (os.cpu_count() or 2) - 2)  # leave the GPU driver thread a core
        if O.ref_binary(np.float32) is None:
            self.err = "reference harness oracle/_ref not built"
            self.t = None
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        try:
            for model, steps in (("bgk", self.bgk_steps), ("mrt", self.mrt_steps)):
                d = os.path.join(self.dir.name, model)
                os.makedirs(d)
                t0 = time.time()
                r = self.O.run_reference(model, self.ni, 0.53, 0.1, steps, 0, threads=self.threads,
                                         outdir=d)
                self.res[model] = {"dump": d, "seconds": time.time() - t0, "mlups": r["mlups"]}
        except Exception as e:  # reported in the bench line
            self.err = f"{type(e).__name__}: {e}"

    def compare(self, model, pops, rho, u, u64=None):
        """Relative max-norms (populations on every cell, rho and u on fluid
        cells) of the GPU's FP32 run against the reference's; with u64 (the
        GPU's FP64 run, which equals the reference's FP64 path), the relative
        L2 distance of u from it for both FP32 runs."""
        if self.t is not None:
            self.t.join()
        if model not in self.res:
            return {"unavailable": self.err or "not run"}
        r = self.O.load_dump(self.res[model]["dump"], np.float32)
        flags = r["flags"]
        fl = flags == 2
        ru = r["u"].reshape(-1, 3)[fl].astype(np.float64)
        out = {"steps": self.bgk_steps if model == "bgk" else self.mrt_steps,
               "ref_threads": self.threads, "ref_seconds": self.res[model]["seconds"],
               "pops": self.O.rel_maxnorm(pops, r["pops"]),
               "rho_fluid": self.O.rel_maxnorm(rho[fl], r["rho"][fl]),
               "u_fluid": self.O.rel_maxnorm(u.reshape(-1, 3)[fl], ru)}
        if u64 is not None:
            v = u64.reshape(-1, 3)[fl]
            nv = np.linalg.norm(v)
            out["ref_fp32_vs_fp64_rel_l2_u"] = float(np.linalg.norm(ru - v) / nv)
            out["ours_fp32_vs_fp64_rel_l2_u"] = float(
                np.linalg.norm(u.reshape(-1, 3)[fl].astype(np.float64) - v) / nv)
        return out

    def close(self):
        if self.t is not None:
            self.t.join()
        self.dir.cleanup()


def blocks_block(F, torch, stream, ni, steps, seed=0):
    """Uneven-block 256^3 cavity with device halos, timed, then checked against
    the single-block run of the same number of steps: flags equal, and the
    populations of every fluid cell (max relative difference; bit-for-bit by
    construction)."""
    from freelb_b200 import geometry as G
    blocks = G.uneven_blocks(ni, edges=(32, 48, 64, 96), seed=seed)
    n = ni + 2
    flags = F.cavity_flags(ni)
    lat = F.Lattice.blocks(G.block_tuples(blocks), 0.53, mode="halo")
    u = np.zeros((n ** 3, 3), dtype=np.float32)
    u[flags == 8, 0] = np.float32(0.1)
    for k, b in enumerate(blocks):
        lat.upload_flags(G.slice_block(flags, n, b), block=k)
        lat.upload_field("u", G.slice_block(u, n, b, comps=3), block=k)
    launch, _, taken = lat.autotune(trial_steps=2, stream=stream)
    with DeviceTimer(torch, stream) as t:
        lat.step(steps, stream)
    stored = sum(b["nx"] * b["ny"] * b["nz"] for b in blocks)
    res = {"blocks": len(blocks), "stored_cells": stored, "halo_records": lat.halo_count(),
           "launch": launch, "glups_stored": stored * steps / (t.ms / 1e3) / 1e9,
           "glups_domain": n ** 3 * steps / (t.ms / 1e3) / 1e9}
    one = F.cavity(ni, tau=0.53, ulid=0.1)
    one.step(taken + steps, stream)
    P = one.download_pops().reshape(19, n, n, n)
    one.close()
    flags_ok, diff, cells = True, 0.0, 0
    pmax = float(np.max(np.abs(P)))
    for k, b in enumerate(blocks):
        fb = lat.download_flags(block=k).reshape(b["nz"], b["ny"], b["nx"])
        fg = G.slice_block(flags, n, b).reshape(b["nz"], b["ny"], b["nx"])
        flags_ok &= bool(np.array_equal(fb, fg))
        pb = lat.download_pops(block=k).reshape(19, b["nz"], b["ny"], b["nx"])
        ps = P[:, b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"], b["ox"]:b["ox"] + b["nx"]]
        m = fg == 2
        d = np.abs(pb[:, m].astype(np.float64) - ps[:, m])
        diff = max(diff, float(d.max()) if d.size else 0.0)
        cells += int(m.sum())
    lat.close()
    res.update({"check_steps": taken + steps, "flags_equal": flags_ok, "fluid_cells": cells,
                "fluid_pops_max_rel_diff": diff / pmax})
    return res


def ensemble_block(F, torch, stream, steps=1000, count=128, seed=0):
    """128 independent cavities (n ~ U{32..128}, Re ~ logU[100, 3000],
    tau = 3 u_lid n / Re + 0.5) in one multi-block handle (tile work table,
    autotuned, CUDA-graph stepping) against one handle per cavity stepped one
    after another, for FP32 and FP16S storage; 1000 steps each, as the
    ensemble configuration asks (~10 s of GPU time for all four runs)."""
    rng = np.random.default_rng(seed)
    sizes = [int(v) for v in rng.integers(32, 129, size=count)]
    res_ = np.exp(rng.uniform(np.log(100.0), np.log(3000.0), size=count))
    taus = [3 * 0.1 * n / r + 0.5 for n, r in zip(sizes, res_)]
    cells = sum((n + 2) ** 3 for n in sizes)
    out = {"cavities": count, "stored_cells": cells, "steps": steps}
    for storage in ("fp32", "fp16s"):
        lat = F.Lattice.blocks([(n + 2, n + 2, n + 2, 0, 0, 0, 1.0 / t)
                                for n, t in zip(sizes, taus)], 0.6, mode="independent",
                               storage=storage)
        for k, n in enumerate(sizes):
            fl = F.cavity_flags(n)
            u = np.zeros(((n + 2) ** 3, 3), dtype=lat.real)
            u[fl == 8, 0] = lat.real(0.1)
            lat.upload_flags(fl, block=k)
            lat.upload_field("u", u, block=k)
        launch, _, _ = lat.autotune(trial_steps=2, stream=stream)
        lat.step(2, stream, graph=True)
        with DeviceTimer(torch, stream) as t:
            lat.step(steps, stream, graph=True)
        out[storage] = {"batched_glups": cells * steps / (t.ms / 1e3) / 1e9, "launch": launch}
        lat.close()
        # one-at-a-time: a handle per cavity, each stepped `steps` times in turn
        lats = [F.cavity(n, tau=t, ulid=0.1, storage=storage) for n, t in zip(sizes, taus)]
        for one in lats:
            one.step(1, stream)
        with DeviceTimer(torch, stream) as t:
            for _ in range(steps):
                for one in lats:
                    one.step(1, stream)
        out[storage]["sequential_glups"] = cells * steps / (t.ms / 1e3) / 1e9
        for one in lats:
            one.close()
    return out


def adjoint_block(F, torch, stream, ni=128, steps=2000, every=100, fd_cells=32, seed=0):
    """128^3 cavity, Re = 500 (tau = 3*0.1*128/500 + 0.5), porosity alpha ~
    U[0, 0.05]; J = sum |u|^2 at T = 2000; checkpoints every 100 steps; FP32
    forward and adjoint, FP64 gradient accumulation.  Two FP32 storage forms:
    FP32S (deviations f - w, the form the gradient bar is met with) and FP32
    storage of f.  Per form: the backward-to-forward time ratio, the full
    gradient (checkpointed forward + backward) against a plain forward, and the
    gradient's relative error against FP64 central differences (h = 1e-4) on 32
    seeded fluid cells, on tau and on u_lid.  The timed pair is the second one
    on the handle (the first allocates the checkpoints)."""
    tau = 3 * 0.1 * ni / 500 + 0.5
    n = ni + 2
    alpha = np.random.default_rng(seed).uniform(0.0, 0.05, size=n ** 3)

    def lattice(storage, a=alpha, t=tau, ulid=0.1):
        lat = F.cavity(ni, tau=t, ulid=ulid, storage=storage, model="brinkman")
        lat.upload_field("alpha", a.astype(lat.real))
        return lat

    def J(a=alpha, t=tau, ulid=0.1):
        m = lattice("fp64", a, t, ulid)
        m.step(steps, stream)
        v = m.objective_u2(stream)
        m.close()
        return v

    h = 1e-4
    flags = F.cavity_flags(ni)
    fluid = np.flatnonzero(flags == 2)
    cells = np.random.default_rng(seed + 1).choice(fluid, size=fd_cells, replace=False)
    fds = []
    for c in cells:
        ap, am = alpha.copy(), alpha.copy()
        ap[c] += h
        am[c] -= h
        fds.append((J(ap) - J(am)) / (2 * h))
    fds = np.array(fds)
    fd_tau = (J(t=tau + h) - J(t=tau - h)) / (2 * h)
    fd_ulid = (J(ulid=0.1 + h) - J(ulid=0.1 - h)) / (2 * h)
    out = {"config": f"{ni}^3, T={steps}, checkpoints every {every}, tau={tau:.4f}",
           "fd_cells": int(fd_cells), "dJ_dtau_fd": fd_tau, "dJ_dulid_fd": fd_ulid}
    for storage in ("fp32s", "fp32"):
        lat = lattice(storage)
        lat.step(2, stream)
        with DeviceTimer(torch, stream) as tf:
            lat.step(steps, stream)
        lat.close()
        lat = lattice(storage)
        lat.adjoint_forward(steps, every, stream)
        lat.adjoint_backward(stream=stream)
        lat.init_equilibrium(1.0, stream)  # back to the initial state, buffers kept
        with DeviceTimer(torch, stream) as tfc:
            lat.adjoint_forward(steps, every, stream)
        with DeviceTimer(torch, stream) as tb:
            g_alpha, g_tau, g_ulid = lat.adjoint_backward(stream=stream)
        lat.close()
        errs = np.abs(g_alpha[cells] - fds) / np.abs(fds)
        out[storage] = {
            "forward_ms_per_step": tf.ms / steps,
            "forward_with_checkpoints_ms_per_step": tfc.ms / steps,
            "backward_ms_per_step": tb.ms / steps,
            "adjoint_to_forward_ratio": tb.ms / tf.ms,
            "full_gradient_to_forward_ratio": (tfc.ms + tb.ms) / tf.ms,
            "dJ_dtau": g_tau, "dJ_dulid": g_ulid,
            "fd_rel_err_alpha_max": float(np.max(errs)),
            "fd_rel_err_alpha_median": float(np.median(errs)),
            "fd_rel_err_alpha_normwise": float(np.linalg.norm(g_alpha[cells] - fds) /
                                               np.linalg.norm(fds)),
            "fd_cells_above_1e-4": int(np.sum(errs > 1e-4)),
            "fd_rel_err_tau": float(abs(g_tau - fd_tau) / abs(fd_tau)),
            "fd_rel_err_ulid": float(abs(g_ulid - fd_ulid) / abs(fd_ulid))}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import freelb_b200 as F

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    ni = args.ni
    n = ni + 2
    cells = n ** 3
    stream = torch.cuda.current_stream(dev)

    # headline: 512^3 BGK FP32, launch shape from the autotuner
    htau = 3 * 0.1 * ni / 10000 + 0.5 if args.model == "les" else 0.53
    lat = F.cavity(ni, tau=htau, ulid=0.1, storage=args.storage, model=args.model)
    lat.set_rounding(args.rounding)
    if args.launch:
        launch = tuple(int(v) for v in args.launch.split(","))
        lat.set_launch(*launch)
    else:
        launch, _, _ = lat.autotune(trial_steps=2, stream=stream)
    for _ in range(args.warmup):
        lat.step(1, stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as cs:
        with DeviceTimer(torch, stream) as t:
            lat.step(args.steps, stream)
    ms32 = max_over_ranks(torch, dist, t.ms, dev)
    clocks = cs.summary()
    bad32 = lat.nonfinite()
    lat.close()

    # end to end through the public API with host buffers: flags + lid velocity
    # field in from pinned host memory, K steps, RHO and VELOCITY back out.
    flags = F.cavity_flags(ni)
    u0 = np.zeros((cells, 3), dtype=np.float32)
    u0[flags == 8, 0] = np.float32(0.1)
    pin_flags = torch.from_numpy(flags).pin_memory().numpy()
    pin_u = torch.from_numpy(u0.reshape(-1)).pin_memory().numpy()
    out_rho = torch.empty(cells, dtype=torch.float32).pin_memory().numpy()
    out_u = torch.empty(3 * cells, dtype=torch.float32).pin_memory().numpy()
    if args.storage == "fp64":
        pin_u = torch.from_numpy(u0.reshape(-1).astype(np.float64)).pin_memory().numpy()
    lat = F.Lattice(n, n, n, 0.53, storage=args.storage)
    lat.set_launch(*launch)
    lat.step(1, stream)  # first-launch costs outside the timed region
    lat.init_equilibrium(1.0, stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    with DeviceTimer(torch, stream) as te:
        lat.upload_flags(pin_flags, stream)
        lat.upload_field("u", pin_u, stream)
        lat.step(args.steps, stream)
        lat.compute_rhou(2, stream)
        import ctypes
        from freelb_b200 import _capi as C
        C.call("flb_download_field", lat._h, C.FIELD_RHO, ctypes.c_void_p(out_rho.ctypes.data),
               C.DTYPE_F32, ctypes.c_void_p(stream.cuda_stream))
        C.call("flb_download_field", lat._h, C.FIELD_VELOCITY,
               ctypes.c_void_p(out_u.ctypes.data), C.DTYPE_F32,
               ctypes.c_void_p(stream.cuda_stream))
    e2e_ms = max_over_ranks(torch, dist, max(te.ms, (time.perf_counter() - t0) * 1000.0), dev)
    lat.close()
    h2d = flags.nbytes + u0.nbytes
    d2h = out_rho.nbytes + out_u.nbytes

    # the reference's CPU path on the same cavity (host cores, bounded sample),
    # before any background CPU work starts
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_cpu(ni, CPU_BASELINE_STEPS, 0)

    extras = {}
    if world == 1 and not args.quick:
        par_ni = 256
        refpar = ReferenceParity(par_ni, 2000, MRT_PARITY_STEPS) if not args.no_parity else None
        # other models and storages on the same 512^3 cavity
        variants = {}
        les_tau = 3 * 0.1 * ni / 10000 + 0.5
        for storage, model, tau, rnd in (("fp16s", "bgk", 0.53, "default"),
                                         ("fp16s", "bgk", 0.53, "stochastic"),
                                         ("fp32", "mrt", 0.53, "default"),
                                         ("fp16s", "mrt", 0.53, "default"),
                                         ("fp16s", "mrt", 0.53, "nearest"),
                                         ("fp32", "les", les_tau, "default"),
                                         ("fp16s", "les", les_tau, "default"),
                                         ("fp16s", "les", les_tau, "stochastic"),
                                         ("fp64", "bgk", 0.53, "default"),
                                         ("fp32s", "bgk", 0.53, "default")):
            ms, lch, vl = timed_cavity(F, torch, stream, ni, args.steps, 2, storage, model,
                                       tau=tau, rounding=rnd)
            bad = vl.nonfinite()
            used = vl.rounding()
            vl.close()
            b = algo_bytes_per_cell(storage)
            ach = cells * b / (ms / args.steps / 1e3) / 1e9
            key = f"{model}_{storage}" + ("" if rnd == "default" else f"_{rnd}")
            variants[key] = {
                "glups": cells * args.steps / (ms / 1e3) / 1e9, "frac": ach / measured_peaks()[0],
                "launch": lch, "nonfinite": bad}
            if storage == "fp16s":
                variants[key]["rounding"] = used
        extras["variants"] = variants
        acc = accuracy_block(F, args.accuracy_ni, args.accuracy_steps,
                             keep_bgk_fp32=args.accuracy_ni == par_ni and args.accuracy_steps == 2000,
                             models=tuple(args.accuracy_models.split(",")))
        extras["accuracy"], kept = acc if isinstance(acc, tuple) else (acc, None)
        extras["blocks_256"] = blocks_block(F, torch, stream, 256, args.steps)
        extras["ensemble_128"] = ensemble_block(F, torch, stream)
        extras["adjoint_128"] = adjoint_block(F, torch, stream)
        if refpar is not None:
            par = {}
            if kept is not None:
                par["bgk_fp32"] = refpar.compare("bgk", *kept)
            del kept
            m = F.cavity(par_ni, tau=0.53, ulid=0.1, storage="fp32", model="mrt")
            m.step(MRT_PARITY_STEPS, stream)
            rho, u = m.rhou(key=2)
            par["mrt_fp32"] = refpar.compare("mrt", m.download_pops(), rho, u)
            m.close()
            refpar.close()
            extras["parity_256_vs_reference"] = par

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    peak, peak_kind = measured_peaks()
    glups32 = cells * args.steps * world / (ms32 / 1000.0) / 1e9
    b32 = algo_bytes_per_cell(args.storage)
    per_launch_ms32 = ms32 / args.steps
    ach32 = cells * b32 / (per_launch_ms32 / 1000.0) / 1e9
    tr32 = profile_traffic(f"{args.storage}_bgk_bytes_per_cell")
    line = {
        "metric": "D3Q19 cavity GLUPs (stored cells)",
        "value": glups32,
        "unit": "GLUPs",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms32 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"fp32": "f32", "fp16s": "f32 (fp16 storage)", "fp64": "f64",
                  "fp32s": "f32 (fp32 deviation storage)"}[args.storage],
        "data": "synthetic",
        "config": {"workload": f"lid-driven cavity {ni}^3 D3Q19 {args.model.upper()} "
                               f"tau={htau:g} u_lid=0.1",
                   "stored_cells": cells, "storage": args.storage, "per_gpu": "independent cavity",
                   "l2": "working set 21.8 GB >> 126 MB L2; no flush needed",
                   "parallelism": f"replicas x{world}", "launch": launch},
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s",
                     "frac": ach32 / peak, "peak_source": peak_kind,
                     "traffic": (tr32 * cells if tr32 else None),
                     "traffic_note": "DRAM bytes per cell of an ncu capture of the 202^3 cavity "
                                     "(profiles/traffic.json) times the stored cells: the "
                                     "traffic grows in proportion to the cells",
                     "algorithmic_bytes_per_cell": b32},
        "e2e": {"value": cells * args.steps * world / (e2e_ms / 1000.0) / 1e9, "unit": "GLUPs",
                "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "job": "flags + VELOCITY in (pinned host), K steps, RHO + VELOCITY out"},
        "gpu_launches": args.steps,
        "nonvoid_glups": ni ** 3 * args.steps * world / (ms32 / 1e3) / 1e9,
        "clocks": clocks,
        "nonfinite": bad32,
    }
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["mlups"] / 1000.0, "unit": "GLUPs",
                                "cores": cpu["threads"], "kind": "reference",
                                "sample": f"{CPU_BASELINE_STEPS} timed steps of the {ni}^3 cavity "
                                          f"on the reference FreeLB OpenMP path ({cpu['binary']})"}
    line.update(extras)
    if extras:
        line["summary"] = summary_of(line)
    print(json.dumps(compact(line)))


def summary_of(line):
    """The secondary figures in a few hundred characters, last on the line (a
    log tail that cuts the line keeps them)."""
    out = {}
    v = line.get("variants", {})
    out["glups"] = {"bgk": [line["value"], v.get("bgk_fp16s", {}).get("glups")],
                    "mrt": [v.get("mrt_fp32", {}).get("glups"), v.get("mrt_fp16s", {}).get("glups")],
                    "les": [v.get("les_fp32", {}).get("glups"), v.get("les_fp16s", {}).get("glups")],
                    "order": "fp32, fp16s (default rounding)"}
    out["roofline_frac_fp16s"] = {m: v.get(f"{m}_fp16s", {}).get("frac") for m in ("bgk", "mrt", "les")}
    acc = line.get("accuracy", {}).get("models", {})
    out["fp16s_rel_l2_u"] = {m: acc[m].get("fp16s_rel_l2_u") for m in acc}
    ens = line.get("ensemble_128", {})
    if ens:
        out["ensemble_batched_vs_sequential"] = {
            s: [ens[s]["batched_glups"], ens[s]["sequential_glups"]] for s in ("fp32", "fp16s")}
    if "blocks_256" in line:
        out["blocks_glups_stored"] = line["blocks_256"]["glups_stored"]
    adj = line.get("adjoint_128", {}).get("fp32s")
    if adj:
        out["adjoint"] = {"backward_to_forward": adj["adjoint_to_forward_ratio"],
                          "fd_rel_err_alpha_max": adj["fd_rel_err_alpha_max"]}
    par = line.get("parity_256_vs_reference", {})
    out["parity_pops_vs_reference"] = {m: par[m].get("pops") for m in par if isinstance(par[m], dict)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ni", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16s", "fp64", "fp32s"],
                    help="population storage of the headline run (profiling)")
    ap.add_argument("--model", default="bgk", choices=["bgk", "mrt", "les"],
                    help="collision model of the headline run (profiling; the headline is BGK)")
    ap.add_argument("--rounding", default="default", choices=["default", "nearest", "stochastic"],
                    help="FP16S rounding of the headline run (profiling)")
    ap.add_argument("--launch", default=None,
                    help="tile_y,ctas_per_sm,cells_per_thread for the headline run instead of "
                         "the autotuner (profiling)")
    ap.add_argument("--accuracy-ni", type=int, default=256,
                    help="cavity size of the FP64-referenced velocity error report (256 or 512)")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="steps of the velocity error report (the configuration's 2000)")
    ap.add_argument("--accuracy-models", default="bgk,mrt,les",
                    help="models of the velocity error report (comma-separated)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the 256^3 parity runs of the reference's CPU path (background)")
    ap.add_argument("--quick", action="store_true",
                    help="headline and e2e only (no variants / accuracy / blocks / ensemble / "
                         "adjoint blocks)")
    ap.add_argument("--only", default=None, choices=["blocks", "ensemble", "accuracy"],
                    help="run one secondary workload alone and print its JSON (profiling): "
                         "the 48 uneven blocks of the 256^3 cavity, the 128-cavity ensemble, "
                         "or the velocity error report at --accuracy-ni")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.only:
        import torch
        import freelb_b200 as F
        torch.cuda.set_device(local_rank)
        stream = torch.cuda.current_stream()
        if args.only == "blocks":
            out = {"blocks_256": blocks_block(F, torch, stream, 256, args.steps)}
        elif args.only == "accuracy":
            out = {"accuracy": accuracy_block(F, args.accuracy_ni, args.accuracy_steps,
                                              models=tuple(args.accuracy_models.split(",")))}
        else:
            out = {"ensemble_128": ensemble_block(F, torch, stream)}
        print(json.dumps(out), flush=True)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
