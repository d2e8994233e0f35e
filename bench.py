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
BYTES_PER_POP = {"fp32": 4, "fp16s": 2, "fp64": 8}


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
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
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
    warm = min(args.warmup, 1)
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

    def timed(storage, model="bgk"):
        lat = F.cavity(ni, tau=0.53, ulid=0.1, storage=storage, model=model)
        for _ in range(args.warmup):
            lat.step(1, stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as cs:
            e0.record(stream)
            lat.step(args.steps, stream)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        finite = lat.nonfinite()
        lat.close()
        return ms, cs.summary(), finite

    ms32, clocks, bad32 = timed("fp32")
    ms16, clocks16, bad16 = timed("fp16s")

    # end to end through the public API with host buffers: flags + lid velocity
    # field in from pinned host memory, K steps, RHO and VELOCITY back out.
    flags = F.cavity_flags(ni)
    u0 = np.zeros((cells, 3), dtype=np.float32)
    u0[flags == 8, 0] = np.float32(0.1)
    pin_flags = torch.from_numpy(flags).pin_memory().numpy()
    pin_u = torch.from_numpy(u0.reshape(-1)).pin_memory().numpy()
    out_rho = torch.empty(cells, dtype=torch.float32).pin_memory().numpy()
    out_u = torch.empty(3 * cells, dtype=torch.float32).pin_memory().numpy()
    lat = F.Lattice(n, n, n, 0.53, storage="fp32")
    lat.step(1, stream)  # first-launch costs outside the timed region
    lat.init_equilibrium(1.0, stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    lat.upload_flags(pin_flags, stream)
    lat.upload_field("u", pin_u, stream)
    lat.step(args.steps, stream)
    lat.compute_rhou(2, stream)
    import ctypes
    from freelb_b200 import _capi as C
    C.call("flb_download_field", lat._h, C.FIELD_RHO, ctypes.c_void_p(out_rho.ctypes.data),
           C.DTYPE_F32, ctypes.c_void_p(stream.cuda_stream))
    C.call("flb_download_field", lat._h, C.FIELD_VELOCITY, ctypes.c_void_p(out_u.ctypes.data),
           C.DTYPE_F32, ctypes.c_void_p(stream.cuda_stream))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    wall_ms = (time.perf_counter() - t0) * 1000.0
    e2e_ms = max(e2e_ms, wall_ms)
    if dist:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    lat.close()
    h2d = flags.nbytes + u0.nbytes
    d2h = out_rho.nbytes + out_u.nbytes

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_cpu(ni, 3, 0)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    peak, peak_kind = measured_peaks()
    glups32 = cells * args.steps * world / (ms32 / 1000.0) / 1e9
    glups16 = cells * args.steps * world / (ms16 / 1000.0) / 1e9
    b32 = algo_bytes_per_cell("fp32")
    b16 = algo_bytes_per_cell("fp16s")
    per_launch_ms32 = ms32 / args.steps
    per_launch_ms16 = ms16 / args.steps
    ach32 = cells * b32 / (per_launch_ms32 / 1000.0) / 1e9
    ach16 = cells * b16 / (per_launch_ms16 / 1000.0) / 1e9
    tr32 = profile_traffic("fp32_bgk_bytes_per_cell")
    tr16 = profile_traffic("fp16s_bgk_bytes_per_cell")
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
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"lid-driven cavity {ni}^3 D3Q19 BGK tau=0.53 u_lid=0.1",
                   "stored_cells": cells, "storage": "fp32", "per_gpu": "independent cavity",
                   "l2": "working set 21.8 GB >> 126 MB L2; no flush needed",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s",
                     "frac": ach32 / peak, "peak_source": peak_kind,
                     "traffic": (tr32 * cells if tr32 else None),
                     "algorithmic_bytes_per_cell": b32},
        "fp16s": {"value": glups16, "unit": "GLUPs", "ms_per_step": ms16 / args.steps,
                  "roofline": {"achieved": ach16, "peak": peak, "unit": "GB/s",
                               "frac": ach16 / peak,
                               "traffic": (tr16 * cells if tr16 else None),
                               "algorithmic_bytes_per_cell": b16},
                  "clocks": clocks16, "nonfinite": bad16},
        "e2e": {"value": cells * args.steps * world / (e2e_ms / 1000.0) / 1e9, "unit": "GLUPs",
                "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "job": "flags + VELOCITY in (pinned host), K steps, RHO + VELOCITY out"},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "nonfinite": bad32,
    }
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["mlups"] / 1000.0, "unit": "GLUPs",
                                "cores": cpu["threads"], "kind": "reference",
                                "sample": f"3 timed steps of the {ni}^3 cavity on the reference "
                                          f"FreeLB OpenMP path ({cpu['binary']})"}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ni", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
