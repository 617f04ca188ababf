"""Benchmark: zone-updates/s of the FP64 GRMHD update on one B200 (and N replicas).

Workload (default): the 3D Fishbone-Moncrief torus of the reference's
configuration 1: 256 (r) x 128 (theta) x 128 (phi) cells including ghosts,
modified Kerr-Schild (a = 0.9375), MP5 + HLLE(LLF) + flux-CT + RK3, CFL 0.4,
FP64, with the positivity fallback on (guard bit 1; with reference semantics
MP5 drives face densities negative at the torus surface and the entropy flux
turns NaN).  One step = one full RK3 step over all interior cells; a zone-
update is one interior cell advanced by one step.  Data are synthetic (the
torus is generated, seeded); the state (~0.3 GB per copy) exceeds the 126 MB
L2, so no flush is needed between steps.

Arms:
  default            GPU arm through the C ABI (value = device-resident steps;
                     e2e = per step: upload prims from pinned host memory,
                     one step, download prims to pinned host memory).
  --impl reference   the CPU restatement of the reference (oracle/, OpenMP over
                     all host cores) on the same workload, one step per sample.

Under torchrun (N > 1) every rank runs an independent replica on its GPU (the
path is single-GPU by design; no collective on the data path); the time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes per unit of each kernel kind (FP64, 8 B/value):
#  flux_*:  per face: read the 8 stencil-owned primitives of its left cell
#           (var 6 is never read) + write 9 fluxes          -> (8 + 9) * 8
#  update:  per cell: read P_cur 9, P_n 9, 3x9 face fluxes of its upper faces,
#           6 CT fluxes; write 9 primitives                  -> (9+9+27+6+9) * 8
#  ct:      per cell: read 6 raw induction fluxes, write 6   -> 12 * 8
#  floors:  per cell: read 9 (vars 1-9), write 6             -> 15 * 8
#  cfl:     per cell: read 9                                 -> 9 * 8
BYTES_PER_UNIT = {"flux_r": 136, "flux_phi": 136, "flux_theta": 136, "update": 480, "flux_ct": 96,
                  "floors": 120, "cfl": 72}


def measured_peaks() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.proc, self.lines = gpu, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload(args) -> dict:
    from raishinsource_b200 import config
    p = config.torus(nr=args.nr, nth=args.nth, nph=args.nph, irec=args.irec)
    p["guard"] = args.guard
    return p


def config_block(args, p) -> dict:
    from raishinsource_b200 import config
    return {"workload": f"fm_torus_3d_{args.nr}x{args.nth}x{args.nph}_{'mp5' if args.irec == 6 else 'weno5'}_fp64",
            "grid_incl_ghosts": [args.nr, args.nth, args.nph], "interior_cells": config.interior_cells(p),
            "metric": "MKS a=0.9375", "scheme": "MP5+HLLE(LLF)+fluxCT+RK3" if args.irec == 6 else
            "WENO5+HLLE(LLF)+fluxCT+RK3", "cfl": p["cfl"], "guard": p["guard"],
            "l2": "inputs larger than L2: one primitive copy is %.0f MB (126 MB L2); no flush" %
                  (72e-6 * p["imax"] * p["jmax"] * p["kmax"])}


def run_gpu(args) -> dict | None:
    import numpy as np
    import torch

    from raishinsource_b200 import Context, config

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    p = workload(args)
    zones = config.interior_cells(p)
    ctx = Context(dev)
    ctx.set_stream(stream.cuda_stream)
    run = ctx.admit(p)
    run.ic_torus(seed=2012 + rank)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # warm-up (also the first use of every kernel)
    run.step(args.warmup)
    torch.cuda.synchronize()
    ctx.profile(False)  # reset launch counters; no per-launch events in the timed region
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(stream)
        run.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    launches = sum(v["launches"] for v in ctx.profile_read().values())
    st = run.stats()
    ref_prims = run.prims() if args.mixed else None  # FP64 state after warm-up + timed steps

    # end to end through the public API with host buffers (pinned)
    e2e = None
    if args.e2e_steps > 0:
        host = torch.empty(run.shape, dtype=torch.float64, pin_memory=True)
        run.download_prims_ptr(host.data_ptr())
        nbytes = host.numel() * 8
        barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.e2e_steps):
            run.upload_prims_ptr(host.data_ptr(), t0=st["time"])
            run.step(1)
            run.download_prims_ptr(host.data_ptr())
        t1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(t0.elapsed_time(t1))
        e2e = {"value": zones * ws * args.e2e_steps / (e_ms * 1e-3), "unit": "zone-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": args.e2e_steps,
               "ms_per_step": e_ms / args.e2e_steps, "api": "rg_run_upload_prims + rg_step + rg_run_download_prims"}

    # FP32-mixed run of the same workload: same IC, same number of steps; timed
    # like the FP64 arm, L1 error of its state against the FP64 state at the end
    mixed = None
    if args.mixed:
        ref_steps = args.warmup + args.steps
        runm = ctx.admit(dict(p, precision="mixed"))
        runm.ic_torus(seed=2012 + rank)
        runm.step(args.warmup)
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        runm.step(args.steps)
        m1.record(stream)
        torch.cuda.synchronize()
        mms = max_over_ranks(m0.elapsed_time(m1))
        got = runm.prims()
        mshares = {}
        if args.prof_steps > 0:
            ctx.profile(True)
            runm.step(args.prof_steps)
            mp = ctx.profile_read()
            ctx.profile(False)
            mt = sum(v["ms"] for v in mp.values())
            mshares = {k: round(v["ms"] / mt, 4) for k, v in mp.items()}
        runm.release()
        n = run.nm1
        sl = (slice(n, -n),) * 3
        l1 = (np.abs(got[sl] - ref_prims[sl]).sum(axis=(0, 1, 2)) /
              np.abs(ref_prims[sl]).sum(axis=(0, 1, 2)).clip(1e-300))
        mixed = {"value": zones * ws * args.steps / (mms * 1e-3), "unit": "zone-updates/s",
                 "ms_per_step": mms / args.steps, "speedup_vs_fp64": ms / mms,
                 "l1_rel_vs_fp64": {"rho": float(l1[0]), "p": float(l1[4]), "B1": float(l1[6]),
                                    "B3": float(l1[8])},
                 "after_steps": ref_steps, "kernel_share": mshares,
                 "precision": "FP32 recon/LLF/CT/RK combine (compensated), FP64 recovery/floors/CFL, "
                              "FP64 fluxes and sources for r < 2 r_H"}

    # per-kernel device times (separate pass: CUDA events around every launch on the library stream)
    roofline, shares = None, {}
    if args.prof_steps > 0:
        ctx.profile(True)
        run.step(args.prof_steps)
        prof = ctx.profile_read()
        ctx.profile(False)
        total = sum(v["ms"] for v in prof.values())
        shares = {k: round(v["ms"] / total, 4) for k, v in prof.items()}
        top = max((k for k in prof if k in BYTES_PER_UNIT), key=lambda k: prof[k]["ms"])
        n_launch = prof[top]["launches"] / (2 if top == "update" else 1)
        nm0, nm1 = run.nm0, run.nm1
        faces = (p["imax"] - 2 * nm0 + 1) * (p["jmax"] - 2 * nm0 + 1) * (p["kmax"] - 2 * nm0 + 1)
        units = {"update": zones,
                 "flux_ct": (p["imax"] - 2 * nm1 + 1) * (p["jmax"] - 2 * nm1 + 1) * (p["kmax"] - 2 * nm1 + 1),
                 "floors": p["imax"] * p["jmax"] * p["kmax"],
                 "cfl": (p["imax"] - 2) * (p["jmax"] - 2) * (p["kmax"] - 2)}
        u = units.get(top, faces)
        per_launch_ms = prof[top]["ms"] / max(n_launch, 1)
        peak, peak_kind = measured_peaks()
        achieved = BYTES_PER_UNIT[top] * u / (per_launch_ms * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "peak_source": peak_kind,
                    "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                    "bytes_per_unit": BYTES_PER_UNIT[top], "units_per_launch": u, "ms_per_launch": per_launch_ms,
                    "note": "FP64-pipe bound path: HBM fraction of algorithmic bytes, see profiles/"}
    run.release()
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return None
    value = zones * ws * args.steps / (ms * 1e-3)
    line = {
        "metric": "zone-updates/s (FP64, one full RK3 step per update)", "value": value, "unit": "zone-updates/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Fishbone-Moncrief torus initial data)",
        "config": dict(config_block(args, p), parallelism=f"replicas x{ws}"),
        "e2e": e2e, "mixed": mixed, "gpu_launches": launches, "clocks": clk.summary(),
        "roofline": roofline,
        "kernel_share": shares,
        "recov": {k: st[k] for k in ("recov_nr2", "recov_fail", "recov_carry", "recov_cap")},
    }
    return line


def time_reference(args, steps: int, label_cores=None) -> dict:
    """The CPU restatement of the reference (oracle/) on the same workload."""
    from oracle import Oracle
    from raishinsource_b200 import config
    p = workload(args)
    zones = config.interior_cells(p)
    o = Oracle(p)
    o.ic_torus(seed=2012)
    o.init_cons()
    t = time.perf_counter()
    o.step(steps)
    sec = time.perf_counter() - t
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": zones * steps / sec, "unit": "zone-updates/s", "cores": cores, "kind": "port",
            "sample": f"{steps} full RK3 step(s) of the {args.nr}x{args.nth}x{args.nph} torus ({zones} zones), "
                      f"{sec:.1f} s, OpenMP over k on all host threads", "seconds": sec}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--nr", type=int, default=256)
    ap.add_argument("--nth", type=int, default=128)
    ap.add_argument("--nph", type=int, default=128)
    ap.add_argument("--irec", type=int, default=6)
    ap.add_argument("--guard", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--prof-steps", type=int, default=3)
    ap.add_argument("--cpu-steps", type=int, default=1, help="steps in the CPU-baseline sample (0 = skip)")
    ap.add_argument("--mixed", type=int, default=1, help="also time the FP32-mixed path (1) or not (0)")
    args = ap.parse_args()
    ws, rank, _ = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return
        ref = time_reference(args, max(1, min(args.steps, 2)))
        line = {"impl": "reference", "metric": "zone-updates/s (FP64, one full RK3 step per update)",
                "value": ref["value"], "unit": "zone-updates/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded Fishbone-Moncrief torus initial data)",
                "config": config_block(args, workload(args)),
                "cpu_baseline": {k: ref[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": ref["value"], "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    line = run_gpu(args)
    if line is None:
        return
    if ws == 1 and args.cpu_steps > 0:
        ref = time_reference(args, args.cpu_steps)
        line["cpu_baseline"] = {k: ref[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
