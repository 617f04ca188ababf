"""Benchmark: zone-updates/s of the GRMHD update on one B200 (and N replicas).

Headline workload: the 3D Fishbone-Moncrief torus of 256 (r) x 128 (theta) x
128 (phi) cells including ghosts, modified Kerr-Schild (a = 0.9375), MP5 +
HLLE(LLF) + flux-CT + RK3, CFL 0.4, FP64, with the positivity fallback on
(guard bit 1; with reference semantics MP5 drives face densities negative at
the torus surface and the entropy flux turns NaN).  One step = one full RK3
step over all interior cells; a zone-update is one interior cell advanced by
one step.  Data are synthetic (seeded torus initial data); the state (~0.3 GB
per copy) exceeds the 126 MB L2, so no flush is needed between steps.

Extra sections of the same JSON line (N = 1 only; each 0 flag skips one):
  mixed          FP32-mixed vs FP64 on the 384 x 192 x 192 torus: both timed
                 over --mixed-steps steps from the same initial data, L1/Linf
                 errors of rho, p and B and the error of the horizon mass and
                 energy accretion rates of the mixed state against the FP64
                 state after those steps.
  torus2d        the 2D torus (256 x 256, phi slab) in FP64, 1000 steps.
  batched_tubes  1024 seeded 1D RMHD Riemann tubes of 400-3200 cells run to
                 t = 0.4 in one batch (rg_step_batch), FP64 and FP32-mixed.
  serving        a seeded Poisson stream of 2D tori (grids 128^2..512^2, half
                 FP64, half mixed, 2000 steps each) served with continuous
                 batching: p50/p99 latency and aggregate zone-updates/s.

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
# DRAM bytes per unit measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of one launch divided by
# its units) on the 192x96x96 torus, whose state already exceeds the L2
# (update: the TMA-staged k_update_tma, stages 2 and 3, whose boxes re-read their j-1 / k-1 halos)
DRAM_BYTES_PER_UNIT = {"update": 472.0, "flux_r": 113.0, "flux_phi": 120.0, "flux_theta": 122.0}
BYTES_PER_UNIT["flux"] = 136
# the TMA-staged face kernels (k_flux_tma, stencil and face metric staged) of the FP64 MP5 path, ncu on the
# 192x96x96 torus
DRAM_BYTES_PER_UNIT["flux"] = (124.0 + 132.0 + 135.0) / 3
# FP64 pipe utilisation of the face kernels from ncu (sm__inst_executed_pipe_fp64, percent of the peak
# sustained rate while active), mean over the three directions (update: over the three stages) on the
# 192x96x96 torus
FP64_PIPE_FRAC = {"flux": 0.481, "update": 0.271}
# algorithmic HBM bytes of one zone-update (FP64): only primitives persist between stages
STEP_BYTES_PER_ZONE = 648
# Executed FP64 operations per zone-update of one full RK3 step (MP5, FP64): ncu
# smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on.sum over every launch of one step
# of the 192x96x96 torus, dadd + dmul + 2 dfma, divided by its interior cells (1,424,896).  It
# includes the Newton iterations of the FP64 divisions and square roots.
FP64_FLOPS_PER_ZONE = 15271.0


def fp64_peak_tflops(device) -> float:
    """FP64 throughput of a plain library DGEMM (torch.matmul, float64,
    8192^3, best of 5 after 2 warm-up): the FP64 roof the step is compared
    with (B200 runs FP64 vector and tensor work at the same rate)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = _events()
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


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


def max_over_ranks(x: float, device: str = "cuda") -> float:
    """The maximum of x over the ranks of the default process group (x itself
    without one): replicas are timed by their slowest rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
    rec = {5: "ppm", 6: "mp5", 7: "weno5"}.get(args.irec, f"irec{args.irec}")
    return {"workload": f"fm_torus_3d_{args.nr}x{args.nth}x{args.nph}_{rec}_fp64",
            "grid_incl_ghosts": [args.nr, args.nth, args.nph], "interior_cells": config.interior_cells(p),
            "metric": "MKS a=0.9375", "scheme": f"{rec.upper()}+HLLE(LLF)+fluxCT+RK3", "cfl": p["cfl"],
            "guard": p["guard"],
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
    # initial data: the host construction, timed, then the device one, which the run keeps
    t = time.perf_counter()
    run.ic_torus(seed=2012 + rank)
    ic_host_s = time.perf_counter() - t
    t = time.perf_counter()
    run.ic_torus_device(seed=2012 + rank)
    ic_device_s = time.perf_counter() - t

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    divb0 = run.divb()
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
    divb1 = run.divb()
    divb = {"guard": p["guard"], "initial": divb0[0] / divb0[1], "after_steps": divb1[0] / divb1[1],
            "steps": args.warmup + args.steps,
            "measure": "max over interior corners of |corner-centred div(sqrt(-g) B)| / max |sqrt(-g) B^d| / dx_d "
                       "(rg_run_divb)",
            "note": "guard 1 keeps the reference's LLF flux of the normal field (hll.f90:109-111), which flux-CT "
                    "does not replace, so div B drifts; guard 3 (Toth's zero normal flux) holds it at round-off"}

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

    # per-kernel device times (separate pass: CUDA events around every launch on the library stream)
    roofline, shares, step_roof = None, {}, None
    peak, peak_kind = measured_peaks()
    if args.prof_steps > 0:
        ctx.profile(True)
        run.step(args.prof_steps)
        prof = ctx.profile_read()
        ctx.profile(False)
        total = sum(v["ms"] for v in prof.values())
        shares = {k: round(v["ms"] / total, 4) for k, v in prof.items()}
        # The face kernels of the three directions are one family (one launch per direction and stage, the
        # same faces per launch): together they are the largest share of the step.
        fam = ("flux_r", "flux_phi", "flux_theta")
        kinds = {"flux": {"ms": sum(prof[k]["ms"] for k in fam), "launches": sum(prof[k]["launches"] for k in fam)}}
        kinds.update({k: prof[k] for k in prof if k in BYTES_PER_UNIT and k not in fam})
        top = max(kinds, key=lambda k: kinds[k]["ms"])
        # one update per stage comprises the cell kernel, the straggler pass and the W-carry pass
        n_launch = 3 * args.prof_steps if top == "update" else kinds[top]["launches"]
        nm0, nm1 = run.nm0, run.nm1
        faces = (p["imax"] - 2 * nm0 + 1) * (p["jmax"] - 2 * nm0 + 1) * (p["kmax"] - 2 * nm0 + 1)
        units = {"update": zones, "flux": faces,
                 "flux_ct": (p["imax"] - 2 * nm1 + 1) * (p["jmax"] - 2 * nm1 + 1) * (p["kmax"] - 2 * nm1 + 1),
                 "floors": p["imax"] * p["jmax"] * p["kmax"],
                 "cfl": (p["imax"] - 2) * (p["jmax"] - 2) * (p["kmax"] - 2)}
        u = units[top]
        per_launch_ms = kinds[top]["ms"] / max(n_launch, 1)
        achieved = BYTES_PER_UNIT[top] * u / (per_launch_ms * 1e-3) / 1e9
        traffic = DRAM_BYTES_PER_UNIT.get(top)
        roofline = {"bound": "hbm", "kernel": "k_flux (r, phi, theta faces)" if top == "flux" else top,
                    "achieved": achieved, "peak": peak, "peak_source": peak_kind,
                    "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None if traffic is None else traffic * u,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per unit on the "
                                      "192x96x96 torus, scaled by the units of one launch "
                                      "(profiles/k_flux_tma_vs_k_flux_fm_torus_3d_192x96x96_mp5.md)",
                    "bytes_per_unit": BYTES_PER_UNIT[top], "units_per_launch": u, "ms_per_launch": per_launch_ms,
                    "share_of_step": round(kinds[top]["ms"] / total, 4),
                    "fp64_pipe_frac": FP64_PIPE_FRAC.get(top),
                    "fp64_pipe_source": "ncu sm__inst_executed_pipe_fp64 (pct of peak sustained active), "
                                        "192x96x96 torus",
                    "note": "FP64-pipe bound kernel: HBM fraction of algorithmic bytes with the FP64 pipe beside it"}
    run.release()
    run.release()
    fp64_peak = fp64_peak_tflops(dev) if (rank == 0 and args.prof_steps > 0) else None
    extra = {}
    if ws == 1:
        sections = (("exact_build", args.exact_steps, section_exact),
                    ("scheme_variants", args.variant_steps, section_variants),
                    ("mixed", args.mixed_steps, section_mixed), ("torus2d", args.torus2d_steps, section_torus2d),
                    ("batched_tubes", args.tubes, section_tubes), ("serving", args.serve_requests, section_serving))
        for name, n, fn in sections:
            if n > 0:
                t = time.perf_counter()
                extra[name] = fn(ctx, args)
                extra[name]["section_wall_s"] = time.perf_counter() - t
                print(f"[bench] section {name} done in {extra[name]['section_wall_s']:.1f} s", file=sys.stderr,
                      flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return None
    value = zones * ws * args.steps / (ms * 1e-3)
    # the whole step against the algorithmic minimum of 648 B per zone-update (FP64 primitives only:
    # one CFL pass, then 2 + 3 + 3 reads/writes of the 9 primitives in the three stages)
    step_gbs = STEP_BYTES_PER_ZONE * zones * args.steps / (ms * 1e-3) / 1e9
    step_roof = {"bound": "hbm", "bytes_per_zone_update": STEP_BYTES_PER_ZONE, "achieved": step_gbs,
                 "peak": peak, "unit": "GB/s", "frac": step_gbs / peak}
    fp64 = None
    if fp64_peak is not None:
        achieved = zones * args.steps / (ms * 1e-3) * FP64_FLOPS_PER_ZONE / 1e12  # per GPU
        fp64 = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "flops_per_unit": FP64_FLOPS_PER_ZONE,
                "peak_source": "measured: torch.matmul float64 8192^3 (cuBLAS DGEMM), best of 5",
                "flops_source": "ncu dadd + dmul + 2 dfma executed per zone-update, 192x96x96 torus"}
    line = {
        "metric": "zone-updates/s (FP64, one full RK3 step per update)", "value": value, "unit": "zone-updates/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Fishbone-Moncrief torus initial data)",
        "config": dict(config_block(args, p), parallelism=f"replicas x{ws}"),
        "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        "roofline": roofline,
        "step_roofline": step_roof,
        "fp64_roofline": fp64,
        "divb": divb,
        "kernel_share": shares,
        "initial_data": {"host_s": ic_host_s, "device_s": ic_device_s,
                         "note": "torus initial data of the headline grid: rg_run_ic_torus (host construction "
                                 "and upload) vs rg_run_ic_torus_device; wall clock of the call"},
        "recov": {k: st[k] for k in ("recov_nr2", "recov_fail", "recov_carry", "recov_cap")},
    }
    line.update(extra)
    return line


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _rel_errs(got, ref, n):
    """Interior L1 (sum |a-b| / sum |b|) and Linf (max |a-b| / max |b|) per variable."""
    import numpy as np
    sl = (slice(n, -n),) * 3
    a, b = got[sl], ref[sl]
    d = np.abs(a - b)
    l1 = d.sum(axis=(0, 1, 2)) / np.abs(b).sum(axis=(0, 1, 2)).clip(1e-300)
    linf = d.max(axis=(0, 1, 2)) / np.abs(b).max(axis=(0, 1, 2)).clip(1e-300)
    names = {"rho": 0, "p": 4, "B1": 6, "B2": 7, "B3": 8}
    return ({k: float(l1[v]) for k, v in names.items()}, {k: float(linf[v]) for k, v in names.items()})


def section_variants(ctx, args) -> dict:
    """The headline grid with the other reconstructions of its workload
    family, PPM and WENO5 (FP64, same seed, same time step rules), timed and
    run for --variant-steps steps, and each compared with MP5 run as long from
    the same seed.  WENO5 and MP5 share the grid (nm1 = 4), so their fields are
    compared cell by cell; PPM's wider ghost zones (nm1 = 5) shift the phi
    grid, so PPM is compared through the phi-averaged fields on the (r, theta)
    cells both interiors cover."""
    import numpy as np
    import torch
    from raishinsource_b200 import config
    stream = torch.cuda.current_stream()
    out, finals = {}, {}
    for name, irec in (("mp5", config.IREC_MP5), ("ppm", config.IREC_PPM), ("weno5", config.IREC_WENO5)):
        p = dict(config.torus(nr=args.nr, nth=args.nth, nph=args.nph, irec=irec), guard=args.guard)
        zones = config.interior_cells(p)
        r = ctx.admit(p)
        r.ic_torus_device(seed=2012)
        r.step(3, strict=False)  # first use of every kernel
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record(stream)
        r.step(args.variant_steps - 3, strict=False)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = r.stats()
        finals[name] = (r.prims(), r.nm1)
        out[name] = {"workload": f"fm_torus_3d_{args.nr}x{args.nth}x{args.nph}_{name}_fp64", "interior_cells": zones,
                     "value": zones * (args.variant_steps - 3) / (ms * 1e-3), "unit": "zone-updates/s",
                     "ms_per_step": ms / (args.variant_steps - 3), "steps": args.variant_steps, "time": st["time"],
                     "finite": bool(np.isfinite(finals[name][0]).all())}
        r.release()
    ref, n_ref = finals["mp5"]
    names = {"rho": 0, "p": 4, "B1": 6, "B2": 7, "B3": 8}
    for name in ("ppm", "weno5"):
        got, n = finals[name]
        if n == n_ref:
            sl = (slice(n, -n),) * 3
            a, b = got[sl], ref[sl]
            how = "cell by cell over the common interior"
        else:
            m = max(n, n_ref)
            a = got[m:-m, n:-n, m:-m].mean(axis=1)
            b = ref[m:-m, n_ref:-n_ref, m:-m].mean(axis=1)
            how = "phi-averaged fields over the (r, theta) cells of both interiors"
        l1 = np.abs(a - b).sum(axis=(0, 1)) if a.ndim == 3 else np.abs(a - b).sum(axis=(0, 1, 2))
        den = np.abs(b).sum(axis=(0, 1)) if b.ndim == 3 else np.abs(b).sum(axis=(0, 1, 2))
        out[name]["l1_rel_vs_mp5"] = {k: float(l1[v] / max(den[v], 1e-300)) for k, v in names.items()}
        out[name]["compared"] = how
    return out


def section_exact(ctx, args) -> dict:
    """The uncontracted build (libraishin_gpu_exact.so: no FMA, rg_pow for every
    power), which agrees with the oracle bit for bit, timed on the headline
    workload in a child process (the library is process-global)."""
    env = dict(os.environ, RAISHIN_GPU_LIB="exact")
    cmd = [sys.executable, os.path.abspath(__file__), "--exact-child", "--steps", str(args.exact_steps),
           "--nr", str(args.nr), "--nth", str(args.nth), "--nph", str(args.nph), "--irec", str(args.irec),
           "--guard", str(args.guard)]
    res = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900)
    if res.returncode != 0:
        return {"error": res.stderr[-500:]}
    return json.loads(res.stdout.strip().splitlines()[-1])


def exact_child(args) -> None:
    import torch
    from raishinsource_b200 import Context, config
    p = workload(args)
    zones = config.interior_cells(p)
    with Context(0) as ctx:
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        r = ctx.admit(p)
        r.ic_torus_device(seed=2012)
        r.step(3)
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        r.step(args.steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        r.release()
    maps = open("/proc/self/maps").read()
    lib = sorted({os.path.basename(x.split()[-1]) for x in maps.splitlines() if "libraishin_gpu" in x})
    print(json.dumps({"workload": config_block(args, p)["workload"], "library": lib, "steps": args.steps, "warmup": 3,
                      "value": zones * args.steps / (ms * 1e-3), "unit": "zone-updates/s",
                      "ms_per_step": ms / args.steps,
                      "note": "no FMA contraction and the library's own pow: bit-identical to the oracle (CPU "
                              "restatement) step after step"}))


def section_mixed(ctx, args) -> dict:
    """FP64 and FP32-mixed runs of the same torus from the same initial data."""
    import torch
    from raishinsource_b200 import config
    nr, nth, nph = (int(x) for x in args.mixed_grid.split(","))
    p = dict(config.torus(nr=nr, nth=nth, nph=nph), guard=args.guard)
    zones = config.interior_cells(p)
    stream = torch.cuda.current_stream()
    out = {"workload": f"fm_torus_3d_{nr}x{nth}x{nph}_mp5", "steps": args.mixed_steps, "interior_cells": zones}
    # a radial shell inside the FP32 region (r > 2 r_H): the last face below r = 6 M, the torus's inner edge
    # (cell centres x1(i) = xmin (xmax/xmin)^((i-1)/(imax-1)), grid.f90 for ix1 = 2)
    x1 = [p["xmin"] * (p["xmax"] / p["xmin"]) ** ((i - 1) / (p["imax"] - 1)) for i in range(1, p["imax"] + 1)]
    shell = max(i for i in range(1, p["imax"]) if 0.5 * (x1[i - 1] + x1[i]) <= 6.0)
    r_shell = 0.5 * (x1[shell - 1] + x1[shell])
    states = {}
    for prec in ("fp64", "mixed"):
        r = ctx.admit(dict(p, precision=prec))
        r.ic_torus_device(seed=2012)
        r.step(3)  # first use of every kernel; counted in the comparison below
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record(stream)
        r.step(args.mixed_steps - 3)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = r.stats()
        states[prec] = (r.prims(), r.horizon_flux(), st, r.radial_flux(shell))
        # per-kind device time of 3 more steps (CUDA events around every launch)
        ctx.profile(True)
        r.step(3)
        prof = ctx.profile_read()
        ctx.profile(False)
        kinds_ms = {k: round(v["ms"] / 3, 4) for k, v in prof.items() if v["ms"] > 0}
        out[prec] = {"value": zones * (args.mixed_steps - 3) / (ms * 1e-3), "unit": "zone-updates/s",
                     "ms_per_step": ms / (args.mixed_steps - 3), "time": st["time"],
                     "recov_nr2": st["recov_nr2"], "recov_fail": st["recov_fail"],
                     "kernel_ms_per_step": kinds_ms}
        r.release()
    (a, (ma, ea), _, (sma, sea)), (b, (mb, eb), _, (smb, seb)) = states["mixed"], states["fp64"]
    l1, linf = _rel_errs(a, b, config.ghost_widths(p["irec"], p.get("ict", 1))[1])
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["l1_rel_mixed_vs_fp64"] = l1
    out["linf_rel_mixed_vs_fp64"] = linf
    out["horizon"] = {"mdot_fp64": mb, "mdot_mixed": ma, "edot_fp64": eb, "edot_mixed": ea,
                      "mdot_rel_err": abs(ma - mb) / max(abs(mb), 1e-300),
                      "edot_rel_err": abs(ea - eb) / max(abs(eb), 1e-300),
                      "note": "inner edge of the interior (just outside the horizon), inside the FP64 region"}
    out["shell_flux"] = {"r": r_shell, "face_index": shell, "mdot_fp64": smb, "mdot_mixed": sma, "edot_fp64": seb,
                         "edot_mixed": sea, "mdot_rel_err": abs(sma - smb) / max(abs(smb), 1e-300),
                         "edot_rel_err": abs(sea - seb) / max(abs(seb), 1e-300),
                         "note": "mass and energy flux through the radial shell at the torus inner edge, inside the "
                                 "FP32 region (r > 2 r_H) of the mixed run (rg_run_radial_flux)"}
    out["precision"] = ("FP32 reconstruction, LLF fluxes, flux-CT and RK combine (compensated accumulation) "
                        "beyond 2 r_H; FP64 recovery, floors, CFL, metric and sources inside 2 r_H")
    return out


def section_torus2d(ctx, args) -> dict:
    import torch
    from raishinsource_b200 import config
    p = dict(config.torus(nr=256, nth=256), guard=args.guard)
    zones = config.interior_cells(p)
    r = ctx.admit(p)
    r.ic_torus(seed=2012)
    r.step(5)
    torch.cuda.synchronize()
    e0, e1 = _events()
    stream = torch.cuda.current_stream()
    e0.record(stream)
    r.step(args.torus2d_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    r.release()
    return {"workload": "fm_torus_2d_256x256_mp5_fp64 (phi slab of 9 stored as one plane)", "steps": args.torus2d_steps,
            "value": zones * args.torus2d_steps / (ms * 1e-3), "unit": "zone-updates/s",
            "ms_per_step": ms / args.torus2d_steps}


def section_tubes(ctx, args) -> dict:
    """Seeded Riemann tubes in one batch, run to t = tmax, FP64 and mixed."""
    import numpy as np
    import torch
    from raishinsource_b200 import config
    rng = np.random.default_rng(2012)
    lengths = rng.integers(400, 3201, size=args.tubes)
    out = {"tubes": args.tubes, "lengths": [int(lengths.min()), int(lengths.max())], "tmax": args.tube_tmax,
           "timed_steps": "to t = tmax" if args.tube_steps <= 0 else args.tube_steps,
           "note": ("zone-updates/s counts interior cells of active tubes; latencies are the wall time at which a "
                    "tube passed tmax, null unless all tubes finished in the timed steps")}
    finals, fails = {}, {}
    for prec in ("fp64", "mixed"):
        runs = []
        for t, n in enumerate(lengths):
            r = ctx.admit(dict(config.tube(n=int(n), tmax=args.tube_tmax, precision=prec), guard=args.guard))
            r.ic_tube(seed=2012, tube=t)
            runs.append(r)
        stream = torch.cuda.current_stream()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0, e1 = _events()
        e0.record(stream)
        # every tube ends within imax steps (dt >= cfl*dx once speeds are clipped to 1); by default only the
        # first --tube-steps steps are timed (see the section notes)
        chunk, steps, done_at = 32, 0, {}
        cap = 2 * (int(lengths.max()) + 16) if args.tube_steps <= 0 else args.tube_steps
        while steps < cap:
            st = ctx.step_batch(runs, chunk, stats=True, strict=False)
            steps += chunk
            now = time.perf_counter() - t0
            for k, x in enumerate(st):
                if k not in done_at and not (x["time"] <= args.tube_tmax):
                    done_at[k] = now
            if len(done_at) == len(runs):
                break
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        zu = sum(x["steps"] * int(n) for x, n in zip(st, lengths))
        info = ctx.batch_info(runs)
        lat = np.array(sorted(done_at.values())) if len(done_at) == len(runs) else None
        out[prec] = {"value": zu / (ms * 1e-3), "unit": "zone-updates/s", "zone_updates": int(zu),
                     "batch_steps": steps, "wall_ms": ms,
                     "p50_run_latency_s": None if lat is None else float(np.percentile(lat, 50)),
                     "p99_run_latency_s": None if lat is None else float(np.percentile(lat, 99)), "tuned": info,
                     "capped_rescale_loops": {"recov_w": int(sum(x["recov_cap"] for x in st)),
                                              "pminmax2b": int(sum(x["floor_cap"] for x in st))},
                     "recov_fail": int(sum(x["recov_fail"] for x in st)),
                     "recov_nr2": int(sum(x["recov_nr2"] for x in st)),
                     "unfinished_tubes": len(runs) - len(done_at)}
        finals[prec] = [r.stored_prims()[0, 0, 0, :] for r in runs]  # rho along the tube
        fails[prec] = [x["recov_fail"] + x["recov_cap"] for x in st]
        for r in runs:
            r.release()
    fin = [np.isfinite(a).all() and np.isfinite(b).all() for a, b in zip(finals["mixed"], finals["fp64"])]
    num = sum(np.abs(a - b).sum() for a, b, f in zip(finals["mixed"], finals["fp64"], fin) if f)
    den = sum(np.abs(b).sum() for b, f in zip(finals["fp64"], fin) if f)
    out["l1_rel_rho_mixed_vs_fp64"] = float(num / den) if den > 0 else None
    # tubes whose recovery never failed nor capped in either precision
    ok = [f and a == 0 and b == 0 for f, a, b in zip(fin, fails["fp64"], fails["mixed"])]
    num = sum(np.abs(a - b).sum() for a, b, f in zip(finals["mixed"], finals["fp64"], ok) if f)
    den = sum(np.abs(b).sum() for b, f in zip(finals["fp64"], ok) if f)
    out["l1_rel_rho_mixed_vs_fp64_no_failed_recovery"] = {"tubes": int(sum(ok)),
                                                          "value": float(num / den) if den > 0 else None}
    out["nonfinite_tubes"] = int(len(fin) - sum(fin))
    return out


def section_serving(ctx, args) -> dict:
    from raishinsource_b200 import serving
    import torch
    reqs = serving.poisson_stream(args.serve_requests, rate=args.serve_rate, seed=2012, steps=args.serve_steps)
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(args.serve_budget_gb * 2**30, 0.8 * free))
    srv = serving.Server(ctx, mem_budget=budget, max_runs=64, tick_steps=50)
    res = srv.serve(reqs)
    srv.close()
    res.pop("done")
    peak, peak_kind = measured_peaks()
    res["hbm"] = {"bytes_per_zone_update": STEP_BYTES_PER_ZONE, "achieved_gbs":
                  STEP_BYTES_PER_ZONE * res["zone_updates_per_s"] / 1e9, "peak": peak, "peak_source": peak_kind,
                  "frac": STEP_BYTES_PER_ZONE * res["zone_updates_per_s"] / 1e9 / peak,
                  "note": "aggregate zone-updates/s times the FP64 algorithmic bytes of one zone-update (648 B; "
                          "the mixed half moves less), against the measured copy bandwidth"}
    res.update({"arrival_rate_per_s": args.serve_rate, "steps_per_request": args.serve_steps,
                "mem_budget_gb": budget / 2**30, "unit": "zone-updates/s",
                "grids": [128, 256, 384, 512], "mix": "half FP64, half FP32-mixed"})
    return res


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
    ap.add_argument("--variant-steps", type=int, default=1000,
                    help="steps of the MP5, PPM and WENO5 runs of the headline grid compared at the end (0: skip)")
    ap.add_argument("--exact-steps", type=int, default=20,
                    help="timed steps of the uncontracted (bit-exact) build on the headline grid (0: skip)")
    ap.add_argument("--exact-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--guard", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--prof-steps", type=int, default=3)
    ap.add_argument("--cpu-steps", type=int, default=1, help="steps in the CPU-baseline sample (0 = skip)")
    ap.add_argument("--mixed-steps", type=int, default=1000, help="steps of the FP64-vs-mixed section (0 = skip)")
    ap.add_argument("--mixed-grid", default="384,192,192", help="imax,kmax,jmax of the mixed section")
    ap.add_argument("--torus2d-steps", type=int, default=1000, help="steps of the 2D torus section (0 = skip)")
    ap.add_argument("--tubes", type=int, default=1024, help="Riemann tubes of the batched section (0 = skip)")
    ap.add_argument("--tube-tmax", type=float, default=0.4)
    ap.add_argument("--tube-steps", type=int, default=0,
                    help="batch steps timed in the tube section (0 = run every tube to tmax)")
    ap.add_argument("--serve-requests", type=int, default=24, help="requests of the serving section (0 = skip)")
    ap.add_argument("--serve-rate", type=float, default=2.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--serve-steps", type=int, default=2000)
    ap.add_argument("--serve-budget-gb", type=float, default=40.0, help="device memory budget for admission")
    args = ap.parse_args()
    ws, rank, _ = dist_env()
    if args.exact_child:
        exact_child(args)
        return
    if args.impl == "reference":
        if rank != 0:
            return
        nref = max(1, min(args.steps, 2))
        ref = time_reference(args, nref)
        line = {"impl": "reference", "metric": "zone-updates/s (FP64, one full RK3 step per update)",
                "value": ref["value"], "unit": "zone-updates/s", "n_gpus": ws, "steps": nref,
                "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded Fishbone-Moncrief torus initial data)",
                "config": dict(config_block(args, workload(args)), parallelism=f"replicas x{ws}"),
                "note": "bounded sample: %d full step(s) of about 2 s each on the host cores, no warm-up" % nref,
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
