"""Continuous batching of independent GRMHD runs on one GPU.

The reference runs one simulation per MPI job (main.f90:586-1151) and has no
notion of a request stream.  Here a stream of run requests (each a
``rg_run_params`` block, torus initial data and a step count) is served by
one context:

* arrival: a request's host-side preparation (grid, metric, Christoffel
  symbols and initial data, ``rg_prep_*``) starts on a worker thread as soon
  as it arrives, while the GPU keeps stepping the admitted runs;
* admission: a prepared request is admitted when a slot is free and its
  device footprint (``rg_run_footprint``) fits the memory budget next to the
  runs already resident; requests that do not fit wait (later, smaller ones
  may pass them);
* stepping: all resident runs advance together in ticks of ``tick_steps``
  steps through ``rg_step_batch`` (one launch per kernel kind and batch class,
  replayed from a CUDA graph), so a request that arrives while others are on
  the GPU joins the next tick and its work overlaps theirs.  Two ticks are
  kept queued on the stream (``rg_ctx_mark`` / ``rg_ctx_wait_mark``), so the
  GPU keeps stepping while the host admits and retires runs;
* completion: a run leaves the batch with the tick that takes its last steps;
  once that tick has completed it is read back, released, and its memory and
  slot go to the waiting requests.

Each run's result is the same alone and in the mix (the batched kernels run
every run's cells through the single-run code); ``tests/test_gpu_serving.py``
checks this.  Latency is measured from arrival to the moment the host has
seen the completion of the tick in which the run finished.
"""
from __future__ import annotations

import concurrent.futures as cf
import dataclasses
import math
import time

import numpy as np

from . import config
from .capi import Context, Prep, footprint


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the stream
    params: dict            # rg_run_params block (config.torus style)
    steps: int
    ic: dict                # torus initial-data arguments (seed, rmax, beta, ...)


@dataclasses.dataclass
class Done:
    rid: int
    arrival: float
    admitted: float
    finished: float
    zones: int
    steps: int
    precision: str
    prims: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def poisson_stream(n: int, rate: float, seed: int = 2012, steps: int = 2000,
                   grids=(128, 256, 384, 512), irec: int = config.IREC_MP5) -> list[Request]:
    """Seeded Poisson arrivals of 2D phi-slab tori: spin a ~ U[0, 0.99],
    r_pmax ~ U[10, 16], beta_min ~ U[30, 300], grid drawn from `grids`
    (n x n in r and theta), FP64 or mixed precision with probability 1/2."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        g = int(rng.choice(grids))
        prec = "mixed" if rng.random() < 0.5 else "fp64"
        a = float(rng.uniform(0.0, 0.99))
        p = dict(config.torus(nr=g, nth=g, akm=a, irec=irec, precision=prec), guard=1)
        ic = dict(seed=int(seed * 1000 + k), rmax=float(rng.uniform(10.0, 16.0)),
                  beta=float(rng.uniform(30.0, 300.0)))
        out.append(Request(k, t, p, steps, ic))
    return out


class Server:
    """Serve a list of requests on one context (see the module docstring)."""

    def __init__(self, ctx: Context, mem_budget: int, max_runs: int = 64, tick_steps: int = 50,
                 prep_workers: int = 4, keep_prims: bool = False):
        self.ctx = ctx
        self.mem_budget = int(mem_budget)
        self.max_runs = int(max_runs)
        self.tick_steps = int(tick_steps)
        self.keep_prims = keep_prims
        self.pool = cf.ThreadPoolExecutor(max_workers=prep_workers)

    @staticmethod
    def _prepare(req: Request) -> Prep:
        prep = Prep(req.params)
        prep.ic_torus(**req.ic)
        return prep

    def serve(self, requests: list[Request], clock=time.perf_counter, max_wall_s: float = 3600.0) -> dict:
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        nxt = 0                                  # next request to arrive
        waiting: list[tuple[Request, cf.Future, int]] = []
        active = []                              # [req, run, steps_done, admitted_at, bytes]
        finishing: dict[int, list] = {}          # tick -> runs that took their last steps in it
        used = 0
        done: list[Done] = []
        ticks = 0
        depth = 2                                # ticks in flight on the stream

        def retire(tick: int):
            # the tick has completed on the device: its finished runs are read back and released
            nonlocal used
            fin = clock() - t0
            for r, run, steps, admitted, nbytes in finishing.pop(tick, []):
                prims = run.prims() if self.keep_prims else None
                done.append(Done(r.rid, r.arrival, admitted, fin, config.interior_cells(r.params), steps,
                                 r.params.get("precision", "fp64"), prims))
                run.release()
                used -= nbytes

        while len(done) < len(reqs):
            now = clock() - t0
            if now > max_wall_s:
                raise RuntimeError(f"serving did not finish within {max_wall_s} s "
                                   f"({len(done)} of {len(reqs)} requests done)")
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                r = reqs[nxt]
                waiting.append((r, self.pool.submit(self._prepare, r), footprint(r.params)))
                nxt += 1
            # admission by slot and footprint; requests whose preparation is done, in arrival order
            for item in list(waiting):
                r, fut, nbytes = item
                if len(active) >= self.max_runs:
                    break
                if not fut.done() or used + nbytes > self.mem_budget:
                    continue
                prep = fut.result()
                run = self.ctx.admit_prep(prep)
                prep.close()
                active.append([r, run, 0, clock() - t0, nbytes])
                used += nbytes
                waiting.remove(item)
            if not active:
                if finishing:                    # drain: the last ticks complete
                    for t in sorted(finishing):
                        self.ctx.wait_mark(t % depth)
                        retire(t)
                    continue
                # idle: wait for the next arrival or a preparation
                if waiting:
                    cf.wait([f for _, f, _ in waiting], timeout=0.01, return_when=cf.FIRST_COMPLETED)
                elif nxt < len(reqs):
                    time.sleep(max(0.0, min(0.01, reqs[nxt].arrival - (clock() - t0))))
                continue
            # at most `depth` ticks in flight: the tick that last used this mark slot completes first
            if ticks >= depth:
                self.ctx.wait_mark(ticks % depth)
                retire(ticks - depth)
            n = min(self.tick_steps, min(a[0].steps - a[2] for a in active))
            self.ctx.step_batch([a[1] for a in active], n)
            self.ctx.mark(ticks % depth)
            for a in list(active):
                a[2] += n
                if a[2] >= a[0].steps:
                    finishing.setdefault(ticks, []).append(tuple(a))
                    active.remove(a)
            ticks += 1
        wall = clock() - t0
        lat = np.array([d.latency for d in done])
        zones = sum(d.zones * d.steps for d in done)
        return {
            "requests": len(done),
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()),
            "wall_s": wall,
            "zone_updates": zones,
            "zone_updates_per_s": zones / wall,
            "ticks": ticks,
            "ticks_in_flight": depth,
            "done": done,
        }

    def close(self):
        self.pool.shutdown(wait=True)
