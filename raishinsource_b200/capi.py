"""ctypes binding of the in-tree libraishin_gpu.so (include/raishin_gpu.h).

This is the host-side mirror of the reference's driver interface: a run is
admitted with its ``pram``-style parameter block, given initial data
(``mdtorus1`` or uploaded primitives), stepped on the GPU, and read back in the
reference layout a(nv,i,j,k).  The per-routine entry points keep the names of
the Fortran subroutines they replace (caluu1, calflx, recov, cdtcfl, bnd4).

There is no CPU fallback: every call goes through the CUDA library, and
loading fails loudly if the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .config import ghost_widths

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libraishin_gpu.so")

STATUS = {0: "RG_OK", 1: "RG_EINVAL_CONFIG", 2: "RG_ENOMEM_ADMIT", 3: "RG_ECUDA", 4: "RG_ENR_CAP",
          5: "RG_ENAN", 6: "RG_ENOTFOUND", 7: "RG_EOVERFLOW"}

#: every entry point include/raishin_gpu.h declares
EXPORTS = ("rg_last_error", "rg_ctx_create", "rg_ctx_destroy", "rg_sync", "rg_ctx_mark", "rg_ctx_wait_mark",
           "rg_ctx_set_stream", "rg_run_admit", "rg_run_release",
           "rg_prep_create", "rg_prep_ic_torus", "rg_run_admit_prep", "rg_prep_destroy",
           "rg_run_footprint", "rg_run_ic_torus", "rg_run_ic_torus_device", "rg_run_ic_tube", "rg_run_upload_prims", "rg_run_download_prims", "rg_run_layout", "rg_run_download_stored", "rg_step",
           "rg_run_stats", "rg_step_batch", "rg_batch_info", "rg_profile", "rg_profile_read", "rg_caluu1", "rg_calflx", "rg_rec2", "rg_calcha", "rg_hll", "rg_ct", "rg_recov", "rg_cdtcfl", "rg_bnd_floor", "rg_bnd4", "rg_infchk", "rg_atmosphere1a", "rg_pminmax2b", "rg_calsf", "rg_rkt", "rg_run_derived", "rg_run_divb", "rg_run_horizon_flux", "rg_run_radial_flux", "rg_run_store", "rg_run_restore", "rg_run_output", "rg_pow_eval", "rg_calflx_static")


class RgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class RunParams(C.Structure):
    _fields_ = [
        ("imax", C.c_int), ("jmax", C.c_int), ("kmax", C.c_int),
        ("metric", C.c_int), ("ix1", C.c_int), ("ix2", C.c_int), ("ix3", C.c_int),
        ("irec", C.c_int), ("model", C.c_int), ("iter", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("R0", C.c_double), ("hslope", C.c_double), ("akm", C.c_double), ("gam", C.c_double),
        ("cfl", C.c_double), ("dmin", C.c_double), ("pmin", C.c_double), ("pmax", C.c_double),
        ("tmax", C.c_double), ("dtmin", C.c_double),
        ("ibc", (C.c_int * 9) * 6),
        ("guard", C.c_int),
        ("precision", C.c_int),
        ("flags", C.c_int),
        ("ict", C.c_int),
        ("iwvec", C.c_int),
    ]


class StepStats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in
                ("steps", "recov_calls", "recov_nr2", "recov_fail", "recov_carry", "recov_cap", "floor_cap",
                 "carry_overflow")] + [("time", C.c_double), ("dt", C.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (building it first if the .so is absent or stale).

    RAISHIN_GPU_LIB=exact loads the uncontracted variant
    (libraishin_gpu_exact.so) instead; any other value is the path of a
    library to load."""
    global _lib
    if _lib is not None:
        return _lib
    from . import build as _build
    path = os.environ.get("RAISHIN_GPU_LIB", path)
    if path == LIB_PATH:
        path = _build.build()
    elif path == "exact":
        path = _build.build(variants=("exact",))
    lib = C.CDLL(path)
    P, D, I = C.c_void_p, C.POINTER(C.c_double), C.c_int
    lib.rg_last_error.restype = C.c_char_p
    lib.rg_ctx_create.argtypes = [I, C.POINTER(C.c_void_p)]
    lib.rg_ctx_destroy.argtypes = [P]
    lib.rg_sync.argtypes = [P]
    lib.rg_ctx_mark.argtypes = [P, I]
    lib.rg_ctx_wait_mark.argtypes = [P, I, I, C.POINTER(C.c_int)]
    lib.rg_ctx_set_stream.argtypes = [P, P]
    lib.rg_run_admit.argtypes = [P, C.POINTER(RunParams), C.POINTER(C.c_int)]
    lib.rg_run_release.argtypes = [P, I]
    lib.rg_prep_create.argtypes = [C.POINTER(RunParams), C.POINTER(C.c_void_p)]
    lib.rg_prep_ic_torus.argtypes = [P, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
    lib.rg_run_admit_prep.argtypes = [P, P, C.POINTER(C.c_int)]
    lib.rg_prep_destroy.argtypes = [P]
    lib.rg_run_footprint.argtypes = [C.POINTER(RunParams), C.POINTER(C.c_size_t)]
    lib.rg_run_ic_torus.argtypes = [P, I, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double]
    lib.rg_run_ic_torus_device.argtypes = [P, I, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double]
    lib.rg_run_ic_tube.argtypes = [P, I, C.c_uint64, C.c_uint64]
    lib.rg_run_upload_prims.argtypes = [P, I, C.c_void_p, C.c_double]
    lib.rg_run_download_prims.argtypes = [P, I, C.c_void_p]
    lib.rg_step.argtypes = [P, I, I, C.POINTER(StepStats)]
    lib.rg_run_layout.argtypes = [P, I, C.POINTER(C.c_size_t), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.rg_run_download_stored.argtypes = [P, I, C.c_void_p]
    lib.rg_run_stats.argtypes = [P, I, C.POINTER(StepStats)]
    lib.rg_step_batch.argtypes = [P, C.POINTER(C.c_int), I, I, C.POINTER(StepStats)]
    lib.rg_batch_info.argtypes = [P, C.POINTER(C.c_int), I, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    lib.rg_profile.argtypes = [P, I]
    lib.rg_profile_read.argtypes = [P, D, C.POINTER(C.c_longlong), I]
    lib.rg_caluu1.argtypes = [P, I, D, D]
    lib.rg_calflx.argtypes = [P, I, D, D]
    lib.rg_recov.argtypes = [P, I, D, D]
    lib.rg_rec2.argtypes = [P, I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rg_calcha.argtypes = [P, I, C.c_void_p, C.c_void_p]
    lib.rg_hll.argtypes = [P, I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rg_ct.argtypes = [P, I, C.c_void_p, C.c_void_p]
    lib.rg_cdtcfl.argtypes = [P, I, D, D]
    lib.rg_bnd_floor.argtypes = [P, I, D, D]
    lib.rg_bnd4.argtypes = [P, I, D, D]
    for f in ("rg_infchk", "rg_atmosphere1a", "rg_pminmax2b"):
        getattr(lib, f).argtypes = [P, I, D]
    lib.rg_calsf.argtypes = [P, I, D, D]
    lib.rg_rkt.argtypes = [P, I, I, C.c_double, D, D, D, D, D]
    lib.rg_run_derived.argtypes = [P, I, I, D]
    lib.rg_calflx_static.argtypes = [P, I, P, P]
    lib.rg_pow_eval.argtypes = [P, D, D, D, C.c_size_t]
    lib.rg_run_horizon_flux.argtypes = [P, I, D, D]
    lib.rg_run_divb.argtypes = [P, I, D, D]
    lib.rg_run_output.argtypes = [P, I, C.c_char_p, I, I]
    lib.rg_run_radial_flux.argtypes = [P, I, I, D, D]
    lib.rg_run_store.argtypes = [P, I, C.c_char_p, I, I, I, C.c_void_p]
    lib.rg_run_restore.argtypes = [P, I, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.c_void_p]
    _lib = lib
    return lib


def _check(lib, rc: int):
    if rc != 0:
        raise RgError(rc, lib.rg_last_error().decode(errors="replace"))


def make_params(p: dict) -> RunParams:
    o = RunParams()
    for name, _ in RunParams._fields_:
        if name == "ibc":
            for s in range(6):
                for m in range(9):
                    o.ibc[s][m] = int(p["ibc"][s][m])
        elif name == "guard":
            o.guard = int(p.get("guard", 0))
        elif name == "flags":
            o.flags = int(p.get("flags", 0))
        elif name == "ict":
            o.ict = int(p.get("ict", 1))
        elif name == "iwvec":
            o.iwvec = int(p.get("iwvec", 1))
        elif name == "precision":
            o.precision = {"fp64": 0, "mixed": 1}[p.get("precision", "fp64")]
        else:
            setattr(o, name, p[name])
    return o


def footprint(p: dict) -> int:
    lib = load()
    n = C.c_size_t(0)
    _check(lib, lib.rg_run_footprint(C.byref(make_params(p)), C.byref(n)))
    return n.value


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """One CUDA stream on one device (rg_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        _check(self.lib, self.lib.rg_ctx_create(int(device), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.rg_ctx_destroy(self.h)
            self.h = None

    def sync(self):
        _check(self.lib, self.lib.rg_sync(self.h))

    def mark(self, slot: int):
        """Record a point of the context stream in slot 0..7 (rg_ctx_mark)."""
        _check(self.lib, self.lib.rg_ctx_mark(self.h, slot))

    def wait_mark(self, slot: int, block: bool = True) -> bool:
        """True once the work before the mark has completed (blocking by default)."""
        done = C.c_int(0)
        _check(self.lib, self.lib.rg_ctx_wait_mark(self.h, slot, int(block), C.byref(done)))
        return bool(done.value)

    def set_stream(self, stream_handle: int):
        """Issue all later work on a caller-owned cudaStream_t (e.g. torch's current stream)."""
        _check(self.lib, self.lib.rg_ctx_set_stream(self.h, C.c_void_p(stream_handle)))

    KINDS = ("cfl", "flux_r", "flux_phi", "flux_theta", "flux_ct", "update", "ghost_fill", "floors", "scalar")

    def profile(self, enable: bool = True):
        """Clear kernel timers/launch counters; with enable, time every launch with CUDA events."""
        _check(self.lib, self.lib.rg_profile(self.h, int(bool(enable))))

    def profile_read(self) -> dict:
        n = len(self.KINDS)
        ms = (C.c_double * n)()
        cnt = (C.c_longlong * n)()
        _check(self.lib, self.lib.rg_profile_read(self.h, ms, cnt, n))
        return {k: {"ms": ms[i], "launches": cnt[i]} for i, k in enumerate(self.KINDS)}

    def pow_eval(self, x, y) -> np.ndarray:
        """x**y elementwise on the device by the uncontracted build's power
        function (rg_pow of include/rg_pow.h; rg_pow_eval)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(np.broadcast_to(y, x.shape), dtype=np.float64)
        out = np.empty_like(x)
        _check(self.lib, self.lib.rg_pow_eval(self.h, _dptr(x), _dptr(y), _dptr(out), x.size))
        return out

    def admit(self, params: dict) -> "Run":
        return Run(self, params)

    def admit_prep(self, prep: Prep) -> "Run":
        """Admit a prepared run (geometry and initial data computed by Prep)."""
        return Run(self, prep.params, prep)

    def step_batch(self, runs, n: int = 1, stats: bool = False, strict: bool = True):
        """Advance several runs together (rg_step_batch); with stats, one dict per run.
        With strict=False a capped rescale loop (RG_ENR_CAP, counted in the stats)
        does not raise."""
        ids = (C.c_int * len(runs))(*[r.id for r in runs])
        st = (StepStats * len(runs))() if stats else None
        rc = self.lib.rg_step_batch(self.h, ids, len(runs), int(n), st)
        if not (rc == 4 and not strict):
            _check(self.lib, rc)
        return [x.as_dict() for x in st] if stats else None

    def batch_info(self, runs) -> dict:
        """Tuned shape of the batch of exactly these runs."""
        ids = (C.c_int * len(runs))(*[r.id for r in runs])
        w, f, nl, ms, tc = C.c_int(0), C.c_int(0), C.c_int(0), C.c_double(0), C.c_int(0)
        _check(self.lib, self.lib.rg_batch_info(self.h, ids, len(runs), C.byref(w), C.byref(f), C.byref(nl),
                                                C.byref(ms), C.byref(tc)))
        return {"width": w.value, "tile_cells": tc.value, "grid_per_sm": f.value, "launches_per_step": nl.value,
                "tuned_ms_per_step": ms.value}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Prep:
    """Host-side preparation of a run (rg_prep_*): geometry and, optionally,
    torus initial data, computed without a context on any thread."""

    def __init__(self, params: dict):
        self.lib = load()
        self.params = dict(params)
        self._p = make_params(params)
        h = C.c_void_p()
        _check(self.lib, self.lib.rg_prep_create(C.byref(self._p), C.byref(h)))
        self.h = h

    def ic_torus(self, seed=2012, amp=0.04, rin=6.0, rmax=12.0, beta=100.0, kappa=1e-3):
        _check(self.lib, self.lib.rg_prep_ic_torus(self.h, seed, amp, rin, rmax, beta, kappa))
        return self

    def close(self):
        if self.h:
            self.lib.rg_prep_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Run:
    """One admitted run: device-resident state of one grid."""

    def __init__(self, ctx: Context, params: dict, prep: "Prep | None" = None):
        self.ctx, self.lib = ctx, ctx.lib
        self.params = dict(params)
        self._p = make_params(params)
        rid = C.c_int(0)
        if prep is None:
            _check(self.lib, self.lib.rg_run_admit(ctx.h, C.byref(self._p), C.byref(rid)))
        else:
            _check(self.lib, self.lib.rg_run_admit_prep(ctx.h, prep.h, C.byref(rid)))
        self.id = rid.value
        self.shape = (params["kmax"], params["jmax"], params["imax"], 9)
        self.nm0, self.nm1 = ghost_widths(params["irec"], params.get("ict", 1))

    def release(self):
        if self.id:
            self.lib.rg_run_release(self.ctx.h, self.id)
            self.id = 0

    def zeros(self):
        return np.zeros(self.shape, dtype=np.float64)

    # initial data / state transfer
    def ic_torus(self, seed=2012, amp=0.04, rin=6.0, rmax=12.0, beta=100.0, kappa=1e-3):
        _check(self.lib, self.lib.rg_run_ic_torus(self.ctx.h, self.id, seed, amp, rin, rmax, beta, kappa))

    def ic_torus_device(self, seed=2012, amp=0.04, rin=6.0, rmax=12.0, beta=100.0, kappa=1e-3):
        """The torus initial data of ic_torus computed on the device (rg_run_ic_torus_device)."""
        _check(self.lib, self.lib.rg_run_ic_torus_device(self.ctx.h, self.id, seed, amp, rin, rmax, beta, kappa))

    def ic_tube(self, seed=2012, tube=0):
        """Seeded 1D Riemann problem (left state for i <= imax/2, pattern of mdshoctub)."""
        _check(self.lib, self.lib.rg_run_ic_tube(self.ctx.h, self.id, seed, tube))

    def upload_prims(self, uri, t0: float = 0.0):
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        _check(self.lib, self.lib.rg_run_upload_prims(self.ctx.h, self.id, uri.ctypes.data, float(t0)))

    def upload_prims_ptr(self, host_ptr: int, t0: float = 0.0):
        """Upload from a raw host pointer (e.g. pinned memory), layout a(nv,i,j,k)."""
        _check(self.lib, self.lib.rg_run_upload_prims(self.ctx.h, self.id, C.c_void_p(host_ptr), float(t0)))

    def prims(self) -> np.ndarray:
        out = self.zeros()
        _check(self.lib, self.lib.rg_run_download_prims(self.ctx.h, self.id, out.ctypes.data))
        return out

    def stored_prims(self) -> np.ndarray:
        """Primitives as stored on the device, shape (9, kplanes, jplanes, imax):
        a slab direction has one plane (rg_run_download_stored)."""
        n, jp, kp = C.c_size_t(0), C.c_int(0), C.c_int(0)
        _check(self.lib, self.lib.rg_run_layout(self.ctx.h, self.id, C.byref(n), C.byref(jp), C.byref(kp)))
        out = np.empty((9, kp.value, jp.value, self.params["imax"]), dtype=np.float64)
        _check(self.lib, self.lib.rg_run_download_stored(self.ctx.h, self.id, out.ctypes.data))
        return out

    def download_prims_ptr(self, host_ptr: int):
        _check(self.lib, self.lib.rg_run_download_prims(self.ctx.h, self.id, C.c_void_p(host_ptr)))

    # time stepping
    def step(self, n: int = 1, stats: bool = False, strict: bool = True):
        """Advance the run n steps (rg_step).  With strict=False a capped
        rescale loop (RG_ENR_CAP, counted in the stats) does not raise."""
        st = StepStats()
        rc = self.lib.rg_step(self.ctx.h, self.id, int(n), C.byref(st) if stats else None)
        if not (rc == 4 and not strict):
            _check(self.lib, rc)
        return st.as_dict() if stats else None

    def stats(self) -> dict:
        st = StepStats()
        _check(self.lib, self.lib.rg_run_stats(self.ctx.h, self.id, C.byref(st)))
        return st.as_dict()

    # reference-interface entry points (host arrays, layout a(nv,i,j,k))
    def caluu1(self, uri) -> np.ndarray:
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = self.zeros()
        _check(self.lib, self.lib.rg_caluu1(self.ctx.h, self.id, _dptr(uri), _dptr(out)))
        return out

    def calflx(self, uri) -> np.ndarray:
        """ww(3,nv,i,j,k) as shape (kmax, jmax, imax, 9, 3)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = np.zeros(self.shape + (3,), dtype=np.float64)
        _check(self.lib, self.lib.rg_calflx(self.ctx.h, self.id, _dptr(uri), _dptr(out)))
        return out

    def rec2(self, uri, cons: bool = True):
        """rg_rec2: (face primitives, face conserved variables, face fluxes),
        each of shape (6, kmax, jmax, imax, 9) in the order ?l, ?r for ? = i, j, k
        (the latter two None unless cons)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = [np.zeros((6,) + self.shape, dtype=np.float64) for _ in range(3 if cons else 1)]
        ptrs = [o.ctypes.data for o in out] + [None] * (3 - len(out))
        _check(self.lib, self.lib.rg_rec2(self.ctx.h, self.id, uri.ctypes.data, *ptrs))
        return tuple(out) + (None,) * (3 - len(out))

    def calcha(self, faces) -> np.ndarray:
        """rg_calcha: speeds (6, kmax, jmax, imax) from face primitives (6, ...)."""
        faces = np.ascontiguousarray(faces, dtype=np.float64)
        out = np.zeros((6,) + self.shape[:3], dtype=np.float64)
        _check(self.lib, self.lib.rg_calcha(self.ctx.h, self.id, faces.ctypes.data, out.ctypes.data))
        return out

    def hll(self, cons, flux, cha, ww) -> np.ndarray:
        """rg_hll: the updated copy of ww (kmax, jmax, imax, 9, 3)."""
        cons = np.ascontiguousarray(cons, dtype=np.float64)
        flux = np.ascontiguousarray(flux, dtype=np.float64)
        cha = np.ascontiguousarray(cha, dtype=np.float64)
        out = np.array(ww, dtype=np.float64, order="C").reshape(self.shape + (3,))
        _check(self.lib, self.lib.rg_hll(self.ctx.h, self.id, cons.ctypes.data, flux.ctypes.data, cha.ctypes.data,
                                         out.ctypes.data))
        return out

    def ct(self, uri, ww) -> np.ndarray:
        """rg_ct: the updated copy of ww (kmax, jmax, imax, 9, 3)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = np.array(ww, dtype=np.float64, order="C").reshape(self.shape + (3,))
        _check(self.lib, self.lib.rg_ct(self.ctx.h, self.id, uri.ctypes.data, out.ctypes.data))
        return out

    def recov(self, uu, uri) -> np.ndarray:
        uu = np.ascontiguousarray(uu, dtype=np.float64).reshape(self.shape)
        out = np.array(uri, dtype=np.float64, order="C").reshape(self.shape)
        _check(self.lib, self.lib.rg_recov(self.ctx.h, self.id, _dptr(uu), _dptr(out)))
        return out

    def derived(self, jslice: int = 0) -> np.ndarray:
        """Derived quantities of the output converter (rg_run_derived):
        (gfa, gfb, b^2, -h u_t, v_r, v_phi, v_theta) per point, shape
        (kmax, jmax, imax, 7), or (kmax, imax, 7) for the plane jslice."""
        p = self.params
        shape = (p["kmax"], p["imax"], 7) if jslice else (p["kmax"], p["jmax"], p["imax"], 7)
        out = np.zeros(shape, dtype=np.float64)
        _check(self.lib, self.lib.rg_run_derived(self.ctx.h, self.id, jslice, _dptr(out)))
        return out

    def calsf(self, uri) -> np.ndarray:
        """sf(2:5,i,j,k) as shape (kmax, jmax, imax, 4)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = np.zeros(self.shape[:3] + (4,), dtype=np.float64)
        _check(self.lib, self.lib.rg_calsf(self.ctx.h, self.id, _dptr(uri), _dptr(out)))
        return out

    def rkt(self, stage: int, dt: float, ww, uo, ucur, sf, unew) -> np.ndarray:
        """One RK3 stage (rg_rkt); returns the updated copy of unew."""
        ww = np.ascontiguousarray(ww, dtype=np.float64).reshape(self.shape + (3,))
        ucur = np.ascontiguousarray(ucur, dtype=np.float64).reshape(self.shape)
        sf = np.ascontiguousarray(sf, dtype=np.float64).reshape(self.shape[:3] + (4,))
        out = np.array(unew, dtype=np.float64, order="C").reshape(self.shape)
        uo_p = None
        if uo is not None:
            uo = np.ascontiguousarray(uo, dtype=np.float64).reshape(self.shape)
            uo_p = _dptr(uo)
        _check(self.lib, self.lib.rg_rkt(self.ctx.h, self.id, stage, dt, _dptr(ww), uo_p, _dptr(ucur), _dptr(sf),
                                         _dptr(out)))
        return out

    def cdtcfl(self, uri) -> float:
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = C.c_double(0.0)
        _check(self.lib, self.lib.rg_cdtcfl(self.ctx.h, self.id, _dptr(uri), C.byref(out)))
        return out.value

    def calflx_static(self, d_prims: int, d_ww: int):
        """Allocation-free flux call on caller-owned device buffers (raw device
        pointers): d_prims 9*N SoA primitives in, d_ww 27*N fluxes out."""
        _check(self.lib, self.lib.rg_calflx_static(self.ctx.h, self.id, C.c_void_p(d_prims), C.c_void_p(d_ww)))

    def store(self, path: str, it0: int = 0, ih0: int = 0, nd: int = 0, uri0=None):
        """Write a restart file in the store1 layout (rg_run_store)."""
        ptr = None
        if uri0 is not None:
            uri0 = np.ascontiguousarray(uri0, dtype=np.float64).reshape(self.shape)
            ptr = uri0.ctypes.data
        _check(self.lib, self.lib.rg_run_store(self.ctx.h, self.id, os.fsencode(path), it0, ih0, nd, ptr))

    def output(self, path: str, myrank: int = 0, npe: int = 1):
        """Write output1's snapshot file of the current state (rg_run_output)."""
        _check(self.lib, self.lib.rg_run_output(self.ctx.h, self.id, os.fsencode(path), int(myrank), int(npe)))

    def restore(self, path: str) -> dict:
        """Read a restart file of this grid (rg_run_restore); returns it0, ih0, nd and uri0."""
        it0, ih0, nd = C.c_int(0), C.c_int(0), C.c_int(0)
        uri0 = self.zeros()
        _check(self.lib, self.lib.rg_run_restore(self.ctx.h, self.id, os.fsencode(path), C.byref(it0), C.byref(ih0),
                                                 C.byref(nd), uri0.ctypes.data))
        return {"it0": it0.value, "ih0": ih0.value, "nd": nd.value, "uri0": uri0}

    def horizon_flux(self) -> tuple[float, float]:
        """(mdot, edot) through the inner edge of the interior (rg_run_horizon_flux)."""
        m, e = C.c_double(0), C.c_double(0)
        _check(self.lib, self.lib.rg_run_horizon_flux(self.ctx.h, self.id, C.byref(m), C.byref(e)))
        return m.value, e.value

    def radial_flux(self, iface: int) -> tuple[float, float]:
        """(mdot, edot) through the radial face iface+1/2 (rg_run_radial_flux)."""
        m, e = C.c_double(0), C.c_double(0)
        _check(self.lib, self.lib.rg_run_radial_flux(self.ctx.h, self.id, int(iface), C.byref(m), C.byref(e)))
        return m.value, e.value

    def divb(self) -> tuple[float, float]:
        """(max |D|, B scale) of the corner-centred div(sqrt(-g) B) of the
        current state (rg_run_divb)."""
        m, b = C.c_double(0), C.c_double(0)
        _check(self.lib, self.lib.rg_run_divb(self.ctx.h, self.id, C.byref(m), C.byref(b)))
        return m.value, b.value

    def bnd_part(self, which: str, uri, urio=None) -> np.ndarray:
        """bnd4 (needs urio), infchk, atmosphere1a or pminmax2b alone; the updated copy of uri."""
        out = np.array(uri, dtype=np.float64, order="C").reshape(self.shape)
        if which == "bnd4":
            urio = np.ascontiguousarray(urio, dtype=np.float64).reshape(self.shape)
            _check(self.lib, self.lib.rg_bnd4(self.ctx.h, self.id, _dptr(out), _dptr(urio)))
        else:
            fn = {"infchk": self.lib.rg_infchk, "atmosphere1a": self.lib.rg_atmosphere1a,
                  "pminmax2b": self.lib.rg_pminmax2b}[which]
            _check(self.lib, fn(self.ctx.h, self.id, _dptr(out)))
        return out

    def bnd_floor(self, uri, urio) -> np.ndarray:
        out = np.array(uri, dtype=np.float64, order="C").reshape(self.shape)
        urio = np.ascontiguousarray(urio, dtype=np.float64).reshape(self.shape)
        _check(self.lib, self.lib.rg_bnd_floor(self.ctx.h, self.id, _dptr(out), _dptr(urio)))
        return out
