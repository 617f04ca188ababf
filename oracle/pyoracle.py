"""ctypes binding of oracle/_build/liboracle.so (test infrastructure only).

Arrays use the reference layout a(nv,i,j,k), which as a C-ordered numpy array
has shape (kmax, jmax, imax, 9).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build_oracle as _build_mod

_LIB = None


class OrcParams(C.Structure):
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
        ("ict", C.c_int),
        ("iwvec", C.c_int),
    ]


class OrcStats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in
                ("recov_calls", "recov_nr2", "recov_fail", "recov_carry", "recov_cap", "floor_cap")]


def build(force: bool = False) -> str:
    return _build_mod.build(force=force)


def _lib():
    global _LIB
    if _LIB is None:
        path = build()
        lib = C.CDLL(path)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        lib.orc_create.restype = P
        lib.orc_create.argtypes = [C.POINTER(OrcParams)]
        lib.orc_destroy.argtypes = [P]
        lib.orc_nm1.argtypes = [P]
        lib.orc_nm1.restype = C.c_int
        lib.orc_ic_torus.argtypes = [P, C.c_ulonglong, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double]
        lib.orc_ic_tube.argtypes = [P, C.c_ulonglong, C.c_ulonglong]
        for f in ("orc_set_prims", "orc_get_prims", "orc_get_cons"):
            getattr(lib, f).argtypes = [P, D]
        lib.orc_init_cons.argtypes = [P]
        lib.orc_step.argtypes = [P, C.c_int]
        lib.orc_step.restype = C.c_int
        lib.orc_time.argtypes = [P]
        lib.orc_time.restype = C.c_double
        lib.orc_dt.argtypes = [P]
        lib.orc_dt.restype = C.c_double
        lib.orc_get_stats.argtypes = [P, C.POINTER(OrcStats)]
        lib.orc_caluu1.argtypes = [P, D, D]
        lib.orc_fluxes.argtypes = [P, D, D]
        lib.orc_recov.argtypes = [P, D, D]
        lib.orc_cdtcfl.argtypes = [P, D]
        lib.orc_cdtcfl.restype = C.c_double
        lib.orc_bnd_floor.argtypes = [P, D, D]
        lib.orc_calsf.argtypes = [P, D, D]
        lib.orc_rec2.argtypes = [P, D, D]
        lib.orc_ct.argtypes = [P, D, D]
        lib.orc_derived.argtypes = [P, D, C.c_int, D]
        lib.orc_rkt.argtypes = [P, C.c_int, C.c_double, D, D, D, D, D]
        lib.orc_get_array.argtypes = [P, C.c_char_p, D, C.c_longlong]
        lib.orc_get_array.restype = C.c_longlong
        lib.orc_rec2_full.argtypes = [P, D, D, D, D]
        lib.orc_bnd_part.argtypes = [P, C.c_int, D, D]
        lib.orc_calcha.argtypes = [P, D, D]
        lib.orc_hll.argtypes = [P, D, D, D, D]
        lib.orc_output1.argtypes = [P, C.c_char_p, C.c_int, C.c_int]
        lib.orc_output1.restype = C.c_int
        lib.orc_set_pow_mode.argtypes = [C.c_int]
        lib.orc_set_pow_mode.restype = C.c_int
        lib.orc_pow_eval.argtypes = [D, D, D, C.c_longlong, C.c_int]
        _LIB = lib
    return _LIB


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_pow_mode(mode: str) -> str:
    """Power function of the oracle's step: "libc" (the C library's pow, as
    the reference's gfortran build calls it; the default) or "rg" (rg_pow of
    include/rg_pow.h, the uncontracted GPU build's).  Returns the previous
    mode.  Process-wide."""
    old = _lib().orc_set_pow_mode({"libc": 0, "rg": 1}[mode])
    return "rg" if old else "libc"


def pow_eval(x: np.ndarray, y: np.ndarray, mode: str) -> np.ndarray:
    """x**y elementwise by the C library's pow ("libc") or rg_pow ("rg")."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(np.broadcast_to(y, x.shape), dtype=np.float64)
    out = np.empty_like(x)
    _lib().orc_pow_eval(_ptr(x), _ptr(y), _ptr(out), x.size, {"libc": 0, "rg": 1}[mode])
    return out


def make_params(p: dict) -> OrcParams:
    o = OrcParams()
    for name, _ in OrcParams._fields_:
        if name == "ibc":
            for s in range(6):
                for m in range(9):
                    o.ibc[s][m] = int(p["ibc"][s][m])
        else:
            default = {"guard": 0, "ict": 1, "iwvec": 1}
            setattr(o, name, p.get(name, default[name]) if name in default else p[name])
    return o


class Oracle:
    """One reference-semantics run on the CPU (single MPI rank)."""

    def __init__(self, params: dict):
        self.params = dict(params)
        self._p = make_params(params)
        self.lib = _lib()
        self.h = self.lib.orc_create(C.byref(self._p))
        self.shape = (params["kmax"], params["jmax"], params["imax"], 9)
        self.nm1 = self.lib.orc_nm1(self.h)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def zeros(self):
        return np.zeros(self.shape, dtype=np.float64)

    def ic_torus(self, seed=2012, amp=0.04, rin=6.0, rmax=12.0, beta=100.0, kappa=1e-3):
        self.lib.orc_ic_torus(self.h, seed, amp, rin, rmax, beta, kappa)

    def ic_tube(self, seed=2012, tube=0):
        """Seeded 1D Riemann problem (left state for i <= imax/2, pattern of mdshoctub)."""
        self.lib.orc_ic_tube(self.h, seed, tube)

    def set_prims(self, uri: np.ndarray):
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        self.lib.orc_set_prims(self.h, _ptr(uri))

    def prims(self) -> np.ndarray:
        out = self.zeros()
        self.lib.orc_get_prims(self.h, _ptr(out))
        return out

    def cons(self) -> np.ndarray:
        out = self.zeros()
        self.lib.orc_get_cons(self.h, _ptr(out))
        return out

    def init_cons(self):
        self.lib.orc_init_cons(self.h)

    def step(self, n: int = 1) -> int:
        return self.lib.orc_step(self.h, int(n))

    @property
    def time(self) -> float:
        return self.lib.orc_time(self.h)

    @property
    def dt(self) -> float:
        return self.lib.orc_dt(self.h)

    def stats(self) -> dict:
        st = OrcStats()
        self.lib.orc_get_stats(self.h, C.byref(st))
        return {n: getattr(st, n) for n, _ in OrcStats._fields_}

    def caluu1(self, uri):
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = self.zeros()
        self.lib.orc_caluu1(self.h, _ptr(uri), _ptr(out))
        return out

    def fluxes(self, uri):
        """ww(3,nv,i,j,k) as shape (kmax, jmax, imax, 9, 3)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = np.zeros(self.shape + (3,), dtype=np.float64)
        self.lib.orc_fluxes(self.h, _ptr(uri), _ptr(out))
        return out

    def ct(self, uri, ww):
        """ct (the run's ict) applied to given fluxes ww of shape (kmax, jmax, imax, 9, 3)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = np.array(ww, dtype=np.float64, order="C").reshape(self.shape + (3,))
        self.lib.orc_ct(self.h, _ptr(uri), _ptr(out))
        return out

    def recov(self, uu, uri):
        uu = np.array(uu, dtype=np.float64, order="C").reshape(self.shape)
        uri = np.array(uri, dtype=np.float64, order="C").reshape(self.shape)
        self.lib.orc_recov(self.h, _ptr(uu), _ptr(uri))
        return uu, uri

    def rec2(self, uri) -> np.ndarray:
        """Face states of rec2: shape (6,) + prims shape, in the order uriil,
        uriir, urijl, urijr, urikl, urikr (unset entries are 0)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = np.zeros((6,) + self.shape, dtype=np.float64)
        self.lib.orc_rec2(self.h, _ptr(uri), _ptr(out))
        return out

    def rec2_full(self, uri):
        """rec2 with caluu3/calflx3: (prims, cons, flux), each of shape (6,) +
        prims shape in the order ?il, ?ir for ? = i, j, k."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = [np.zeros((6,) + self.shape, dtype=np.float64) for _ in range(3)]
        self.lib.orc_rec2_full(self.h, _ptr(uri), _ptr(out[0]), _ptr(out[1]), _ptr(out[2]))
        return tuple(out)

    def calcha(self, faces):
        """calcha from face primitives (6, kmax, jmax, imax, 9): cmax/cmin per
        direction, shape (6, kmax, jmax, imax) (cmaxi, cmini, cmaxj, cminj, cmaxk, cmink)."""
        faces = np.ascontiguousarray(faces, dtype=np.float64)
        out = np.zeros((6,) + self.shape[:3], dtype=np.float64)
        self.lib.orc_calcha(self.h, _ptr(faces), _ptr(out))
        return out

    def hll(self, cons, flux, cha, ww):
        """hll from face conserved variables and fluxes (6, ...) and speeds (6, ...);
        returns the updated copy of ww (kmax, jmax, imax, 9, 3)."""
        cons = np.ascontiguousarray(cons, dtype=np.float64)
        flux = np.ascontiguousarray(flux, dtype=np.float64)
        cha = np.ascontiguousarray(cha, dtype=np.float64)
        out = np.array(ww, dtype=np.float64, order="C").reshape(self.shape + (3,))
        self.lib.orc_hll(self.h, _ptr(cons), _ptr(flux), _ptr(cha), _ptr(out))
        return out

    def derived(self, uri, jslice: int = 0) -> np.ndarray:
        """The output converter's derived quantities (gfa, gfb, b^2, -h u_t,
        v_r, v_phi, v_theta): shape (kmax, jmax, imax, 7), or (kmax, imax, 7)
        for the phi plane jslice."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        p = self.params
        shape = (p["kmax"], p["imax"], 7) if jslice else (p["kmax"], p["jmax"], p["imax"], 7)
        out = np.zeros(shape, dtype=np.float64)
        self.lib.orc_derived(self.h, _ptr(uri), jslice, _ptr(out))
        return out

    def calsf(self, uri) -> np.ndarray:
        """sf(2:5,i,j,k) of every cell, shape (kmax, jmax, imax, 4)."""
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        out = np.zeros(self.shape[:3] + (4,), dtype=np.float64)
        self.lib.orc_calsf(self.h, _ptr(uri), _ptr(out))
        return out

    def rkt(self, stage: int, dt: float, ww, uo, ucur, sf, unew) -> np.ndarray:
        """One RK3 stage of rkt.f90; returns the updated copy of unew."""
        ww = np.ascontiguousarray(ww, dtype=np.float64).reshape(self.shape + (3,))
        ucur = np.ascontiguousarray(ucur, dtype=np.float64).reshape(self.shape)
        sf = np.ascontiguousarray(sf, dtype=np.float64).reshape(self.shape[:3] + (4,))
        uo = ucur if uo is None else np.ascontiguousarray(uo, dtype=np.float64).reshape(self.shape)
        out = np.array(unew, dtype=np.float64, order="C").reshape(self.shape)
        self.lib.orc_rkt(self.h, stage, dt, _ptr(ww), _ptr(uo), _ptr(ucur), _ptr(sf), _ptr(out))
        return out

    def cdtcfl(self, uri) -> float:
        uri = np.ascontiguousarray(uri, dtype=np.float64).reshape(self.shape)
        return self.lib.orc_cdtcfl(self.h, _ptr(uri))

    def output1(self, path: str, myrank: int = 0, npe: int = 1):
        """Write the current primitives as output1's structr file (restar.f90:91-185)."""
        if self.lib.orc_output1(self.h, os.fsencode(path), myrank, npe) != 0:
            raise OSError("orc_output1 failed: " + path)

    def bnd_part(self, which: str, uri, urio=None):
        """bnd4, infchk, atmosphere1a or pminmax2b alone; returns the updated copy of uri."""
        out = np.array(uri, dtype=np.float64, order="C").reshape(self.shape)
        po = None
        if urio is not None:
            urio = np.ascontiguousarray(urio, dtype=np.float64).reshape(self.shape)
            po = _ptr(urio)
        code = {"bnd4": 0, "infchk": 1, "atmosphere1a": 2, "pminmax2b": 3}[which]
        self.lib.orc_bnd_part(self.h, code, _ptr(out), po)
        return out

    def bnd_floor(self, uri, urio):
        uri = np.array(uri, dtype=np.float64, order="C").reshape(self.shape)
        urio = np.ascontiguousarray(urio, dtype=np.float64).reshape(self.shape)
        self.lib.orc_bnd_floor(self.h, _ptr(uri), _ptr(urio))
        return uri

    def array(self, name: str) -> np.ndarray:
        p = self.params
        cap = 64 * p["imax"] * p["kmax"] + max(p["imax"], p["jmax"], p["kmax"])
        buf = np.zeros(cap, dtype=np.float64)
        n = self.lib.orc_get_array(self.h, name.encode(), _ptr(buf), cap)
        if n < 0:
            raise KeyError(name)
        return buf[:n].copy()
