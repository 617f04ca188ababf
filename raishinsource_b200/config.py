"""Run-parameter blocks for the GRMHD update.

The reference configures everything at compile time in ``module pram``
(pram.f90:1-80).  Here one run is described by a plain dict with the same
field names, which :mod:`raishinsource_b200.capi` packs into the C struct
``rg_run_params`` (include/raishin_gpu.h).

Conventions kept from the reference (coord.f90:597-610, grid.f90:25-46):
index i = x1 = r, j = x2 = phi, k = x3 = theta; ghost cells are inside
imax/jmax/kmax; x1(1) = xmin and x1(imax) = xmax are the first and last cell
centres, ghosts included.
"""
from __future__ import annotations

import math

PI = 3.14159265358979323  # pram.f90:30

# reconstruction selectors (pram.f90:122-131 / rec.f90:61-112)
IREC_MC, IREC_MINMOD, IREC_MUSCL, IREC_PPM, IREC_MP5, IREC_WENO5, IREC_WENOZ = 1, 2, 3, 5, 6, 7, 9
IREC_CENO, IREC_MPWENO, IREC_WENOM, IREC_LIMO3, IREC_MVL, IREC_KOREN = 4, 8, 10, 11, 12, 13
SECOND_ORDER = (IREC_MC, IREC_MINMOD, IREC_MUSCL, IREC_LIMO3, IREC_MVL, IREC_KOREN)

# rg_run_params.flags: compute every cell of a slab direction instead of one plane
FLAG_FULL = 1

# boundary codes (bnd.f90:398-413)
BC_PERIODIC, BC_COPY, BC_ANTISYM, BC_SYM, BC_OUTFLOW18 = 1, 5, 12, 14, 18


def ghost_widths(irec: int, ict: int = 1) -> tuple[int, int]:
    """(nm0, nm1) of main.f90:176-199: nm1 = nm0 + ict (ict = 1: flux-CT)."""
    nm0 = 2 if irec in SECOND_ORDER else (4 if irec == IREC_PPM else 3)
    return nm0, nm0 + ict


def torus_bcs() -> list[list[int]]:
    """pram.f90:75-80: r copy (vars 2-4 outflow-only at r_out), phi periodic,
    theta symmetric with u^theta and B^theta antisymmetric."""
    return [
        [5] * 9,
        [5, 18, 18, 18, 5, 5, 5, 5, 5],
        [1] * 9,
        [1] * 9,
        [14, 14, 14, 12, 14, 14, 14, 14, 12],
        [14, 14, 14, 12, 14, 14, 14, 14, 12],
    ]


def torus(nr: int = 256, nth: int = 256, nph: int | None = None, irec: int = IREC_MP5,
          akm: float = 0.9375, rmin: float = 1.9, rmax: float = 50.0, cfl: float = 0.4,
          precision: str = "fp64", ict: int = 1) -> dict:
    """Fishbone-Moncrief torus in modified Kerr-Schild coordinates.

    ``nr`` x ``nth`` x ``nph`` are imax x kmax x jmax including ghosts.  With
    ``nph=None`` the run is the 2D axisymmetric case: a periodic phi slab of
    jmax = 2*nm1+1 cells (one interior cell).  phi spans 2*pi over the
    interior: dphi = 2*pi/(jmax-2*nm1), x2(j) = (j-nm1-1/2)*dphi.  ``ict``
    selects the constrained transport (1 flux-CT, 2 modified flux-CT, 3 upwind
    flux-CT, 0 none).
    """
    _, nm1 = ghost_widths(irec, ict)
    jmax = 2 * nm1 + 1 if nph is None else int(nph)
    dphi = 2.0 * math.pi / (jmax - 2 * nm1)
    ymin = (0.5 - nm1) * dphi
    ymax = ymin + (jmax - 1) * dphi
    return dict(
        imax=int(nr), jmax=jmax, kmax=int(nth), metric=403, ix1=2, ix2=1, ix3=2, irec=irec, model=7,
        iter=5000, xmin=rmin, xmax=rmax, ymin=ymin, ymax=ymax, zmin=0.02, zmax=PI - 0.02,
        R0=0.0, hslope=0.5, akm=akm, gam=4.0 / 3.0, cfl=cfl, dmin=1.0e-4, pmin=1.0e-6, pmax=1.0e6,
        tmax=1.0e30, dtmin=1.0e-9, ibc=torus_bcs(), precision=precision, ict=ict,
    )


def tube(n: int = 400, irec: int = IREC_MP5, cfl: float = 0.4, tmax: float = 0.4,
         precision: str = "fp64", ict: int = 1) -> dict:
    """1D RMHD shock tube in Minkowski space (metric 1, model 2): x in [1, 2]
    (cell centres, ghosts included; x > 0 because the floors use x**-1.5),
    Gamma = 5/3, copy boundaries in x and a 2*nm1+1 slab with copy
    boundaries in y and z.  (With periodic y and z the reference's
    single-rank periodic fill never refreshes the cells that are ghosts in
    both, bnd.f90:50-70/160-180/272-292, and flux-CT reads them.)"""
    _, nm1 = ghost_widths(irec, ict)
    imax = int(n) + 2 * nm1
    w = 2 * nm1 + 1
    dx = 1.0 / (imax - 1)
    return dict(
        imax=imax, jmax=w, kmax=w, metric=1, ix1=1, ix2=1, ix3=1, irec=irec, model=2, iter=5000,
        xmin=1.0, xmax=2.0, ymin=0.0, ymax=(w - 1) * dx, zmin=0.0, zmax=(w - 1) * dx,
        R0=0.0, hslope=0.5, akm=0.0, gam=5.0 / 3.0, cfl=cfl, dmin=1.0e-4, pmin=1.0e-6, pmax=1.0e6,
        tmax=tmax, dtmin=1.0e-9,
        ibc=[[5] * 9] * 6, precision=precision, ict=ict,
    )


def interior_cells(p: dict) -> int:
    """Zone count of one full step: interior cells (main.f90 loops nm1+1..n-nm1)."""
    _, nm1 = ghost_widths(p["irec"], p.get("ict", 1))
    return (p["imax"] - 2 * nm1) * (p["jmax"] - 2 * nm1) * (p["kmax"] - 2 * nm1)
