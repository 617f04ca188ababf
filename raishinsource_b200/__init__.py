"""B200-native RAISHIN GRMHD finite-volume update (Kerr metric) on sm_100a.

The package is the host-side mirror of the reference driver (main.f90) over the
C ABI of ``libraishin_gpu.so`` (include/raishin_gpu.h):

    from raishinsource_b200 import config, Context
    with Context(0) as ctx:
        run = ctx.admit(config.torus(nr=256, nth=128, nph=128))
        run.ic_torus(seed=2012)
        run.step(1000)
        uri = run.prims()          # a(nv,i,j,k) as (kmax, jmax, imax, 9)
"""
from . import config  # noqa: F401
from .capi import Context, Run, RgError, footprint, load  # noqa: F401

__all__ = ["config", "Context", "Run", "RgError", "footprint", "load"]
