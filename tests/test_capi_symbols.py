"""The C-ABI library builds, loads without a GPU and exports every entry point
that include/raishin_gpu.h declares (no compute calls)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "raishin_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(rg_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "rg_step" in syms and "rg_recov" in syms and "rg_calflx" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    """Both variants (product and uncontracted) export the whole ABI."""
    from raishinsource_b200 import build
    from raishinsource_b200.capi import EXPORTS
    syms = declared_symbols()
    assert sorted(EXPORTS) == syms
    for variant in build.VARIANTS:
        lib = ctypes.CDLL(build.build(variants=(variant,)))
        for s in syms:
            assert hasattr(lib, s), (variant, s)


def test_footprint_and_param_checks_run_on_cpu():
    from raishinsource_b200 import config, footprint
    from raishinsource_b200.capi import RgError
    p = config.torus(nr=256, nth=128, nph=128)
    b = footprint(p)
    assert 2e9 < b < 6e9
    for irec in (config.IREC_MC, config.IREC_MINMOD, config.IREC_MUSCL, config.IREC_WENOZ, config.IREC_LIMO3,
                 config.IREC_MVL, config.IREC_KOREN):
        assert footprint(dict(p, irec=irec)) > 0
    for irec in (config.IREC_CENO, config.IREC_MPWENO, config.IREC_WENOM):
        assert footprint(dict(p, irec=irec)) > 0
    for ict in (0, 2):
        assert footprint(dict(p, ict=ict)) > 0
    # upflct keeps six planes of EMF differences besides the step state
    n = config.torus(nr=256, nth=128, nph=128, ict=3)
    assert footprint(n) > footprint(dict(n, ict=2))
    # recov2 keeps 22 planes of stage scratch
    assert footprint(dict(p, iwvec=2)) > footprint(p)
    for bad_ct in (dict(n, precision="mixed"), dict(p, ict=4),  # upflct is FP64 only; no ict 4
                   dict(p, iwvec=2, precision="mixed"), dict(p, iwvec=3)):  # recov2 is FP64 only
        try:
            footprint(bad_ct)
        except RgError as e:
            assert e.code == 1
        else:
            raise AssertionError("must be rejected: %s" % bad_ct)
    bad = dict(p, irec=14)  # no such scheme
    try:
        footprint(bad)
    except RgError as e:
        assert e.code == 1
    else:
        raise AssertionError("irec=14 must be rejected")


def test_library_load_error_path_without_gpu():
    """rg_ctx_create returns an error status, never aborts, when no device exists."""
    from raishinsource_b200.capi import load
    lib = load()
    h = ctypes.c_void_p()
    rc = lib.rg_ctx_create(0, ctypes.byref(h))
    try:
        import torch
        gpu = torch.cuda.is_available()
    except Exception:
        gpu = False
    if gpu:
        assert rc == 0
        lib.rg_ctx_destroy(h)
    else:
        assert rc != 0
        assert lib.rg_last_error()
