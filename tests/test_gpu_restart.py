"""GPU: restart files in the layout of store1 / restar2 (restar.f90:5-88,
273-346): gfortran sequential unformatted records, each framed by its 4-byte
length, (myrank, nd), (it0, ih0), (time), then per cell in (k, j, i) order the
records uu, u0, uri, uri0 of nine doubles.  The file is parsed here
independently of the library."""
import struct

import numpy as np
import pytest

from conftest import field_err
from oracle import Oracle
from raishinsource_b200 import config

pytestmark = pytest.mark.gpu


def read_records(path):
    recs = []
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (n,) = struct.unpack_from("<i", data, off)
        body = data[off + 4: off + 4 + n]
        (m,) = struct.unpack_from("<i", data, off + 4 + n)
        assert m == n
        recs.append(body)
        off += n + 8
    return recs


def test_store_layout_and_restore(gpu_ctx, tmp_path):
    p = dict(config.torus(nr=40, nth=32, nph=12), guard=1)
    o = Oracle(p)
    o.ic_torus(seed=17)
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    ic = o.prims()
    st = r.step(3, stats=True)
    cur = r.prims()
    path = str(tmp_path / "restart000.outdat")
    r.store(path, it0=3, ih0=1, nd=7, uri0=ic)
    recs = read_records(path)
    ncell = p["imax"] * p["jmax"] * p["kmax"]
    assert len(recs) == 3 + 4 * ncell
    assert struct.unpack("<ii", recs[0]) == (0, 7)
    assert struct.unpack("<ii", recs[1]) == (3, 1)
    assert struct.unpack("<d", recs[2])[0] == st["time"]
    body = np.frombuffer(b"".join(recs[3:]), dtype="<f8").reshape(ncell, 4, 9)
    uri = body[:, 2].reshape(cur.shape)
    assert np.array_equal(uri, cur)
    assert np.array_equal(body[:, 3].reshape(ic.shape), ic)
    # uu and u0 are caluu1 of uri and uri0
    assert field_err(body[:, 0].reshape(cur.shape), o.caluu1(cur)).max() < 1e-12
    assert field_err(body[:, 1].reshape(ic.shape), o.caluu1(ic)).max() < 1e-12
    # restart into a fresh run: same state and time; stepping on matches the original run
    r2 = gpu_ctx.admit(p)
    info = r2.restore(path)
    assert (info["it0"], info["ih0"], info["nd"]) == (3, 1, 7)
    assert np.array_equal(info["uri0"], ic)
    assert np.array_equal(r2.prims(), cur)
    a = r.step(2, stats=True)
    b = r2.step(2, stats=True)
    assert a["time"] == b["time"]
    assert np.array_equal(r.prims(), r2.prims())
    r.release()
    r2.release()


@pytest.mark.parametrize("nph", [12, None])
def test_output1_snapshot_equals_oracle_file(gpu_ctx, tmp_path, nph):
    """rg_run_output formats output1's records on the device and writes them
    through pinned buffers: the file equals the oracle's restatement of
    output1 (restar.f90:91-185) byte for byte, for a 3D run and a 2D run whose
    phi slab is stored as one plane."""
    p = dict(config.torus(nr=40, nth=32, nph=nph), guard=1)
    o = Oracle(p)
    o.ic_torus(seed=23)
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    a, b = str(tmp_path / "dev.outdat"), str(tmp_path / "orc.outdat")
    r.output(a, myrank=0, npe=1)
    r.release()
    o.output1(b, myrank=0, npe=1)
    da, db = open(a, "rb").read(), open(b, "rb").read()
    assert len(da) == len(db) == 56 + p["imax"] * p["jmax"] * p["kmax"] * 112
    assert da == db
