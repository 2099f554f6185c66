"""Parcel and grid dumps in the reference's binary format (writebinary.F90) and
the restart reader (readfromfile_parcelsetup.F90).  Needs a CUDA device.

  * a parcel dump holds the header and the 17 properties exactly as the
    reference writes them, bit for bit;
  * a restart from it continues the run with the same bits as the run that
    wrote it (FP64);
  * a grid dump's freshly gridded fields, hgliq and b + 12.5 hgliq match the
    oracle to 1e-12, its u, v, w and vol match the oracle after a step;
  * restart files of several ranks append, keeping only this domain's parcels.
"""
import math
import os

import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


def _vortical(pm, n, seed=9, amp=1.0):
    ic = pm.thermal_parcels(n, n, n)
    rng = np.random.default_rng(seed)
    for q in "pqr":
        ic[q] = amp * np.sin(ic["x"] * rng.integers(1, 3)) * np.cos(ic["y"] + ic["z"] * rng.uniform(0.5, 2))
    return ic


def test_parcel_dump_format_and_restart(pm, tmp_path):
    n = 16
    ic = _vortical(pm, n)
    cap = 2 * len(ic["x"])
    a = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=cap)
    a.upload(**ic)
    a.step(2)
    path = os.fspath(tmp_path / "parcels_00000_00002.dat")
    a.write_parcels(path, time=0.02)
    d = pm.read_parcel_dump(path)
    assert d["time"] == 0.02 and d["n"] == a.n
    np.testing.assert_allclose(d["bounds"], [0, TWO_PI, 0, TWO_PI, 0, math.pi], rtol=1e-15)
    assert os.path.getsize(path) == 8 * 7 + 8 + 17 * 8 * a.n
    for q in pm.DUMP_PROPS:
        np.testing.assert_array_equal(d[q], a.get(q), err_msg=q)
    b = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=cap)
    assert b.read_parcels(path) == 0.02
    assert b.n == a.n
    for q in pm.DUMP_PROPS:
        np.testing.assert_array_equal(b.get(q), a.get(q), err_msg=q)
    a.step(1)
    b.step(1)
    assert b.n == a.n
    for q in ["x", "y", "z", "p", "q", "r", "vol", "tag"]:
        np.testing.assert_array_equal(b.get(q), a.get(q), err_msg=q)
    for gname in ["u", "v", "w"]:
        np.testing.assert_array_equal(b.grid(gname), a.grid(gname), err_msg=gname)


def test_grid_dump_vs_oracle(pm, tmp_path):
    from oracle import Oracle
    n = 16
    ic = _vortical(pm, n)
    k = len(ic["x"])
    rng = np.random.default_rng(4)
    ic["h"] = rng.uniform(0.0, 1.2, k)  # some parcels above saturation exp(-z): hgliq > 0
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * k)
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * k)
    g.upload(**ic)
    o.set_parcels(**ic)
    g.step(1)
    o.step()
    path = os.fspath(tmp_path / "grids_00000_00001.dat")
    g.write_grids(path, time=0.01)
    d = pm.read_grid_dump(path)
    assert d["sizes"] == (n, n, n + 1) and d["time"] == 0.01
    for gname in ["u", "v", "w", "vol"]:
        assert rel(d[gname], o.grid(gname)) < 1e-10, gname
    o.cache_weights()
    for q in ["p", "q", "r", "b"]:
        o.par2grid(q, q)
    o.par2grid("h", "hg")
    z = np.arange(n + 1)[:, None, None] * (math.pi / n)
    hgliq = np.maximum(0.0, o.grid("hg") - np.exp(-z))
    assert hgliq.max() > 0
    ref = {"p": o.grid("p"), "q": o.grid("q"), "r": o.grid("r"), "hg": o.grid("hg"), "hgliq": hgliq,
           "b": o.grid("b") + 12.5 * hgliq}
    for gname, v in ref.items():
        assert rel(d[gname], v) < 1e-12, gname
    # the model's own grids are left as the step made them
    assert rel(g.grid("u"), o.grid("u")) < 1e-10


def test_mixed_dump_round_trip(pm, tmp_path):
    n = 16
    ic = _vortical(pm, n)
    cap = 2 * len(ic["x"])
    a = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=cap, precision="mixed")
    a.upload(**ic)
    a.step(1)
    p1 = os.fspath(tmp_path / "m1.dat")
    p2 = os.fspath(tmp_path / "m2.dat")
    a.write_parcels(p1)
    b = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=cap, precision="mixed")
    b.read_parcels(p1)
    b.write_parcels(p2)
    with open(p1, "rb") as f1, open(p2, "rb") as f2:
        assert f1.read() == f2.read()  # FP32 values survive FP64 files exactly
    g1 = os.fspath(tmp_path / "g1.dat")
    a.write_grids(g1)
    d = pm.read_grid_dump(g1)
    assert rel(d["u"], a.grid("u")) == 0.0


def test_restart_appends_rank_files_and_keeps_the_domain(pm, tmp_path):
    n = 8
    rng = np.random.default_rng(1)

    def dump(path, m, xlo, xhi):
        x = rng.uniform(xlo, xhi, m)
        cols = {q: rng.standard_normal(m) for q in pm.DUMP_PROPS}
        cols["x"], cols["y"], cols["z"] = x, rng.uniform(0, TWO_PI, m), rng.uniform(0, math.pi, m)
        cols["vol"] = np.full(m, 0.01)
        cols["tag"] = np.arange(m, dtype=np.float64)
        with open(path, "wb") as f:
            np.array([0.5, 0, TWO_PI, 0, TWO_PI, 0, math.pi]).tofile(f)
            np.array([m], np.int64).tofile(f)
            for q in pm.DUMP_PROPS:
                cols[q].tofile(f)
        return cols
    p0, p1 = os.fspath(tmp_path / "parcels_00000_00007.dat"), os.fspath(tmp_path / "parcels_00001_00007.dat")
    c0 = dump(p0, 300, 0.0, math.pi)
    c1 = dump(p1, 200, math.pi, TWO_PI + 1.0)  # some beyond x = 2 pi: not this domain's
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=1000)
    g.read_parcels(p0)
    g.read_parcels(p1, append=True)
    inside = c1["x"] < TWO_PI
    assert g.n == 300 + int(inside.sum())
    for q in pm.DUMP_PROPS:
        np.testing.assert_array_equal(g.get(q), np.concatenate([c0[q], c1[q][inside]]), err_msg=q)
