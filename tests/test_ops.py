"""Kernel-level entry points against the oracle: multi-field par2grid and
grid2par (both precisions), vort2vel's inversion on given grids, and the
renumbering of parcel slots into cell order.  Needs a CUDA device.

Bars as in test_gpu_parity: grid2par bit-exact on the FP64 path, par2grid and
the transforms <= 1e-12 relative; the mixed form within FP32 rounding
(<= 1e-5 relative).
"""
import math

import numpy as np
import pytest

from helpers import rel, rel_l2

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


def _random_parcels(n, cells_per_dim, seed):
    rng = np.random.default_rng(seed)
    k = 8 * cells_per_dim ** 3
    x = rng.uniform(0, TWO_PI, k)
    y = rng.uniform(0, TWO_PI, k)
    z = rng.uniform(0, math.pi, k)
    vol = np.full(k, (TWO_PI / n) ** 2 * (math.pi / n) / 8)
    f = {q: np.sin(2 * x + q) * np.cos(y - 0.5 * q) * np.cos(3 * z) for q in range(4)}
    return {"x": x, "y": y, "z": z, "vol": vol, "p": f[0], "q": f[1], "r": f[2], "b": f[3],
            "tag": np.arange(k, dtype=np.float64)}


def test_par2grid_and_grid2par_multi_vs_oracle(pm):
    from oracle import Oracle
    n = 16
    ic = _random_parcels(n, n, 7)
    k = len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=k)
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=k)
    g.upload(**ic)
    o.set_parcels(**ic)
    o.cache_weights()  # the oracle's par2grid and grid2par use the cached binning
    g.par2grid_multi(["p", "q", "r", "b"], ["p", "q", "r", "b"])
    for q in ["p", "q", "r", "b"]:
        o.par2grid(q, q)
        assert rel(g.grid(q), o.grid(q)) < 1e-12, q
    rng = np.random.default_rng(3)
    names = ["u", "v", "w", "dp", "dq", "dr"]
    props = ["dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt"]
    for nm in names:
        gr = rng.standard_normal((n + 1, n, n))
        g.set_grid(nm, gr)
        o.set_grid(nm, gr)
    g.grid2par_multi(names, props)
    for nm, pr in zip(names, props):
        o.grid2par(nm, pr)
        np.testing.assert_array_equal(g.get(pr), o.get(pr), err_msg=pr)


def test_mixed_multi_ops_vs_fp64(pm):
    n = 16
    ic = _random_parcels(n, n, 8)
    k = len(ic["x"])
    a = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=k)
    b = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=k, precision="mixed")
    a.upload(**ic)
    b.upload(**ic)
    for c in (a, b):
        c.par2grid_multi(["p", "q", "r"], ["p", "q", "r"])
    for q in ["p", "q", "r"]:
        assert rel_l2(b.grid(q), a.grid(q)) < 1e-5, q
    rng = np.random.default_rng(4)
    names = ["u", "v", "w"]
    props = ["dxdt", "dydt", "dzdt"]
    for nm in names:
        gr = rng.standard_normal((n + 1, n, n))
        a.set_grid(nm, gr)
        b.set_grid(nm, gr)
    for c in (a, b):
        c.grid2par_multi(names, props)
    for pr in props:
        assert rel(b.get(pr), a.get(pr)) < 1e-5, pr


def test_vort2vel_grids_vs_oracle(pm):
    """The inversion alone on a divergence-free random vorticity with the wall
    conditions (the vort2vel-alone workload at 32^3)."""
    from oracle import Oracle
    n = 32
    p, q, r = pm.random_vorticity(n, n, n, kmax=12, seed=4)
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=16)
    m = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=16, precision="mixed")
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=16)
    for c in (g, m, o):
        c.set_grid("p", p)
        c.set_grid("q", q)
        c.set_grid("r", r)
    g.vort2vel_grids()
    m.vort2vel_grids()
    o.vort2vel_grids()
    for nm in ["u", "v", "w", "p", "q", "r"]:
        assert rel(g.grid(nm), o.grid(nm)) < 1e-12, nm
        assert rel_l2(m.grid(nm), o.grid(nm)) < 1e-5, nm
    for nm in ["u_s", "v_s", "w_s"]:
        assert rel(g.spec(nm), o.spec(nm)) < 1e-12, nm


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sort_parcels_keeps_the_parcel_set(pm, precision):
    n = 16
    ic = _random_parcels(n, n, 9)
    k = len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=k, precision=precision)
    g.upload(**ic)
    g.par2grid("p", "p") if precision == "fp64" else g.par2grid_multi(["p"], ["p"])
    before = g.grid("p")
    props = {q: g.get(q) for q in ["x", "y", "z", "p", "vol", "tag"]}
    g.sort_parcels()
    after = {q: g.get(q) for q in props}
    order = np.argsort(after["tag"])
    tags = after["tag"][order].astype(np.int64)
    np.testing.assert_array_equal(tags, np.arange(k))
    for q in props:  # the same parcels, permuted together
        np.testing.assert_array_equal(after[q][order], props[q][tags], err_msg=q)
    cells = g.cell_ids()  # x-fastest ids ((k*ny + j)*nx + i); slots now in z-fastest cell order
    ck, cj, ci = cells // (n * n), (cells // n) % n, cells % n
    zf = (ci * n + cj) * n + ck
    assert np.all(np.diff(zf) >= 0)
    g.par2grid("p", "p") if precision == "fp64" else g.par2grid_multi(["p"], ["p"])
    # slot order inside each cell is kept, so every sum runs in the same order
    np.testing.assert_array_equal(g.grid("p"), before)
