"""Parity of the B200 library (through its C ABI) with the CPU oracle and the
golden fixtures.  Needs a CUDA device.

Bars:
  * integer / index work (binning, haloswap re-slot, split and mixing
    bookkeeping: counts, keep, slots, backfill order, tags): bit-exact;
  * FP64 work with the reference's operation order and no FMA (grid2par, RK4,
    diffx/diffy/filter, the compact z solves, new-parcel positions): bit-exact;
  * FP64 sums whose order differs (par2grid's deterministic tile reduction vs
    the oracle's serial loop, the FFT algorithm): relative error <= 1e-12;
  * pow (splitting) may differ in the last bit between CUDA and glibc: 1e-14.
"""
import math

import numpy as np
import pytest

from helpers import ALL, geom, lattice_parcels, load, rel, rel_l2

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


def _pair(pm, nx, ny, nz, lx, ly, lz, props, n, cap, dtm=0.01, counters=None):
    from oracle import Oracle
    g = pm.Context(nx, ny, nz, lx, ly, lz, dtm=dtm, dtmax=dtm, max_parcels=cap)
    o = Oracle(nx, ny, nz, lx, ly, lz, dtm=dtm, dtmax=dtm, max_parcels=cap)
    full = {q: np.zeros(cap) for q in ALL}
    for q, v in props.items():
        full[q][:len(v)] = v
    for q in ALL:
        g.set(q, full[q], cap)
    o.set_parcels(**full)
    g.set_count(n)
    o.set_count(n)
    if counters is not None:
        g.set_counters(counters)
        o.set_counters(counters)
    return g, o


def _from_fixture(pm, name, counters, **kw):
    d = load(name)
    nx, ny, nz, lx, ly, lz = geom(d)
    cap = int(d["cap"])
    g, o = _pair(pm, nx, ny, nz, lx, ly, lz, {q: d["in_" + q][:cap] for q in ALL}, int(d["n_in"]), cap,
                 counters=counters, **kw)
    return d, g, o, cap


# ---- golden fixtures ------------------------------------------------------------------
@pytest.mark.parametrize("case", ["mix_case", "mix_case_last_slot"])
def test_mixing_golden(pm, case):
    d, g, _, cap = _from_fixture(pm, case, [0, 0, 1, 0, 3])
    g.parcel_mixing()
    info = g.info()
    assert g.n == int(d["n_out"])
    assert info.n_removed == int(d["nremove"]) and info.n_added == int(d["nadd"])
    for q in ["tag", "x", "y", "z", "stretch"]:
        np.testing.assert_array_equal(g.get(q, cap), d["out_" + q][:cap], err_msg=q)
    for q in ["vol", "b", "h", "p", "q", "r"]:
        assert rel(g.get(q, cap), d["out_" + q][:cap]) < 1e-12, q


def test_haloswap_golden(pm):
    d, g, _, cap = _from_fixture(pm, "haloswap_case", None)
    g.parcel_haloswap()
    assert g.n == int(d["n_in"])
    assert g.info().n_migrated == int((d["index"] != 0).sum())
    for q in ALL:
        np.testing.assert_array_equal(g.get(q, cap), d["out_" + q][:cap], err_msg=q)


def test_splitting_golden(pm):
    d, g, _, cap = _from_fixture(pm, "split_case", [0, 0, 1, 3, 0], dtm=float(d_dt()))
    g.parcel_splitting()
    n = int(d["n_out"])
    assert g.n == n
    for q in ["tag", "p", "q", "r", "b", "h", "dpdt"]:
        np.testing.assert_array_equal(g.get(q, n), d["out_" + q][:n], err_msg=q)
    for q in ["x", "y", "z", "vol", "stretch"]:
        assert rel(g.get(q, n), d["out_" + q][:n]) < 1e-14, q


def d_dt():
    return float(load("split_case")["dt"])


def test_par2grid_golden(pm):
    d = load("par2grid_case")
    nx, ny, nz, lx, ly, lz = geom(d)
    n = int(d["n_in"])
    g = pm.Context(nx, ny, nz, lx, ly, lz, max_parcels=n)
    g.upload(**{q: d["in_" + q][:n] for q in ["x", "y", "z", "vol", "b"]})
    g.par2grid("b", "b")
    assert rel(g.grid("b"), d["grid"]) < 1e-12
    # deterministic: a second call gives identical bits
    first = g.grid("b")
    g.par2grid("b", "b")
    np.testing.assert_array_equal(g.grid("b"), first)


# ---- model-core routines against the oracle ------------------------------------------
def _reference_accepts(x, n_cells, length):
    """parcel_interpolation.F90:214-237 for one coordinate (halo origin -2d)."""
    d = length / n_cells
    f = np.floor((x + 2 * d) / d)
    dl = ((x + 2 * d) - f * d) / d
    return (f >= 2) & (f <= n_cells + 2) & (dl >= 0) & (dl <= 1)


def test_binning_bit_exact(pm):
    from oracle import Oracle
    nx, ny, nz = 64, 48, 16
    rng = np.random.default_rng(7)
    n = 200000
    L = (1.0, TWO_PI, 0.5)  # with Lx = 1 the last ulp below Lx has delx = 0 exactly
    x = rng.uniform(0, L[0], n)
    y = rng.uniform(0, L[1], n)
    z = rng.uniform(0, L[2], n)
    # positions on cell faces and one ulp either side (those the reference's
    # own arithmetic accepts), and the last ulp below Lx, which bins into the
    # halo cell i = nx+3 with delx = 0 (parcel_interpolation.F90:214-216),
    # whose weight the reference folds onto x = 0
    m = n // 4
    k = rng.integers(0, nx, m)
    face = k * (L[0] / nx)
    u = rng.integers(0, 3, m)
    cand = np.where(u == 0, face, np.where(u == 1, np.nextafter(face, np.inf), np.nextafter(face, -np.inf)))
    cand = np.clip(cand, 0, None)
    x[:m] = np.where(_reference_accepts(cand, nx, L[0]), cand, x[:m])
    ky = rng.integers(0, ny, m)
    fy = ky * (L[1] / ny)
    cy = np.clip(np.where(u == 0, fy, np.where(u == 1, np.nextafter(fy, np.inf), np.nextafter(fy, -np.inf))), 0, None)
    ok_y = _reference_accepts(cy, ny, L[1])
    assert 0.5 < ok_y.mean() < 1.0  # some face positions are rejected by the reference itself
    y[:m] = np.where(ok_y, cy, y[:m])
    x[m:m + 10] = np.nextafter(L[0], 0)
    assert np.floor((x[m] + 2 * L[0] / nx) / (L[0] / nx)) == nx + 2
    g = pm.Context(nx, ny, nz, *L, max_parcels=n)
    o = Oracle(nx, ny, nz, *L, max_parcels=n)
    P = {"x": x, "y": y, "z": z, "vol": np.ones(n)}
    g.upload(**P)
    o.set_parcels(**P)
    cells = g.cell_ids()
    np.testing.assert_array_equal(cells, o.cache_weights())
    assert np.all(cells[m:m + 10] % nx == 0)


def test_binning_rejects_what_the_reference_rejects(pm):
    """One ulp below the face x = 31 dx, (x - xmin)/dx rounds up to the face
    while delx = -4.5e-15: the reference stops ("delx wrong size",
    parcel_interpolation.F90:235); both implementations report out-of-box.
    (Exact cell faces hit this too for a few percent of the faces, so a
    simulation aborts only for parcels within an ulp or two of a face.)"""
    from oracle import Oracle
    nx = 32
    x = np.array([1.0, np.nextafter(31 * (TWO_PI / nx), -np.inf)])
    P = {"x": x, "y": np.ones(2), "z": np.ones(2), "vol": np.ones(2)}
    g = pm.Context(nx, nx, 16, TWO_PI, TWO_PI, math.pi, max_parcels=4)
    o = Oracle(nx, nx, 16, TWO_PI, TWO_PI, math.pi, max_parcels=4)
    g.upload(**P)
    o.set_parcels(**P)
    with pytest.raises(pm.PmpicError) as e:
        g.cell_ids()
    assert e.value.code == -3
    with pytest.raises(Exception, match="delx"):
        o.cache_weights()


def test_grid2par_bit_exact(pm):
    from oracle import Oracle
    nx, ny, nz = 32, 32, 24
    ic = pm.thermal_parcels(nx, ny, nz)
    n = len(ic["x"])
    g = pm.Context(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=n)
    o = Oracle(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=n)
    g.upload(**ic)
    o.set_parcels(**ic)
    f = np.random.default_rng(3).standard_normal((nz + 1, ny, nx))
    g.set_grid("u", f)
    o.set_grid("u", f)
    o.cache_weights()
    g.grid2par("u", "dxdt")
    o.grid2par("u", "dxdt")
    np.testing.assert_array_equal(g.get("dxdt"), o.get("dxdt"))


def test_par2grid_vs_oracle(pm):
    from oracle import Oracle
    nx, ny, nz = 48, 32, 20
    ic = pm.thermal_parcels(nx, ny, nz)
    n = len(ic["x"])
    g = pm.Context(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=n)
    o = Oracle(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=n, threads=1)
    g.upload(**ic)
    o.set_parcels(**ic)
    o.cache_weights()
    for prop in ["b", "h"]:
        g.par2grid(prop, "b")
        o.par2grid(prop, "b")
        assert rel(g.grid("b"), o.grid("b")) < 1e-12


# four-step register path for rows of 16..256 (x: 32, 64, 128, 256, 16; y with
# nx % 16 == 0: 64, 16, 256, 128), generic Stockham for the others (y 48, x 40, y 24)
@pytest.mark.parametrize("shape", [(32, 48, 16), (40, 24, 8), (64, 64, 32), (128, 16, 4), (16, 128, 4),
                                   (256, 256, 3)])
def test_fft_vs_oracle(pm, shape):
    from oracle import Oracle
    nx, ny, nz = shape
    g = pm.Context(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=8)
    o = Oracle(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=8)
    rng = np.random.default_rng(4)
    f = rng.standard_normal((nz + 1, ny, nx))
    sg, so = g.fft_forward(f), o.fft_forward(f)
    assert rel(sg, so) < 1e-13
    s = rng.standard_normal((nz + 1, ny + 2, nx + 2))
    assert rel(g.fft_backward(s), o.fft_backward(s)) < 1e-13


def test_spectral_operators_bit_exact(pm):
    from oracle import Oracle
    nx, ny, nz = 32, 24, 20
    g = pm.Context(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=8)
    o = Oracle(nx, ny, nz, TWO_PI, TWO_PI, math.pi, max_parcels=8)
    rng = np.random.default_rng(5)
    s = rng.standard_normal((nz + 1, ny + 2, nx + 2))
    for op in ["diffx", "diffy", "filter", "diffz"]:
        np.testing.assert_array_equal(getattr(g, op)(s), getattr(o, op)(s), err_msg=op)
    bot, top = rng.standard_normal((2, ny + 2, nx + 2))
    np.testing.assert_array_equal(g.diffz(s, bot, top), o.diffz(s, bot, top))
    for df0 in (False, True):
        np.testing.assert_array_equal(g.laplinv(s, df0), o.laplinv(s, df0))


def test_linear_fields_known_answer(pm):
    """grid2partest.F90:119-265 (64^3, L=6000, 2^3 ppc) on the GPU."""
    nx = ny = nz = 64
    L = 6000.0
    P = lattice_parcels(nx, ny, nz, L, L, L)
    n = len(P["x"])
    P.update(p=P["x"].copy(), q=P["y"].copy(), r=P["z"].copy())
    g = pm.Context(nx, ny, nz, L, L, L, max_parcels=n)
    g.upload(**P)
    dx, dz = L / nx, L / nz
    xg = np.arange(nx) * dx
    zg = np.arange(nz + 1) * dz
    u = np.ascontiguousarray(np.broadcast_to(xg[None, None, :], (nz + 1, ny, nx)))
    w = np.ascontiguousarray(np.broadcast_to(zg[:, None, None], (nz + 1, ny, nx)))
    g.set_grid("u", u)
    g.set_grid("w", w)
    x, y = P["x"], P["y"]
    inner = (x > dx) & (x < L - 2 * dx) & (y > dx) & (y < L - 2 * dx)
    g.grid2par("u", "dxdt")
    assert np.abs(g.get("dxdt") - x)[inner].max() < 1e-9
    g.grid2par("w", "dzdt")
    assert np.abs(g.get("dzdt") - P["z"])[inner].max() < 1e-9
    g.par2grid("p", "p")
    sl = (slice(1, nz), slice(1, ny - 1), slice(1, nx - 1))
    assert np.abs(g.grid("p")[sl] - u[sl]).max() < 1e-9
    g.par2grid("r", "r")
    assert np.abs(g.grid("r")[sl] - w[sl]).max() < 1e-9


# ---- components -------------------------------------------------------------------------
def _vortical_ic(pm, n, seed=9, amp=1.0):
    ic = pm.thermal_parcels(n, n, n)
    rng = np.random.default_rng(seed)
    k = len(ic["x"])
    for q in "pqr":
        ic[q] = amp * np.sin(ic["x"] * rng.integers(1, 3)) * np.cos(ic["y"] + ic["z"] * rng.uniform(0.5, 2))
    return ic


def test_vort2vel_and_tendency_vs_oracle(pm):
    n = 32
    ic = _vortical_ic(pm, n)
    cap = 2 * len(ic["x"])
    g, o = _pair(pm, n, n, n, TWO_PI, TWO_PI, math.pi, ic, len(ic["x"]), cap)
    g.vort2vel()
    o.vort2vel()
    for name in ["p", "q", "r", "u", "v", "w"]:
        assert rel(g.grid(name), o.grid(name)) < 1e-12, name
    for name in ["u_s", "v_s", "w_s"]:
        assert rel(g.spec(name), o.spec(name)) < 1e-12, name
    for q in ["dxdt", "dydt", "dzdt"]:
        assert rel(g.get(q), o.get(q)) < 1e-12, q
    assert g.info().dtm == o.info().dtm
    g.vorticity_tendency()
    o.vorticity_tendency()
    for name in ["b", "dp", "dq", "dr"]:
        assert rel(g.grid(name), o.grid(name)) < 1e-11, name
    for q in ["btot", "dpdt", "dqdt", "drdt"]:
        assert rel(g.get(q), o.get(q)) < 1e-11, q


def test_rk4_stages_bit_exact(pm):
    """Four RK4 stages with identical tendencies, each followed by the parcel
    haloswap; parcels are pushed across the periodic faces and the walls."""
    nx = ny = nz = 16
    rng = np.random.default_rng(21)
    ic = pm.thermal_parcels(nx, ny, nz)
    n = len(ic["x"])
    props = dict(ic)
    for q in ["dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt"]:
        props[q] = rng.standard_normal(n) * 8.0
    g, o = _pair(pm, nx, ny, nz, TWO_PI, TWO_PI, math.pi, props, n, 2 * n, dtm=0.05)
    migrated = 0
    for stage in range(4):
        g.rk4_integrator()
        o.rk4_integrator()
        assert g.info().n_migrated == o.info().n_migrated
        migrated += o.info().n_migrated
        for q in ALL:
            np.testing.assert_array_equal(g.get(q), o.get(q), err_msg=f"{q} stage {stage + 1}")
    assert migrated > 0


def test_config0_twenty_steps(pm):
    """Config 0: 32^3 plume, dt = 0.01, 20 steps; gridded velocity within
    relative L2 1e-10 of the oracle, identical parcel counts and dt."""
    from oracle import Oracle
    n = 32
    ic = pm.thermal_parcels(n, n, n)
    cap = 2 * len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=cap)
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=cap)
    g.upload(**ic)
    o.set_parcels(**ic)
    for _ in range(20):
        g.step(1)
        o.step()
        assert g.n == o.n
        assert g.info().dtm == o.info().dtm
    for name in ["u", "v", "w"]:
        assert rel_l2(g.grid(name), o.grid(name)) < 1e-10, name
    for q in ["x", "y", "z", "p", "q", "r", "b", "h", "vol"]:
        assert rel(g.get(q), o.get(q)) < 1e-9, q


def test_split_and_mix_steps_vs_oracle(pm):
    """Steps with splitting and mixing active from the first step: stretch
    just below 4 with vorticity, and a tenth of the parcels below vmin."""
    from oracle import Oracle
    n = 16
    ic = _vortical_ic(pm, n, amp=3.0)
    k = len(ic["x"])
    rng = np.random.default_rng(33)
    ic["stretch"] = rng.uniform(3.9, 4.0, k)
    vmin = (TWO_PI / n) ** 2 * (math.pi / n) / 216
    ic["vol"][rng.uniform(size=k) < 0.1] = 0.5 * vmin
    cap = 4 * k
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.02, dtmax=0.02, max_parcels=cap)
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.02, dtmax=0.02, max_parcels=cap)
    g.upload(**ic)
    o.set_parcels(**ic)
    g.step(1)
    o.step()
    ig, io = g.info(), o.info()
    assert io.n_split > 0 and io.n_removed > 0 and io.n_added >= 0
    assert (ig.n_split, ig.n_removed, ig.n_added) == (io.n_split, io.n_removed, io.n_added)
    assert g.n == o.n
    np.testing.assert_array_equal(g.get("tag"), o.get("tag"))
    for q in ["x", "y", "z", "vol", "b", "h", "p", "q", "r"]:
        assert rel(g.get(q), o.get(q)) < 1e-10, q
    for name in ["u", "v", "w"]:
        assert rel_l2(g.grid(name), o.grid(name)) < 1e-10, name


def test_mixing_far_from_events_bit_exact(pm):
    """Mixing with parcels removed in one corner region and cells emptied in
    another: a kept parcel more than one cell from every removed or new
    parcel's cell sees +0.0 residuals at its corners, so the reference's
    redistribution gives it (f v + 0) / v and leaves its volume.  The FP64 path
    computes that without reading the grids: those parcels equal the oracle's
    bit for bit (and the formula, evaluated by numpy); the others agree with
    the oracle to 1e-12 (its grids sum in another order)."""
    from oracle import Oracle
    n = 16
    ic = _vortical_ic(pm, n)
    dx, dz = TWO_PI / n, math.pi / n
    vmin = dx * dx * dz / 216
    ci = np.floor(ic["x"] / dx).astype(int) % n
    cj = np.floor(ic["y"] / dx).astype(int) % n
    ck = np.minimum(np.floor(ic["z"] / dz).astype(int), n - 1)
    region = (ci < 2) & (cj < 2) & (ck < 2)
    ic["vol"][np.nonzero(region)[0][::3]] = 0.5 * vmin
    keep = ~((ci == 8) & (cj == 9) & (ck == 10))  # an emptied cell: a new parcel there
    ic = {q: v[keep] for q, v in ic.items()}
    ci, cj, ck = ci[keep], cj[keep], ck[keep]
    k = len(ic["x"])
    ic["tag"] = np.arange(k, dtype=np.float64) + 1000.0
    before = {q: ic[q].copy() for q in ["x", "y", "z", "b", "h", "p", "q", "r", "vol"]}
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k)
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k)
    g.upload(**ic)
    o.set_parcels(**ic)
    g.set_counters([3, 3, 4, 3, 3])
    o.set_counters([3, 3, 4, 3, 3])
    g.parcel_mixing()
    o.parcel_mixing()
    ig, io = g.info(), o.info()
    assert ig.n_removed == io.n_removed > 0 and ig.n_added == io.n_added > 0 and g.n == o.n
    np.testing.assert_array_equal(g.get("tag"), o.get("tag"))
    for q in ["b", "h", "p", "q", "r", "vol"]:
        assert rel(g.get(q), o.get(q)) < 1e-12, q

    def dist(a, c):  # periodic distance in cells
        return np.minimum((a - c) % n, (c - a) % n)
    near_new = (dist(ci, 8) <= 1) & (dist(cj, 9) <= 1) & (np.abs(ck - 10) <= 1)
    near_rem = (np.minimum(dist(ci, 0), dist(ci, 1)) <= 1) & (np.minimum(dist(cj, 0), dist(cj, 1)) <= 1) & (ck <= 2)
    far = np.nonzero(~near_new & ~near_rem)[0]  # original indices
    assert len(far) > k // 2
    # their final slots, by tag (a new parcel keeps its slot's old tag; no far
    # parcel's slot takes one), checked by the unchanged position
    tags = g.get("tag")
    order = np.argsort(tags, kind="stable")
    pos = np.searchsorted(tags[order], ic["tag"][far])
    slot = order[pos]
    assert np.all(tags[slot] == ic["tag"][far])
    for q in ["x", "y", "z"]:
        np.testing.assert_array_equal(g.get(q)[slot], before[q][far], err_msg=q)
    for q in ["b", "h", "p", "q", "r", "vol"]:
        a, b = g.get(q)[slot], o.get(q)[slot]
        np.testing.assert_array_equal(a, b, err_msg=q)
        want = before[q][far] if q == "vol" else (before[q][far] * before["vol"][far] + 0.0) / before["vol"][far]
        np.testing.assert_array_equal(a, want, err_msg=q)


def test_mixing_new_parcels_without_removals(pm):
    """Cells emptied of parcels (inside, at both walls, across the periodic
    corner) and no parcel below vmin: mixing adds a parcel in each.  Without a
    removed parcel the kept volume grid is made in full and the kept b, h, p,
    q, r sums only at the corners of the new parcels' cells, from those cells'
    parcels directly.  Counts, slots and tags equal the oracle's; parcels, the
    volume grid and the kept sums at those corners agree to 1e-12 (the sums run
    in another order); parcels away from the new cells equal it bit for bit."""
    from oracle import Oracle
    n = 16
    ic = _vortical_ic(pm, n)
    dx, dz = TWO_PI / n, math.pi / n
    ci = np.floor(ic["x"] / dx).astype(int) % n
    cj = np.floor(ic["y"] / dx).astype(int) % n
    ck = np.minimum(np.floor(ic["z"] / dz).astype(int), n - 1)
    emptied = [(5, 5, 5), (5, 6, 5), (10, 3, 0), (12, 12, n - 1), (0, 0, 8), (n - 1, n - 1, 8)]
    drop = np.zeros(len(ic["x"]), bool)
    for c in emptied:
        drop |= (ci == c[0]) & (cj == c[1]) & (ck == c[2])
    ic = {q: v[~drop] for q, v in ic.items()}
    k = len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k)
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k)
    g.upload(**ic)
    o.set_parcels(**ic)
    g.set_counters([3, 3, 4, 3, 3])
    o.set_counters([3, 3, 4, 3, 3])
    g.parcel_mixing()
    o.parcel_mixing()
    ig, io = g.info(), o.info()
    assert ig.n_removed == io.n_removed == 0
    assert ig.n_added == io.n_added >= len(emptied) and g.n == o.n
    np.testing.assert_array_equal(g.get("tag"), o.get("tag"))
    for q in ["x", "y", "z"]:
        np.testing.assert_array_equal(g.get(q), o.get(q), err_msg=q)
    for q in ["b", "h", "p", "q", "r", "vol"]:
        assert rel(g.get(q), o.get(q)) < 1e-12, q
    assert rel(g.grid("vol"), o.grid("vol")) < 1e-12
    pts = {(c[2] + a, (c[1] + b) % n, (c[0] + d) % n) for c in emptied for a in (0, 1) for b in (0, 1) for d in (0, 1)}
    idx = tuple(np.array(sorted(pts)).T)
    for name in ["b", "hg", "p", "q", "r"]:
        a, b = g.grid(name)[idx], o.grid(name)[idx]
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), name
    # parcels of the original slots more than one cell from every emptied cell
    def dist(a, c):
        return np.minimum((a - c) % n, (c - a) % n)
    ci, cj, ck = ci[~drop], cj[~drop], ck[~drop]
    far = np.ones(k, bool)
    for c in emptied:
        far &= ~((dist(ci, c[0]) <= 1) & (dist(cj, c[1]) <= 1) & (np.abs(ck - c[2]) <= 1))
    assert far.sum() > k // 2
    for q in ["b", "h", "p", "q", "r", "vol"]:
        np.testing.assert_array_equal(g.get(q)[:k][far], o.get(q)[:k][far], err_msg=q)


def test_deterministic_steps(pm):
    """No floating-point atomics: two runs give identical bits."""
    n = 32
    ic = _vortical_ic(pm, n)
    res = []
    for _ in range(2):
        g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * len(ic["x"]))
        g.upload(**ic)
        g.step(2)
        res.append({q: g.get(q) for q in ["x", "y", "z", "p", "q", "r"]} | {"u": g.grid("u")})
        g.close()
    for q in res[0]:
        np.testing.assert_array_equal(res[0][q], res[1][q], err_msg=q)


# ---- errors come back as codes, the context stays usable -------------------------------
def test_capacity_error_is_reported(pm):
    n = 8
    ic = _vortical_ic(pm, n, amp=3.0)
    k = len(ic["x"])
    ic["stretch"] = np.full(k, 3.999)
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.02, dtmax=0.02, max_parcels=k + 10)
    g.upload(**ic)
    with pytest.raises(pm.PmpicError) as e:
        g.step(1)
    assert e.value.code == -2  # PMPIC_ERR_CAPACITY
    assert g.n == k  # state not advanced past the failure point
    g.upload(**ic)   # and the context is still usable


def test_out_of_box_error_is_reported(pm):
    g = pm.Context(8, 8, 8, 1.0, 1.0, 1.0, max_parcels=16)
    g.upload(x=np.array([0.5, 0.5]), y=np.array([0.5, 0.5]), z=np.array([0.5, 3.0]), vol=np.ones(2))
    with pytest.raises(pm.PmpicError) as e:
        g.par2grid("b", "b")
    assert e.value.code == -3  # PMPIC_ERR_OUT_OF_BOX
    g.upload(x=np.array([0.5]), y=np.array([0.5]), z=np.array([0.5]), vol=np.ones(1))


# ---- full size (256^3): size-independent properties ------------------------------------
def test_full_size_step_properties(pm):
    """The 256^3 plume (134M parcels): one step conserves the parcel count
    through migration, the FFT round trip holds, par2grid of a constant is the
    constant, and no device error is raised."""
    n = 256
    ic = pm.thermal_parcels(n, n, n)
    k = len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.0025, dtmax=0.0025, max_parcels=int(1.1 * k))
    g.upload(**ic)
    ones = np.ones(k)
    g.set("btot", ones)
    g.par2grid("btot", "b")
    assert np.abs(g.grid("b") - 1.0).max() < 1e-13
    rng = np.random.default_rng(1)
    f = rng.standard_normal((n + 1, n, n))
    assert np.abs(g.fft_backward(g.fft_forward(f)) - f).max() < 1e-12
    del f
    vol0 = g.get("vol").sum()
    g.step(1)
    info = g.info()
    assert info.error == 0
    assert g.n == k + info.n_split + info.n_added - info.n_removed
    assert abs(g.get("vol").sum() - vol0) / vol0 < 1e-12
    np.testing.assert_array_equal(np.sort(g.get("tag")), np.arange(k, dtype=float))
