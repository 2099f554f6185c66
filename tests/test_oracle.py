"""The oracle pinned against the reference's known-answer tests and the golden
fixtures (CPU only).

Known answers re-implemented from the reference:
  * components/grid2partest (grid2partest.F90:119-265, grid2par.mcf): linear
    fields u=x, v=y, w=z recovered by grid2par at the parcels and by par2grid
    at the grid points within 1e-9, away from the periodic edges;
  * components/laplinv_test (laplinv.F90:93-198): analytic potentials for the
    compact Laplacian inversion (both boundary conditions);
  * the report's mixing conservation test (report.tex:264, parcel_mixing.F90:
    87-103, 412-422): total volume and volume-integrated humidity conserved;
  * the report's splitting geometry (report.tex:250).
Golden fixtures (tests/golden, from make_golden.py's independent restatement):
mixing, parcel haloswap, splitting and par2grid, compared bit for bit.
"""
import math

import numpy as np
import pytest

from helpers import ALL, geom, lattice_parcels, load, rel
from oracle import Oracle


def _oracle_from(d, cap=None, threads=1, **kw):
    nx, ny, nz, lx, ly, lz = geom(d)
    cap = int(d["cap"]) if cap is None else cap
    o = Oracle(nx, ny, nz, lx, ly, lz, max_parcels=cap, threads=threads, **kw)
    n = int(d["n_in"])
    full = {q: d["in_" + q] for q in ALL}
    o.set_parcels(**{q: v[:cap] for q, v in full.items()})
    o.set_count(n)
    return o


# ---- golden fixtures (bit-exact) ---------------------------------------------------
@pytest.mark.parametrize("case", ["mix_case", "mix_case_last_slot"])
def test_mixing_matches_golden(case):
    d = load(case)
    o = _oracle_from(d)
    o.set_counters([0, 0, 1, 0, 3])  # mixing runs on the 4th RK substep
    o.parcel_mixing()
    info = o.info()
    assert o.n == int(d["n_out"])
    assert info.n_removed == int(d["nremove"])
    assert info.n_added == int(d["nadd"])
    cap = int(d["cap"])
    for q in ALL:
        np.testing.assert_array_equal(o.get(q, cap), d["out_" + q][:cap], err_msg=q)


def test_mixing_last_slot_quirk():
    """`keep(n)=2` only for n < numparcels_local: a new parcel in the last slot
    keeps keep = 0 and is overwritten by the backfill (parcel_mixing.F90:191-193,
    347-389)."""
    d = load("mix_case_last_slot")
    n = int(d["n_in"])
    assert list(d["new_slots"]) == [n - 2, n - 1]
    assert int(d["n_out"]) == n - 1
    assert d["keep"][n - 2] == 2 and d["keep"][n - 1] == 0


def test_haloswap_matches_golden():
    d = load("haloswap_case")
    o = _oracle_from(d)
    o.parcel_haloswap()
    assert o.n == int(d["n_in"])
    assert set(np.unique(d["index"])) == set(range(9))  # every direction occurs
    cap = int(d["cap"])
    for q in ALL:
        np.testing.assert_array_equal(o.get(q, cap), d["out_" + q][:cap], err_msg=q)


def test_splitting_matches_golden():
    d = load("split_case")
    o = _oracle_from(d, dtm=float(d["dt"]), dtmax=float(d["dt"]))
    o.set_counters([0, 0, 1, 3, 0])
    o.parcel_splitting()
    assert o.n == int(d["n_out"])
    n = o.n
    # splitting is followed by a parcel haloswap (parcel_splitting.F90:158),
    # which re-slots the children that left the box
    assert o.info().n_migrated > 0
    for q in ["x", "y", "z", "p", "q", "r", "vol", "stretch", "tag", "b", "h", "dpdt"]:
        np.testing.assert_array_equal(o.get(q, n), d["out_" + q][:n], err_msg=q)


def test_par2grid_matches_golden():
    d = load("par2grid_case")
    nx, ny, nz, lx, ly, lz = geom(d)
    n = int(d["n_in"])
    o = Oracle(nx, ny, nz, lx, ly, lz, max_parcels=n, threads=1)
    o.set_parcels(**{q: d["in_" + q][:n] for q in ["x", "y", "z", "vol", "b"]})
    o.cache_weights()
    o.par2grid("b", "b")
    np.testing.assert_array_equal(o.grid("b"), d["grid"])


# ---- known answers from the reference's own test components --------------------------
def test_grid2partest_linear_fields():
    """grid2partest.F90:119-265 with grid2par.mcf (64^3, L=6000, 2^3 ppc)."""
    nx = ny = nz = 64
    L = 6000.0
    P = lattice_parcels(nx, ny, nz, L, L, L)
    n = len(P["x"])
    o = Oracle(nx, ny, nz, L, L, L, max_parcels=n)
    P.update(p=P["x"].copy(), q=P["y"].copy(), r=P["z"].copy())
    o.set_parcels(**P)
    dx, dy, dz = L / nx, L / ny, L / nz
    xg = np.arange(nx) * dx
    yg = np.arange(ny) * dy
    zg = np.arange(nz + 1) * dz
    u = np.broadcast_to(xg[None, None, :], (nz + 1, ny, nx))
    v = np.broadcast_to(yg[None, :, None], (nz + 1, ny, nx))
    w = np.broadcast_to(zg[:, None, None], (nz + 1, ny, nx))
    o.set_grid("u", u); o.set_grid("v", v); o.set_grid("w", w)
    o.cache_weights()
    x, y = P["x"], P["y"]
    top_x, top_y = L - dx, L - dy
    inner = (x > dx) & (x < top_x - dx) & (y > dy) & (y < top_y - dy)
    for gname, prop, ref in [("u", "dxdt", x), ("v", "dydt", y), ("w", "dzdt", P["z"])]:
        o.grid2par(gname, prop)
        got = o.get(prop)
        assert np.abs(got - ref)[inner].max() < 1e-9, gname
    # par2grid of p=x, q=y, r=z recovers the grid coordinates (check_grid)
    for prop, gname, ref in [("p", "p", u), ("q", "q", v), ("r", "r", w)]:
        o.par2grid(prop, gname)
        g = o.grid(gname)
        sl = (slice(1, nz), slice(1, ny - 1), slice(1, nx - 1))
        assert np.abs(g[sl] - ref[sl]).max() < 1e-9, gname


def _laplinv_error(nz, df0):
    Lz = math.pi
    nx = ny = 8
    o = Oracle(nx, ny, nz, 2 * math.pi, 2 * math.pi, Lz, max_parcels=4)
    _, _, k2, _ = o.wavenumbers()
    z = np.arange(nz + 1) * (Lz / nz)
    jp, ip = 4, 2  # ky = 2, kx = 1, real-real entry
    if not df0:
        c = np.poly1d(np.poly([0.0, 0.2 * Lz, 0.7 * Lz, Lz]))       # A(0) = A(Lz) = 0
    else:
        c = np.poly1d(np.polymul(np.poly([0.0, 0.0]), np.poly([Lz, Lz])))  # C'(0) = C'(Lz) = 0
    A = c(z)
    B = c.deriv(2)(z) - k2[jp, ip] * A
    s = np.zeros((nz + 1, ny + 2, nx + 2))
    s[:, jp, ip] = B
    out = o.laplinv(s, df0)
    others = out.copy()
    others[:, jp, ip] = 0
    assert np.all(others == 0)
    return np.abs(out[:, jp, ip] - A).max() / np.abs(A).max()


def test_laplinv_dirichlet_known_answer():
    """Quartic potential with A = 0 at the walls: the compact scheme is exact for
    it up to the REAL(4) literals 1./12., 5./6. (fft_ops.F90:512-513), which
    leave an O(1e-8) consistency floor that does not shrink with resolution."""
    errs = [_laplinv_error(n, False) for n in (16, 32, 64)]
    assert max(errs) < 2e-8
    assert min(errs) > 1e-10  # the single-precision floor is really there


def test_laplinv_neumann_converges():
    """dA/dz = 0 at the walls: third-order convergence (boundary rows
    fft_ops.F90:578-587) until the single-precision floor."""
    e = [_laplinv_error(n, True) for n in (16, 32, 64)]
    orders = [math.log2(e[i] / e[i + 1]) for i in range(2)]
    assert all(2.8 < p < 3.2 for p in orders), orders


def test_diffz_known_answers():
    Lz = math.pi
    for nz, tol in [(32, 1e-6), (64, 1e-7)]:
        o = Oracle(8, 8, nz, 2 * math.pi, 2 * math.pi, Lz, max_parcels=4)
        z = np.arange(nz + 1) * (Lz / nz)
        s = np.zeros((nz + 1, 10, 10))
        s[:, 3, 5] = np.cos(math.pi * z / Lz)
        d = o.diffz(s)
        exact = -(math.pi / Lz) * np.sin(math.pi * z / Lz)
        assert rel(d[:, 3, 5], exact) < tol
    # with wall values the reference's rows 1 and n are b=1, c=1/3 (fft_ops.F90
    # :442-455), not the 2/3 of its comment (:414-417): the wall rows are
    # inconsistent, so only the interior converges
    for nz in (64, 128):
        o = Oracle(8, 8, nz, 2 * math.pi, 2 * math.pi, Lz, max_parcels=4)
        z = np.arange(nz + 1) * (Lz / nz)
        c = np.poly1d(np.poly([0.0, 0.3 * Lz, Lz]))
        s = np.zeros((nz + 1, 10, 10))
        s[:, 3, 5] = c(z)
        bot = np.zeros((10, 10)); top = np.zeros((10, 10))
        bot[3, 5] = c.deriv(2)(0.0); top[3, 5] = c.deriv(2)(Lz)
        d = o.diffz(s, bot, top)[:, 3, 5]
        m = slice(nz // 4, 3 * nz // 4)
        ex = c.deriv()(z)
        assert np.abs(d[m] - ex[m]).max() / np.abs(ex).max() < 2e-8
        assert abs(d[0] - ex[0]) / abs(ex[0]) > 0.2  # the wall-row quirk does not converge


def test_mixing_conserves_volume_and_humidity():
    """report.tex:264: half of the parcels shrunk below vmin; global volume and
    volume-integrated humidity and buoyancy conserved to 1e-13."""
    import pmpic_b200 as pm
    N = 16
    ic = pm.thermal_parcels(N, N, N)
    n = len(ic["x"])
    rng = np.random.default_rng(5)
    vmin = (2 * math.pi / N) ** 2 * (math.pi / N) / 216
    ic["vol"][rng.uniform(size=n) < 0.5] = 0.5 * vmin
    o = Oracle(N, N, N, 2 * math.pi, 2 * math.pi, math.pi, max_parcels=2 * n)
    o.set_parcels(**ic)
    v0 = o.get("vol").sum()
    h0 = (o.get("h") * o.get("vol")).sum()
    b0 = (o.get("b") * o.get("vol")).sum()
    o.set_counters([0, 0, 1, 0, 3])
    o.parcel_mixing()
    assert o.info().n_removed > 0 and o.info().n_added > 0
    v1 = o.get("vol").sum()
    h1 = (o.get("h") * o.get("vol")).sum()
    b1 = (o.get("b") * o.get("vol")).sum()
    assert abs(v1 - v0) / v0 < 1e-13
    assert abs(h1 - h0) / abs(h0) < 1e-13
    assert abs(b1 - b0) / abs(b0) < 1e-13


def test_splitting_geometry():
    """report.tex:250: children at x +- (vol/4 pi)^(1/3) w/|w|, half volume,
    stretch reset, the child appended after the existing parcels in index
    order (parcel_splitting.F90:76-127)."""
    rng = np.random.default_rng(11)
    n0 = 200
    L = 2 * math.pi
    o = Oracle(16, 16, 16, L, L, math.pi, dtm=0.05, dtmax=0.05, max_parcels=2 * n0, threads=1)
    P = {"x": rng.uniform(1, L - 1, n0), "y": rng.uniform(1, L - 1, n0), "z": rng.uniform(1, 2, n0),
         "p": rng.standard_normal(n0), "q": rng.standard_normal(n0), "r": rng.standard_normal(n0),
         "dpdt": rng.standard_normal(n0), "dqdt": rng.standard_normal(n0), "drdt": rng.standard_normal(n0),
         "vol": rng.uniform(0.5, 1.5, n0) * 1e-3, "stretch": rng.uniform(3.0, 4.2, n0),
         "tag": np.arange(n0, dtype=float)}
    o.set_parcels(**P)
    o.set_counters([0, 0, 1, 3, 0])
    o.parcel_splitting()
    n1 = o.n
    assert o.info().n_migrated == 0
    x, y, z, vol, st, tag = (o.get(q) for q in ["x", "y", "z", "vol", "stretch", "tag"])
    split = np.where(vol[:n0] < P["vol"])[0]
    assert len(split) == n1 - n0 > 0
    child = np.arange(n0, n1)
    np.testing.assert_array_equal(tag[child], split.astype(float))  # index order
    w = np.stack([P["p"], P["q"], P["r"]])[:, split]
    w = w / np.sqrt((w ** 2).sum(0))
    r = (P["vol"][split] / 4 / math.pi) ** (1 / 3)
    for pos, k in [(x, 0), (y, 1), (z, 2)]:
        start = P["xyz"[k]][split]
        np.testing.assert_allclose(pos[child] - start, r * w[k], rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(start - pos[split], r * w[k], rtol=1e-6, atol=1e-12)
    np.testing.assert_array_equal(vol[child], P["vol"][split] / 2)
    np.testing.assert_array_equal(vol[split], P["vol"][split] / 2)
    assert np.all(st[child] == 0) and np.all(st[split] == 0)


def test_haloswap_conserves_count_and_wraps():
    d = load("haloswap_case")
    o = _oracle_from(d)
    nx, ny, nz, lx, ly, lz = geom(d)
    o.parcel_haloswap()
    x, y, z = o.get("x"), o.get("y"), o.get("z")
    assert o.n == int(d["n_in"])
    assert np.all((x >= 0) & (x < lx + 1e-9) & (y >= 0) & (y < ly + 1e-9))
    assert np.all((z >= 0) & (z <= lz))
    np.testing.assert_array_equal(np.sort(o.get("tag")), np.sort(d["in_tag"][:o.n]))


def test_oracle_rejects_out_of_box():
    o = Oracle(8, 8, 8, 1.0, 1.0, 1.0, max_parcels=4)
    o.set_parcels(x=np.array([0.5, 0.5]), y=np.array([0.5, 0.5]), z=np.array([0.5, 2.0]),
                  vol=np.ones(2))
    with pytest.raises(Exception, match="out of box"):
        o.cache_weights()


def test_conserved_sums_are_the_rounded_exact_totals():
    """The oracle's compensated totals of vol, h*vol and b*vol equal the FP64
    rounding of the exact totals (rational arithmetic), on values spread over
    many magnitudes and signs, where a plain running sum loses digits."""
    from fractions import Fraction
    rng = np.random.default_rng(11)
    n = 4000
    vol = rng.uniform(0.5, 1.5, n) * 10.0 ** rng.integers(-8, 3, n)
    h = rng.standard_normal(n) * 10.0 ** rng.integers(-6, 6, n)
    b = rng.standard_normal(n)
    o = Oracle(8, 8, 8, 1.0, 1.0, 1.0, max_parcels=n)
    o.set_parcels(x=np.full(n, 0.5), y=np.full(n, 0.5), z=np.full(n, 0.5), vol=vol, h=h, b=b)
    got = o.conserved_sums()
    exact = [sum(Fraction(v) for v in vol), sum(Fraction(v) * Fraction(w) for v, w in zip(vol, h)),
             sum(Fraction(v) * Fraction(w) for v, w in zip(vol, b))]
    for g, e in zip(got, exact):
        assert g == float(e), (g, float(e))
    o.close()
