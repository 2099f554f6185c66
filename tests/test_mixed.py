"""The mixed-precision form (PMPIC_MIXED) against the FP64 oracle and the
plain FP64 GPU path.  Needs a CUDA device.

The mixed form computes in FP32 (interpolation, transforms, tendencies, RK4),
keeps positions as an integer cell index plus an FP32 offset, and keeps the
zero mode (the mean flow of vort2vel.F90:230-241) in FP64.  Its results are
not bit-identical to FP64 and are measured by their error against the FP64 oracle:

  * gridded velocity u, v, w after the 20 steps of the 32^3 plume (dt 0.01):
    relative L2 error <= 1e-4;
  * split and mixing bookkeeping (counts, slots, tags) on inputs whose
    decisions lie far from the thresholds: identical to the oracle;
  * transfers: FP64 -> mixed -> FP64 within one FP32 rounding of the offset;
  * total parcel volume through a mixing step: conserved to FP32 rounding.
"""
import math

import numpy as np
import pytest

from helpers import rel, rel_l2

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi
TOL_VEL = 1e-4  # relative L2 of gridded velocity vs the FP64 oracle


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


def test_mixed_transfer_round_trip(pm):
    n = 16
    ic = _vortical(pm, n)
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * len(ic["x"]), precision="mixed")
    g.upload(**ic)
    dx, dz = TWO_PI / n, math.pi / n
    for q, d in [("x", dx), ("y", dx), ("z", dz)]:
        # the offset is an FP32 fraction of a cell: error below one FP32 ulp of 1 cell
        assert np.abs(g.get(q) - ic[q]).max() <= d * 2.0 ** -23, q
    for q in ["p", "q", "r", "b", "h", "vol"]:
        np.testing.assert_allclose(g.get(q), ic[q].astype(np.float32).astype(np.float64), rtol=0, atol=0)
    np.testing.assert_array_equal(g.get("tag"), ic["tag"])


def test_mixed_transfers_in_several_staged_chunks(pm):
    """Host transfers of the mixed form go through two device staging halves
    in chunks of half the staging size (the staging holds min(max_parcels,
    2^24) values), copied on a separate stream while the context's stream
    converts.  With max_parcels = n (odd) every property crosses three chunks
    and both halves: the round trip is what one chunk gives (positions within
    one FP32 rounding of the offset, fields rounded to FP32, tags exact), and a
    property set afterwards reads back as set."""
    rng = np.random.default_rng(17)
    n = 4097
    ic = {"x": rng.uniform(0, TWO_PI, n), "y": rng.uniform(0, TWO_PI, n), "z": rng.uniform(0, math.pi, n)}
    for q in ["p", "q", "r", "b", "h", "stretch"]:
        ic[q] = rng.standard_normal(n)
    ic["vol"] = rng.uniform(0.5, 1.5, n) * 1e-3
    ic["tag"] = np.arange(n, dtype=np.float64) * 3 + 1
    g = pm.Context(16, 16, 16, TWO_PI, TWO_PI, math.pi, max_parcels=n, precision="mixed")
    g.upload(**ic)
    dx, dz = TWO_PI / 16, math.pi / 16
    out = g.download()
    for q, d in [("x", dx), ("y", dx), ("z", dz)]:
        assert np.abs(out[q] - ic[q]).max() <= d * 2.0 ** -23, q
    for q in ["p", "q", "r", "b", "h", "vol", "stretch"]:
        np.testing.assert_array_equal(out[q], ic[q].astype(np.float32).astype(np.float64), err_msg=q)
    np.testing.assert_array_equal(out["tag"], ic["tag"])
    v = rng.standard_normal(n)
    g.set("p", v)
    np.testing.assert_array_equal(g.get("p"), v.astype(np.float32).astype(np.float64))


def test_mixed_config0_twenty_steps_vs_oracle(pm):
    """Config 0: 32^3 plume, dt = 0.01, 20 steps."""
    from oracle import Oracle
    n = 32
    ic = pm.thermal_parcels(n, n, n)
    cap = 2 * len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=cap, precision="mixed")
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=cap)
    g.upload(**ic)
    o.set_parcels(**ic)
    for _ in range(20):
        g.step(1)
        o.step()
    errs = {name: rel_l2(g.grid(name), o.grid(name)) for name in ["u", "v", "w"]}
    for name, e in errs.items():
        assert e < TOL_VEL, (name, e)


def test_mixed_split_and_mix_bookkeeping_vs_oracle(pm):
    """Splitting and mixing active in the first step, on inputs whose decisions
    lie far from the thresholds (stretch 3.5 or 4.5; volume 0.5 vmin or the
    lattice volume): counts and tags identical to the oracle."""
    from oracle import Oracle
    n = 16
    ic = _vortical(pm, n, amp=3.0)
    k = len(ic["x"])
    rng = np.random.default_rng(33)
    ic["stretch"] = np.where(rng.uniform(size=k) < 0.1, 4.5, 3.5)
    vmin = (TWO_PI / n) ** 2 * (math.pi / n) / 216
    ic["vol"][rng.uniform(size=k) < 0.1] = 0.5 * vmin
    cap = 4 * k
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.02, dtmax=0.02, max_parcels=cap, precision="mixed")
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.02, dtmax=0.02, max_parcels=cap)
    g.upload(**ic)
    o.set_parcels(**ic)
    g.step(1)
    o.step()
    ig, io = g.info(), o.info()
    assert io.n_split > 0 and io.n_removed > 0
    assert (ig.n_split, ig.n_removed, ig.n_added) == (io.n_split, io.n_removed, io.n_added)
    assert g.n == o.n
    np.testing.assert_array_equal(g.get("tag"), o.get("tag"))
    for q in ["x", "y", "z"]:
        assert rel(g.get(q), o.get(q)) < 1e-5, q
    for name in ["u", "v", "w"]:
        assert rel_l2(g.grid(name), o.grid(name)) < TOL_VEL, name


def test_mixed_kept_binning_counts_match_a_fresh_binning(pm):
    """Within a step the mixed form keeps the binning's cell ids and counts
    current through the RK4 stages, the haloswap, splitting and mixing instead
    of recounting.  After steps with splits, removals and new parcels, a
    par2grid through those kept counts equals, bit for bit, the par2grid of a
    fresh context holding the same parcels (which bins from scratch; the cell
    index orders each cell by slot either way)."""
    n = 16
    ic = _vortical(pm, n, amp=3.0)
    k = len(ic["x"])
    rng = np.random.default_rng(41)
    ic["stretch"] = np.where(rng.uniform(size=k) < 0.1, 4.5, 3.5)
    vmin = (TWO_PI / n) ** 2 * (math.pi / n) / 216
    ic["vol"][rng.uniform(size=k) < 0.1] = 0.5 * vmin
    ic["vol"][ic["x"] < 0.3] = 0.5 * vmin  # most of a column of cells emptied: new parcels there
    cap = 4 * k
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.02, dtmax=0.02, max_parcels=cap, precision="mixed")
    g.upload(**ic)
    g.step(1)
    info = g.info()
    assert info.n_split > 0 and info.n_removed > 0 and info.n_added > 0
    g.step(1)
    g.par2grid_multi(["p", "q", "r"], ["p", "q", "r"])  # through the kept counts
    kept = {q: g.grid(q) for q in ["p", "q", "r"]}
    f = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.02, dtmax=0.02, max_parcels=cap, precision="mixed")
    f.upload(**{q: g.get(q) for q in pm.DUMP_PROPS})
    assert f.n == g.n
    f.par2grid_multi(["p", "q", "r"], ["p", "q", "r"])  # a fresh binning
    for q in ["p", "q", "r"]:
        np.testing.assert_array_equal(kept[q], f.grid(q), err_msg=q)
    np.testing.assert_array_equal(g.cell_ids(), f.cell_ids())


def test_mixed_mixing_conserves_volume(pm):
    """parcel_mixing moves volume between removed, new and kept parcels and
    conserves its total (the report's check, report.tex:264); FP32 volumes
    sum to the FP64 total within FP32 rounding."""
    n = 16
    ic = _vortical(pm, n)
    k = len(ic["x"])
    rng = np.random.default_rng(5)
    vmin = (TWO_PI / n) ** 2 * (math.pi / n) / 216
    ic["vol"][rng.uniform(size=k) < 0.5] = 0.5 * vmin
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * k, precision="mixed")
    g.upload(**ic)
    v0 = np.sum(g.get("vol"))
    g.set_counters([3, 3, 4, 3, 3])  # the next callbacks are the fourth substep's
    g.parcel_mixing()
    v1 = np.sum(g.get("vol"))
    assert g.info().n_removed > 0
    assert abs(v1 - v0) / v0 < 1e-5


def test_mixed_deterministic(pm):
    n = 16
    ic = _vortical(pm, n)
    res = []
    for _ in range(2):
        g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * len(ic["x"]), precision="mixed")
        g.upload(**ic)
        g.step(2)
        res.append({q: g.get(q) for q in ["x", "z", "p", "vol"]} | {"u": g.grid("u")})
        g.close()
    for q in res[0]:
        np.testing.assert_array_equal(res[0][q], res[1][q], err_msg=q)


def test_mixed_rejects_fp64_kernel_ops(pm):
    g = pm.Context(8, 8, 8, 1.0, 1.0, 1.0, max_parcels=16, precision="mixed")
    g.upload(x=np.array([0.5]), y=np.array([0.5]), z=np.array([0.5]), vol=np.ones(1))
    with pytest.raises(pm.PmpicError) as e:
        g.par2grid("b", "b")
    assert e.value.code == -9  # PMPIC_ERR_STATE


def test_mixed_mixing_without_events_keeps_parcels(pm):
    """A mixing call that removes no parcel and adds none leaves every residual
    grid at zero; the mixed form then skips the redistribution: the parcels are
    unchanged bit for bit, the counts report no event, and the kept volume grid
    (the model's vol grid of construct_grids, which the dumps write) is still
    built, within FP32 rounding of the oracle's.  Without removed parcels the
    mixed form builds the other kept grids (b, hg, p, q, r) only at the corners
    of new parcels' cells (covered by the next test): elsewhere they are
    scratch."""
    from oracle import Oracle
    n = 16
    ic = _vortical(pm, n)
    k = len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k, precision="mixed")
    g.upload(**ic)
    props = ["x", "y", "z", "p", "q", "r", "b", "h", "vol", "stretch", "tag"]
    before = {q: g.get(q) for q in props}
    g.set_counters([3, 3, 4, 3, 3])  # the next callbacks are the fourth substep's
    g.parcel_mixing()
    info = g.info()
    assert info.n_removed == 0 and info.n_added == 0 and g.n == k
    for q in props:
        np.testing.assert_array_equal(g.get(q), before[q], err_msg=q)
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k)
    o.set_parcels(**ic)
    o.set_counters([3, 3, 4, 3, 3])
    o.parcel_mixing()
    assert o.info().n_removed == 0 and o.info().n_added == 0
    assert rel(g.grid("vol"), o.grid("vol")) < 1e-5


def test_mixed_new_parcels_without_removals_vs_oracle(pm):
    """Cells emptied of parcels (inside, at both walls, across the periodic
    corner), no parcel below vmin: mixing adds a parcel in each under-populated
    cell.  The mixed form makes the kept volume grid in full and the kept b, h,
    p, q, r sums only at the corners of the new parcels' cells, from the cells'
    parcels directly.  Counts, slots and tags equal the oracle's; the new and
    the redistributed parcels, the volume grid and the kept sums at those
    corners agree with the FP64 oracle within FP32 rounding."""
    from oracle import Oracle
    n = 16
    ic = _vortical(pm, n)
    dx, dz = TWO_PI / n, math.pi / n
    ci = np.floor(ic["x"] / dx).astype(int) % n
    cj = np.floor(ic["y"] / dx).astype(int) % n
    ck = np.minimum(np.floor(ic["z"] / dz).astype(int), n - 1)
    emptied = [(5, 5, 5), (5, 6, 5), (10, 3, 0), (12, 12, n - 1), (0, 0, 8), (n - 1, n - 1, 8)]
    drop = np.zeros(len(ic["x"]), bool)
    for c in emptied:
        drop |= (ci == c[0]) & (cj == c[1]) & (ck == c[2])
    assert drop.sum() >= len(emptied)
    ic = {q: v[~drop] for q, v in ic.items()}
    k = len(ic["x"])
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k, precision="mixed")
    g.upload(**ic)
    g.set_counters([3, 3, 4, 3, 3])
    g.parcel_mixing()
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k)
    o.set_parcels(**ic)
    o.set_counters([3, 3, 4, 3, 3])
    o.parcel_mixing()
    ig, io = g.info(), o.info()
    assert ig.n_removed == io.n_removed == 0
    assert ig.n_added == io.n_added >= len(emptied) and g.n == o.n
    np.testing.assert_array_equal(g.get("tag"), o.get("tag"))
    for q in ["x", "y", "z", "b", "h", "p", "q", "r", "vol"]:
        assert rel(g.get(q), o.get(q)) < 1e-5, q
    assert rel(g.grid("vol"), o.grid("vol")) < 1e-5
    # the kept sums at the corners of the emptied cells (grids are (z, y, x))
    pts = {(c[2] + a, (c[1] + b) % n, (c[0] + d) % n) for c in emptied for a in (0, 1) for b in (0, 1) for d in (0, 1)}
    idx = tuple(np.array(sorted(pts)).T)
    for name in ["b", "hg", "p", "q", "r"]:
        a, b = g.grid(name)[idx], o.grid(name)[idx]
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max(), name


def test_mixed_mixing_redistributes_only_near_events(pm):
    """A few parcels shrunk below vmin in one region: the mixed form applies the
    residuals to the kept parcels whose cells are within one cell of a removed
    or a new parcel's cell (only their corners can hold residuals) and leaves
    every other parcel bit for bit as it was; parcels, counts and the volume
    total agree with the FP64 oracle within FP32 rounding."""
    from oracle import Oracle
    n = 16
    ic = _vortical(pm, n)
    k = len(ic["x"])
    vmin = (TWO_PI / n) ** 2 * (math.pi / n) / 216
    dx, dz = TWO_PI / n, math.pi / n
    region = (ic["x"] < 2 * dx) & (ic["y"] < 2 * dx) & (ic["z"] < 2 * dz)
    shrink = np.nonzero(region)[0][::3]
    ic["vol"][shrink] = 0.5 * vmin
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k, precision="mixed")
    g.upload(**ic)
    before = {q: g.get(q) for q in ["b", "h", "p", "q", "r", "vol"]}
    g.set_counters([3, 3, 4, 3, 3])
    g.parcel_mixing()
    o = Oracle(n, n, n, TWO_PI, TWO_PI, math.pi, max_parcels=2 * k)
    o.set_parcels(**ic)
    o.set_counters([3, 3, 4, 3, 3])
    o.parcel_mixing()
    ig, io = g.info(), o.info()
    assert ig.n_removed == io.n_removed == len(shrink)
    assert (ig.n_removed, ig.n_added) == (io.n_removed, io.n_added) and g.n == o.n
    np.testing.assert_array_equal(g.get("tag"), o.get("tag"))
    for q in ["b", "h", "p", "q", "r", "vol"]:
        assert rel(g.get(q), o.get(q)) < 1e-5, q
    # parcels whose cell is more than one cell away (periodically) from the region are untouched
    tag = g.get("tag").astype(np.int64)
    ci = np.floor(g.get("x") / dx).astype(int) % n
    cj = np.floor(g.get("y") / dx).astype(int) % n
    ck = np.floor(g.get("z") / dz).astype(int)
    far = ((ci >= 3) & (ci <= n - 2)) | ((cj >= 3) & (cj <= n - 2)) | (ck >= 3)
    assert far.sum() > k // 2
    for q in ["b", "h", "p", "q", "r", "vol"]:
        np.testing.assert_array_equal(g.get(q)[far], before[q][tag[far]], err_msg=q)


def test_mixed_step_does_not_depend_on_gather_windows(pm):
    """The RK4 stage stages each CTA's gather window (the packed grids around
    the cell its first parcel reached at the previous stage) in shared memory;
    parcels outside the window gather from the packed grids in global memory,
    with the same values and arithmetic.  A context that already ran a step
    keeps its window hints through a new upload, so the first stage of its
    next step stages windows; a fresh context's first stage has no hint and
    gathers from global memory.  The same upload stepped once gives the same
    bits in both."""
    n = 32
    ic = _vortical(pm, n)
    k = len(ic["x"])
    dt = 0.01
    g = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=dt, dtmax=dt, max_parcels=2 * k, precision="mixed")
    c0 = g.counters()
    g.upload(**ic)
    g.step(1)
    g.upload(**ic)  # the hints of the step's last stage stay
    g.set_counters(c0)
    f = pm.Context(n, n, n, TWO_PI, TWO_PI, math.pi, dtm=dt, dtmax=dt, max_parcels=2 * k, precision="mixed")
    f.upload(**ic)
    g.step(1)
    f.step(1)
    assert g.n == f.n
    for q in pm.IO_PROPS:
        np.testing.assert_array_equal(g.get(q), f.get(q), err_msg=q)
    for name in ["u", "v", "w"]:
        np.testing.assert_array_equal(g.grid(name), f.grid(name), err_msg=name)
