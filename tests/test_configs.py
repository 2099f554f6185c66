"""Parity at the benchmark configurations, against the oracle, through the C ABI.
Needs a CUDA device.

* Interpolation at 128^3: 8 parcels per cell (16.8 M) at seeded uniform random
  positions, fields that are sums of 16 random Fourier modes (|k| <= 8, N(0, 1)
  amplitudes).  Cell binning bit for bit (both forms); par2grid of 4 fields and
  grid2par of 6 within 1e-12 on the FP64 path (parcel_interpolation.F90:186-481);
  the FP32 form's errors are asserted below 1e-5 relative and printed.
* vort2vel's inversion alone at 256^3 on a divergence-free k^-5/3 vorticity
  (|k| <= 64, unit RMS, wall conditions): velocity, corrected vorticity and the
  filtered spectra within 1e-12 on the FP64 path (vort2vel.F90:98-400); the
  mixed form's velocity within 1e-4.
* One full model step of the thermal plume on the FP64 path at 256^3
  (128^3 when the host has too little memory for the oracle at 256^3; the test
  prints which): parcel count and split / mixing counts equal, the slot -> tag
  map bit for bit, every parcel property within 1e-12, gridded u, v, w within
  1e-10.  The GPU state is written by the device set-up (positions, h, vol and
  tags bit for bit the oracle's; b within the rounding of the device cos).
* 100 steps of the 64^3 plume in both forms against the FP64 oracle: the FP64
  path's gridded velocity within 1e-9 and its parcel count and tags identical;
  the mixed form's gridded velocity within 1e-4 relative L2 and its parcel
  count identical.
"""
import math
import os

import numpy as np
import pytest

from helpers import rel, rel_l2

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi
THREADS = os.cpu_count() or 1
# the jittered thermal of the plume workloads, in the box [0, 2 pi]^2 x [0, pi]
THERMAL = dict(sub=2, jitter=0.25, seed=1, xc=math.pi, yc=math.pi, zc=0.6, radius=0.4, excess=1.0,
               h_in=0.95, h_env0=0.3, z_strat=1.2, n2=1.0)


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


def fourier_field(x, y, z, nmodes, kmax, rng, lx=TWO_PI, ly=TWO_PI, lz=math.pi):
    """Sum of nmodes random Fourier modes with 0 < |k| <= kmax and N(0, 1)
    amplitudes, periodic in x and y and cos(m pi z / lz) in z.  Evaluated in
    FP64 with torch on the GPU (input generation only: the same arrays go to
    the oracle and to the library)."""
    import torch
    tx, ty, tz = (torch.as_tensor(np.asarray(a, dtype=np.float64)).cuda() for a in (x, y, z))
    out = torch.zeros(torch.broadcast_shapes(tx.shape, ty.shape, tz.shape), dtype=torch.float64, device="cuda")
    done = 0
    while done < nmodes:
        a, b, m = rng.integers(-kmax, kmax + 1), rng.integers(-kmax, kmax + 1), rng.integers(0, kmax + 1)
        kx, ky, kz = TWO_PI * a / lx, TWO_PI * b / ly, math.pi * m / lz
        if not (0 < kx * kx + ky * ky + kz * kz <= kmax * kmax):
            continue
        amp, ph = rng.standard_normal(), rng.uniform(0, TWO_PI)
        out += amp * torch.cos(kx * tx + ky * ty + ph) * torch.cos(kz * tz)
        done += 1
    return out.cpu().numpy()


def test_interpolation_128(pm):
    from oracle import Oracle
    G = 128
    P = 8 * G ** 3
    rng = np.random.default_rng(2)
    x = rng.uniform(0, TWO_PI, P)
    y = rng.uniform(0, TWO_PI, P)
    z = rng.uniform(0, math.pi, P)
    vol = np.full(P, (TWO_PI / G) ** 2 * (math.pi / G) / 8)
    frng = np.random.default_rng(3)
    p4 = ["p", "q", "r", "b"]
    g6 = ["u", "v", "w", "dp", "dq", "dr"]
    props6 = ["dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt"]
    fields = {q: fourier_field(x, y, z, 16, 8, frng) for q in p4}
    zg, yg, xg = np.meshgrid(np.arange(G + 1) * (math.pi / G), np.arange(G) * (TWO_PI / G),
                             np.arange(G) * (TWO_PI / G), indexing="ij")
    grids = {g: fourier_field(xg, yg, zg, 16, 8, frng) for g in g6}

    o = Oracle(G, G, G, TWO_PI, TWO_PI, math.pi, max_parcels=P, threads=THREADS)
    o.set_parcels(x=x, y=y, z=z, vol=vol, **fields)
    ref_cells = o.cache_weights()
    ref_grid = {}
    for q in p4:
        o.par2grid(q, q)
        ref_grid[q] = o.grid(q)
    for g, q in zip(g6, props6):
        o.set_grid(g, grids[g])
        o.grid2par(g, q)
    ref_par = {q: o.get(q) for q in props6}
    o.close()

    errs = {}
    for prec in ("fp64", "mixed"):
        ctx = pm.Context(G, G, G, TWO_PI, TWO_PI, math.pi, max_parcels=P, precision=prec)
        ctx.upload(x=x, y=y, z=z, vol=vol, **fields, tag=np.arange(P, dtype=np.float64))
        np.testing.assert_array_equal(ctx.cell_ids(), ref_cells, err_msg=prec)
        ctx.par2grid_multi(p4, p4)
        for g in g6:
            ctx.set_grid(g, grids[g])
        ctx.grid2par_multi(g6, props6)
        for q in p4:
            errs[(prec, "par2grid", q)] = (rel(ctx.grid(q), ref_grid[q]), rel_l2(ctx.grid(q), ref_grid[q]))
        for q in props6:
            errs[(prec, "grid2par", q)] = (rel(ctx.get(q), ref_par[q]), rel_l2(ctx.get(q), ref_par[q]))
        ctx.close()
    for k, (emax, el2) in sorted(errs.items()):
        print(f"{k}: max rel {emax:.3e}, rel L2 {el2:.3e}")
        bound = 1e-12 if k[0] == "fp64" else 1e-5
        assert emax < bound and el2 < bound, (k, emax, el2)


def test_vort2vel_256(pm):
    from oracle import Oracle
    G = 256
    p, q, r = pm.random_vorticity(G, G, G, kmax=64, seed=4)
    o = Oracle(G, G, G, TWO_PI, TWO_PI, math.pi, max_parcels=16, threads=THREADS)
    for name, a in (("p", p), ("q", q), ("r", r)):
        o.set_grid(name, a)
    o.vort2vel_grids()
    grids = ("u", "v", "w", "p", "q", "r")
    specs = ("u_s", "v_s", "w_s")
    ref = {k: o.grid(k) for k in grids}
    ref_s = {k: o.spec(k) for k in specs}
    o.close()
    for prec in ("fp64", "mixed"):
        ctx = pm.Context(G, G, G, TWO_PI, TWO_PI, math.pi, max_parcels=16, precision=prec)
        for name, a in (("p", p), ("q", q), ("r", r)):
            ctx.set_grid(name, a)
        ctx.vort2vel_grids()
        out = {k: ctx.grid(k) for k in grids}
        out_s = {k: ctx.spec(k) for k in specs}
        ctx.close()
        for k in grids:
            e = rel_l2(out[k], ref[k])
            print(f"{prec} {k}: rel L2 {e:.3e}, max rel {rel(out[k], ref[k]):.3e}")
            if prec == "fp64":
                assert e < 1e-12 and rel(out[k], ref[k]) < 1e-12, (k, e)
            elif k in ("u", "v", "w"):
                assert e < 1e-4, (prec, k, e)
        for k in specs:
            e = rel_l2(out_s[k], ref_s[k])
            print(f"{prec} {k}: rel L2 {e:.3e}")
            assert e < (1e-12 if prec == "fp64" else 1e-4), (prec, k, e)


def _oracle_fits(G, cap):
    """Whether the oracle's state at G^3 (about 290 bytes per parcel slot plus
    the grids) fits in the host's available memory with a margin."""
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        return False
    need = 290 * cap + 40 * 8 * (G + 1) * (G + 4) ** 2
    return avail > 1.3 * need


def test_plume_step_fp64(pm):
    """One model step (4 RK4 substeps, splitting, mixing) of the thermal plume at
    dt = 0.0025 on the FP64 path against the oracle."""
    from oracle import Oracle
    G = 256
    cap = int(1.05 * 8 * G ** 3)
    if not _oracle_fits(G, cap):
        G = 128
        cap = int(1.05 * 8 * G ** 3)
    print(f"plume step at {G}^3")
    o = Oracle(G, G, G, TWO_PI, TWO_PI, math.pi, dtm=0.0025, dtmax=0.0025, max_parcels=cap, threads=THREADS)
    o.setup_thermal(**THERMAL)
    ctx = pm.Context(G, G, G, TWO_PI, TWO_PI, math.pi, dtm=0.0025, dtmax=0.0025, max_parcels=cap)
    ctx.setup_thermal(nx=G, ny=G, nz=G, **THERMAL)
    n0 = ctx.n
    assert n0 == o.n == 8 * G ** 3
    ctx.step(1)
    o.step()
    gi, oi = ctx.info(), o.info()
    assert ctx.n == o.n
    assert (gi.n_split, gi.n_removed, gi.n_added) == (oi.n_split, oi.n_removed, oi.n_added)
    assert gi.limiter == oi.limiter == 0
    n = o.n
    np.testing.assert_array_equal(ctx.get("tag"), o.get("tag"))
    for k in ("u", "v", "w"):
        a, b = ctx.grid(k), o.grid(k)
        print(f"{k}: max rel {rel(a, b):.3e}")
        assert rel(a, b) < 1e-10, k
    for k in ("x", "y", "z", "p", "q", "r", "b", "h", "vol", "stretch"):
        a, b = ctx.get(k), o.get(k)
        assert a.shape == (n,)
        assert rel(a, b) < 1e-12, k
    ctx.close()
    o.close()


def test_plume_100_steps_vs_oracle(pm):
    """100 steps of the 64^3 plume (dt = 0.01): the FP64 path and the mixed form
    against the FP64 oracle."""
    from oracle import Oracle
    G, dt, steps = 64, 0.01, 100
    cap = int(1.2 * 8 * G ** 3)
    o = Oracle(G, G, G, TWO_PI, TWO_PI, math.pi, dtm=dt, dtmax=dt, max_parcels=cap, threads=THREADS)
    o.setup_thermal(**THERMAL)
    for _ in range(steps):
        o.step()
    ref = {k: o.grid(k) for k in ("u", "v", "w")}
    ref_tag = o.get("tag")
    n_ref = o.n
    o.close()
    for prec in ("fp64", "mixed"):
        ctx = pm.Context(G, G, G, TWO_PI, TWO_PI, math.pi, dtm=dt, dtmax=dt, max_parcels=cap, precision=prec)
        ctx.setup_thermal(nx=G, ny=G, nz=G, **THERMAL)
        ctx.step(steps)
        for k in ("u", "v", "w"):
            a = ctx.grid(k)
            e2, em = rel_l2(a, ref[k]), rel(a, ref[k])
            print(f"{prec} {k}: rel L2 {e2:.3e}, max rel {em:.3e} after {steps} steps")
            assert e2 < (1e-9 if prec == "fp64" else 1e-4), (prec, k, e2)
        print(f"{prec}: parcels {ctx.n} (oracle {n_ref})")
        assert ctx.n == n_ref, prec
        if prec == "fp64":
            np.testing.assert_array_equal(ctx.get("tag"), ref_tag)
        ctx.close()


def test_plume_invariants_after_100_steps(pm):
    """Size-independent properties of the reference's algorithm on the GPU path,
    both forms, after 100 steps of the 128^3 plume (dt 0.005):
    * every interior cell holds at least three parcels after mixing (a cell with
      fewer kept parcels gets a new one, parcel_mixing.F90:160-212);
    * without splits and removals (this plume has none), every set-up tag
      survives exactly once through the haloswap re-slots and mixing, and the
      new parcels carry the zero tag of the unused slots they are appended to
      (the reference does not set a new parcel's tag);
    * every position lies in the box, z in [0, Lz];
    * the total volume equals the set-up's (splitting halves, mixing moves
      volume between parcels: the compensated total is conserved to rounding);
    * the step info's counters add up: final count = initial + added + split -
      removed over the run."""
    G, dt, steps = 128, 0.005, 100
    for prec in ("fp64", "mixed"):
        cap = int(1.1 * 8 * G ** 3)
        ctx = pm.Context(G, G, G, TWO_PI, TWO_PI, math.pi, dtm=dt, dtmax=dt, max_parcels=cap, precision=prec)
        ctx.setup_thermal(nx=G, ny=G, nz=G, **THERMAL)
        n0 = ctx.n
        v0 = ctx.conserved_sums()[0]
        added = removed = split = 0
        for _ in range(steps):
            ctx.step(1)
            inf = ctx.info()
            added += inf.n_added
            removed += inf.n_removed
            split += inf.n_split
        n = ctx.n
        assert n == n0 + added + split - removed, (prec, n, n0, added, split, removed)
        x, y, z = ctx.get("x"), ctx.get("y"), ctx.get("z")
        assert x.min() >= 0 and x.max() < TWO_PI and y.min() >= 0 and y.max() < TWO_PI, prec
        assert z.min() >= 0 and z.max() <= math.pi, prec
        cells = ctx.cell_ids()
        per_cell = np.bincount(cells, minlength=G ** 3)
        assert per_cell.min() >= 3, (prec, per_cell.min())
        tag = ctx.get("tag").astype(np.int64)
        if split == 0 and removed == 0:
            # every set-up tag once; the new parcels keep their slot's tag, 0 in the
            # never-used slots they are appended to (the reference does not set it)
            cnt = np.bincount(tag)
            assert len(cnt) == n0 and (cnt[1:] == 1).all() and cnt[0] == 1 + added, prec
        v1 = ctx.conserved_sums()[0]
        tol = 1e-12 if prec == "fp64" else 1e-5
        assert abs(v1 - v0) <= tol * v0, (prec, v0, v1)
        print(f"{prec}: {steps} steps, parcels {n0} -> {n} (added {added}, split {split}, removed {removed}), "
              f"min parcels per cell {per_cell.min()}, volume {v0!r} -> {v1!r}")
        ctx.close()
