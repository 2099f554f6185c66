"""The reference's test components for the parcel migration path:
euler_integrator (euler_integrator.F90:53-86) and prescribed_parcel_velocity
(velocity.F90: the quadrant tags of its initialisation, :72-84, and the
analytic tendencies of its eleven profiles, :96-255).

CPU: the oracle's restatement against an independent numpy statement of the
same formulas (profiles, tags, the explicit step).  GPU: the library against
the oracle -- tags and the constant profiles bit for bit, the transcendental
profiles (tanh, atan2, exp, sin, cos of CUDA against glibc) within 1e-14
relative, and several Euler steps that move parcels across the periodic
boundaries: positions, tags and slot order bit for bit, the same migrations.
"""
import math

import numpy as np
import pytest

TWO_PI = 2 * math.pi
N = 16


def _parcels(k, seed):
    rng = np.random.default_rng(seed)
    return {"x": rng.uniform(0, TWO_PI, k), "y": rng.uniform(0, TWO_PI, k), "z": rng.uniform(0, math.pi, k),
            "p": rng.standard_normal(k), "q": rng.standard_normal(k), "r": rng.standard_normal(k),
            "vol": np.full(k, 0.01), "tag": np.arange(k, dtype=np.float64)}


def _numpy_profile(profile, x, y):
    """velocity.F90:103-250 with the global grid of setup_grid.F90:87-93
    (bottom 0, top = the last grid point L - L/N)."""
    top = TWO_PI - TWO_PI / N
    x0, y0, r0 = top / 2.0, top / 2.0, top / 8.0
    z = np.zeros_like(x)
    if profile == 0:
        return z, np.tanh((x - x0) / r0)
    if profile == 9:
        theta = np.arctan2(y - y0, x - x0)
        r2 = (x - x0) * (x - x0) + (y - y0) * (y - y0)
        v0 = np.exp(-r2 / r0 / r0 / 2) / x0 * 10
        return v0 * np.sqrt(r2) * np.sin(theta), -v0 * np.sqrt(r2) * np.cos(theta)
    if profile == 10:
        xc1, yc1, xc2, yc2 = 0.25 * top, 0.25 * top, 0.75 * top, 0.75 * top
        r1 = np.sqrt((x - xc1) ** 2 + (y - yc1) ** 2)
        r2 = np.sqrt((x - xc2) ** 2 + (y - yc2) ** 2)
        e1, e2 = np.exp(-r1 * r1 / r0 / r0 / 4), np.exp(-r2 * r2 / r0 / r0 / 4)
        return -(x - xc1) / r1 * e1 + (x - xc2) / r2 * e2, -(y - yc1) / r1 * e1 + (y - yc2) / r2 * e2
    dirs = {1: (0, 1), 2: (1, 1), 3: (1, 0), 4: (1, -1), 5: (0, -1), 6: (-1, -1), 7: (-1, 0), 8: (-1, 1)}
    u, v = dirs[profile]
    return z + u, z + v


def test_oracle_profiles_tags_and_step_vs_numpy():
    from oracle import Oracle
    k = 4000
    ic = _parcels(k, 1)
    o = Oracle(N, N, N, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * k)
    o.set_parcels(**ic)
    for profile in range(11):
        o.prescribed_velocity(profile)
        u, v = _numpy_profile(profile, ic["x"], ic["y"])
        np.testing.assert_allclose(o.get("dxdt"), u, rtol=1e-14, atol=1e-15, err_msg=str(profile))
        np.testing.assert_allclose(o.get("dydt"), v, rtol=1e-14, atol=1e-15, err_msg=str(profile))
        assert np.all(o.get("dzdt") == 0.0)
    o.prescribed_velocity_tag()
    top = TWO_PI - TWO_PI / N
    np.testing.assert_array_equal(o.get("tag"), 2.0 * (ic["y"] > top / 2) + 1.0 * (ic["x"] > top / 2))
    # one explicit step that moves no parcel out of the domain: x += dxdt * dt exactly
    o.set_parcels(**ic)
    o.prescribed_velocity(9)
    d = {q: o.get(q) for q in ["dxdt", "dydt", "dzdt"]}
    o.euler_integrator()
    assert o.n == k
    for q, dq in [("x", "dxdt"), ("y", "dydt")]:
        moved = ic[q] + d[dq] * 0.01
        inside = (moved > 0.1) & (moved < TWO_PI - 0.1)
        np.testing.assert_array_equal(o.get(q)[inside], moved[inside], err_msg=q)


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


@pytest.mark.gpu
def test_prescribed_velocity_and_tags_vs_oracle(pm):
    from oracle import Oracle
    k = 20000
    ic = _parcels(k, 2)
    g = pm.Context(N, N, N, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * k)
    o = Oracle(N, N, N, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * k)
    g.upload(**ic)
    o.set_parcels(**ic)
    for profile in range(11):
        g.prescribed_velocity(profile)
        o.prescribed_velocity(profile)
        for q in ["dxdt", "dydt", "dzdt"]:
            a, b = g.get(q), o.get(q)
            if profile in (0, 9, 10):
                np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-15, err_msg=f"{profile} {q}")
            else:
                np.testing.assert_array_equal(a, b, err_msg=f"{profile} {q}")
    g.prescribed_velocity_tag()
    o.prescribed_velocity_tag()
    np.testing.assert_array_equal(g.get("tag"), o.get("tag"))
    with pytest.raises(Exception):
        g.prescribed_velocity(11)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("profile", [2, 4, 6, 8])  # NE, SE, SW, NW: across both periodic boundaries
def test_euler_migration_vs_oracle(pm, profile):
    from oracle import Oracle
    k = 12000
    ic = _parcels(k, 3 + profile)
    dt = 0.15  # about 0.4 of a cell per step: parcels cross the boundaries every few steps
    g = pm.Context(N, N, N, TWO_PI, TWO_PI, math.pi, dtm=dt, dtmax=dt, max_parcels=2 * k)
    o = Oracle(N, N, N, TWO_PI, TWO_PI, math.pi, dtm=dt, dtmax=dt, max_parcels=2 * k)
    g.upload(**ic)
    o.set_parcels(**ic)
    migrated = 0
    for _ in range(6):
        for c in (g, o):
            c.prescribed_velocity(profile)
            c.euler_integrator()
        ig, io = g.info(), o.info()
        assert ig.n_migrated == io.n_migrated
        migrated += ig.n_migrated
        assert g.n == o.n == k
        for q in ["x", "y", "z", "p", "q", "r", "tag"]:
            np.testing.assert_array_equal(g.get(q), o.get(q), err_msg=q)
    assert migrated > 0
    g.close()
