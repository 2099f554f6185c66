"""Initial conditions written on the device.

basic_parcelsetup (basic_parcelsetup.F90:22-134) and plume_parcelsetup
(plume_parcelsetup.F90:58-334): the oracle's restatements against independent
numpy statements of the same loops (CPU), then the
device set-up against the oracle, bit for bit, for both forms (GPU).  The
jittered thermal of the benchmark workloads: the device generator against the
host one (GPU).
"""
import math

import numpy as np
import pytest

IO = ["x", "y", "z", "p", "q", "r", "b", "h", "vol", "stretch", "tag"]
REF_CFG = dict(lam=1.0, H=0.8, z_c=2.5, mu=0.9, z_d=4.0, z_m=5.0, r_plume=0.8, e_values=(0.3, -0.4, 0.5))
# grids: the reference's config.mcf (32^3 cells on [0, 6.28]^3) and a non-cubic box
GRIDS = [(32, 32, 32, 6.28, 6.28, 6.28), (24, 20, 12, 2 * math.pi, 5.0, math.pi)]


def _walk(start, step, count):
    out, v = [], start
    for _ in range(count):
        out.append(v)
        v = v + step
    return np.array(out)


def numpy_plume(nx, ny, nz, lx, ly, lz, lam, H, z_c, mu, z_d, z_m, r_plume, e_values):
    """plume_parcelsetup.F90:58-334 for one process on [0, lx) x [0, ly) x [0, lz]
    (nz cells, nz + 1 points), written from the Fortran independently of the oracle."""
    fdthetal0 = float(np.float32(0.01))  # a default-real literal widened to double
    glat = (1.0 / fdthetal0) * 0.125
    h_pl = math.exp(-z_c)
    h_bg = mu * h_pl
    z_b = math.log(H / h_bg)
    dbdz = glat * (h_pl - math.exp(-z_m)) / (z_m - z_d)
    b_pl = dbdz * (z_d - z_b)
    z_b, r = z_b * lam, r_plume * lam
    e = [v / r / r for v in e_values]
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    xc = ((lx - dx) + dx - 0.0) / 2 + 0.0
    yc = ((ly - dy) + dy - 0.0) / 2 + 0.0
    zc = r
    out = {k: [] for k in ["x", "y", "z", "b", "h", "vol"]}
    # plume lattice, 4 per cell per direction
    X = _walk(0.0 + dx / 4 / 2.0, dx / 4, nx * 4)
    Y = _walk(0.0 + dy / 4 / 2.0, dy / 4, ny * 4)
    Z = _walk(0.0 + dz / 4 / 2.0, dz / 4, int(math.ceil(2.0 * r / (dz / 4))))
    xp, yp, zp = (X - xc)[:, None, None], (Y - yc)[None, :, None], (Z - zc)[None, None, :]
    inside = zp * zp + xp * xp + yp * yp <= r * r
    shape = inside.shape
    for k, v in [("x", X[:, None, None]), ("y", Y[None, :, None]), ("z", Z[None, None, :])]:
        out[k].append(np.broadcast_to(v, shape)[inside])
    bb = b_pl * (1.0 + e[0] * xp * yp + e[1] * xp * zp + e[2] * yp * zp)
    out["b"].append(np.broadcast_to(bb, shape)[inside])
    out["h"].append(np.full(inside.sum(), h_pl))
    out["vol"].append(np.full(inside.sum(), (dx / 4) * (dy / 4) * (dz / 4)))
    n_plume = int(inside.sum())
    # environment lattice, 2 per cell per direction
    X = _walk(0.0 + dx / 2 / 2.0, dx / 2, nx * 2)
    Y = _walk(0.0 + dy / 2 / 2.0, dy / 2, ny * 2)
    Z = _walk(0.0 + dz / 2 / 2.0, dz / 2, nz * 2)
    xp, yp, zp = (X - xc)[:, None, None], (Y - yc)[None, :, None], (Z - zc)[None, None, :]
    outside = zp * zp + yp * yp + xp * xp > r * r
    shape = outside.shape
    for k, v in [("x", X[:, None, None]), ("y", Y[None, :, None]), ("z", Z[None, None, :])]:
        out[k].append(np.broadcast_to(v, shape)[outside])
    bz = np.array([0.0 if z < z_b else dbdz / lam * (z - z_b) for z in Z])
    hz = np.array([h_bg if z < z_b else H * math.exp(-z / lam) for z in Z])
    out["b"].append(np.broadcast_to(bz[None, None, :], shape)[outside])
    out["h"].append(np.broadcast_to(hz[None, None, :], shape)[outside])
    out["vol"].append(np.full(outside.sum(), (dx / 2) * (dy / 2) * (dz / 2)))
    return {k: np.concatenate(v) for k, v in out.items()}, n_plume


@pytest.mark.parametrize("grid", GRIDS)
def test_oracle_plume_vs_numpy(grid):
    from oracle import Oracle
    want, n_plume = numpy_plume(*grid, **REF_CFG)
    n = len(want["x"])
    o = Oracle(*grid, max_parcels=n + 10)
    assert o.setup_plume(**REF_CFG) == n_plume
    assert o.n == n
    for k, v in want.items():
        np.testing.assert_array_equal(o.get(k), v, err_msg=k)
    for k in ["p", "q", "r", "stretch", "tag"]:
        assert np.all(o.get(k) == 0.0)
    assert 0 < n_plume < n


@pytest.mark.parametrize("cfg", [
    dict(lam=0.8, H=0.7, z_c=2.5, mu=0.85, z_d=3.5, z_m=4.5, r_plume=0.5, e_values=(0.1, 0.2, -0.3)),
    dict(lam=1.3, H=0.9, z_c=1.2, mu=0.95, z_d=2.0, z_m=2.6, r_plume=0.55, e_values=(-0.5, 0.0, 0.25)),
])
def test_oracle_plume_other_parameters_vs_numpy(cfg):
    from oracle import Oracle
    grid = (20, 16, 24, 5.0, 4.0, 3.5)
    want, n_plume = numpy_plume(*grid, **cfg)
    o = Oracle(*grid, max_parcels=len(want["x"]))
    assert o.setup_plume(**cfg) == n_plume
    for k, v in want.items():
        np.testing.assert_array_equal(o.get(k), v, err_msg=k)
    assert np.any(o.get("b")[n_plume:] > 0)  # part of the environment lies in the stratified layer


def test_oracle_plume_parameter_checks():
    from oracle import Oracle, OracleError
    o = Oracle(16, 16, 16, 6.28, 6.28, 6.28, max_parcels=100000)
    for bad in [dict(H=1.2), dict(mu=0.7), dict(mu=1.1), dict(r_plume=5.0)]:
        with pytest.raises(OracleError):
            o.setup_plume(**{**REF_CFG, **bad})
    small = Oracle(16, 16, 16, 6.28, 6.28, 6.28, max_parcels=1000)
    with pytest.raises(OracleError):
        small.setup_plume(**REF_CFG)


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


@pytest.mark.gpu
@pytest.mark.parametrize("grid", GRIDS)
def test_device_plume_vs_oracle(pm, grid):
    from oracle import Oracle
    o = Oracle(*grid, max_parcels=400000)
    n_plume = o.setup_plume(**REF_CFG)
    g = pm.Context(*grid, max_parcels=400000)
    g.upload(**{k: np.full(1000, 0.5) for k in IO})  # state to be replaced
    assert g.setup_plume(**REF_CFG) == n_plume
    assert g.n == o.n
    for k in IO + ["dxdt", "btot"]:
        np.testing.assert_array_equal(g.get(k), o.get(k), err_msg=k)
    # the mixed form holds the same parcels as an upload of the oracle's
    m = pm.Context(*grid, max_parcels=400000, precision="mixed")
    u = pm.Context(*grid, max_parcels=400000, precision="mixed")
    assert m.setup_plume(**REF_CFG) == n_plume
    u.upload(**{k: o.get(k) for k in IO})
    assert m.n == u.n
    for k in IO:
        np.testing.assert_array_equal(m.get(k), u.get(k), err_msg=k)
    for c in (g, m, u):
        c.close()


@pytest.mark.gpu
def test_device_plume_errors(pm):
    g = pm.Context(16, 16, 16, 6.28, 6.28, 6.28, max_parcels=1000)
    for bad in [dict(H=1.2), dict(mu=0.7), dict(r_plume=5.0)]:
        with pytest.raises(pm.PmpicError):
            g.setup_plume(**{**REF_CFG, **bad})
    with pytest.raises(pm.PmpicError):  # more parcels than max_parcels
        g.setup_plume(**REF_CFG)
    g.close()


@pytest.mark.gpu
def test_device_plume_then_steps_vs_oracle(pm):
    from oracle import Oracle
    grid = GRIDS[0]
    o = Oracle(*grid, dtm=0.02, dtmax=0.02, max_parcels=600000)
    g = pm.Context(*grid, dtm=0.02, dtmax=0.02, max_parcels=600000)
    o.setup_plume(**REF_CFG)
    g.setup_plume(**REF_CFG)
    o.step()
    g.step()
    assert g.n == o.n
    for k in ["x", "y", "z", "p", "q", "r"]:
        a, b = g.get(k), o.get(k)
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b))), k


def numpy_basic(nx, ny, nz, lx, ly, lz, s):
    """basic_parcelsetup.F90:91-115 on [0, lx) x [0, ly) x [0, lz] (one process),
    parcel t decoded as cell t // s^3 (x outer, z inner) and sub-lattice point
    t % s^3 (x outer), with x_coords(n) = -2 dx + (n - 1) dx + 0."""
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    t = np.arange(nx * ny * nz * s ** 3)
    cell, w = t // s ** 3, t % s ** 3
    i, j, k = cell // (ny * nz) + 3, (cell // nz) % ny + 3, cell % nz + 1
    ii, jj, kk = w // (s * s), (w // s) % s, w % s

    def coord(pmin, n, d):
        return pmin + (n - 1).astype(np.float64) * d + 0.0

    out = {}
    for key, pmin, d, idx, sub in [("x", -2.0 * dx, dx, i, ii), ("y", -2.0 * dy, dy, j, jj),
                                   ("z", 0.0 * dz + 0.0, dz, k, kk)]:
        c0 = coord(pmin, idx, d)
        step = (coord(pmin, idx + 1, d) - c0) / s
        out[key] = c0 + step / 2 + sub.astype(np.float64) * step
    out["vol"] = np.ones(len(t))
    return out


@pytest.mark.parametrize("s", [1, 2, 3])
def test_oracle_basic_vs_numpy(s):
    from oracle import Oracle, OracleError
    grid = (16, 12, 8, 2 * math.pi, 5.0, math.pi)
    want = numpy_basic(*grid, s)
    o = Oracle(*grid, max_parcels=len(want["x"]))
    o.setup_basic(s)
    assert o.n == len(want["x"])
    for k, v in want.items():
        np.testing.assert_array_equal(o.get(k), v, err_msg=k)
    for k in ["p", "q", "r", "b", "h", "stretch", "tag"]:
        assert np.all(o.get(k) == 0.0)
    with pytest.raises(OracleError):
        Oracle(*grid, max_parcels=len(want["x"]) - 1).setup_basic(s)


@pytest.mark.gpu
@pytest.mark.parametrize("s", [2, 3])
def test_device_basic_vs_oracle(pm, s):
    from oracle import Oracle
    grid = (16, 12, 8, 2 * math.pi, 5.0, math.pi)
    cap = 16 * 12 * 8 * s ** 3
    o = Oracle(*grid, max_parcels=cap)
    o.setup_basic(s)
    g = pm.Context(*grid, max_parcels=cap)
    g.setup_basic(s)
    assert g.n == o.n
    for k in IO:
        np.testing.assert_array_equal(g.get(k), o.get(k), err_msg=k)
    m = pm.Context(*grid, max_parcels=cap, precision="mixed")
    u = pm.Context(*grid, max_parcels=cap, precision="mixed")
    m.setup_basic(s)
    u.upload(**{k: o.get(k) for k in IO})
    for k in IO:
        np.testing.assert_array_equal(m.get(k), u.get(k), err_msg=k)
    with pytest.raises(pm.PmpicError):
        pm.Context(*grid, max_parcels=cap - 1).setup_basic(s)
    for c in (g, m, u):
        c.close()


THERMAL = dict(nx=24, ny=20, nz=12, lx=2 * math.pi, ly=5.0, lz=math.pi, seed=11)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_thermal_vs_host(pm, precision):
    host = pm.thermal_parcels(**THERMAL)
    n = len(host["x"])
    g = pm.Context(24, 20, 12, 2 * math.pi, 5.0, math.pi, max_parcels=n, precision=precision)
    u = pm.Context(24, 20, 12, 2 * math.pi, 5.0, math.pi, max_parcels=n, precision=precision)
    g.setup_thermal(**THERMAL)
    u.upload(**host)
    assert g.n == n
    for k in IO:
        a, b = g.get(k), u.get(k)
        if k == "b":  # the device cos against glibc's, inside the thermal
            np.testing.assert_allclose(a, b, rtol=1e-15 if precision == "fp64" else 1.2e-7, atol=1e-15)
        else:
            np.testing.assert_array_equal(a, b, err_msg=k)
    with pytest.raises(pm.PmpicError):
        pm.Context(24, 20, 12, 2 * math.pi, 5.0, math.pi, max_parcels=n - 1).setup_thermal(**THERMAL)
    g.close()
    u.close()
