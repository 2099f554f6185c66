"""NetCDF files of writenetcdf.F90 (write_ncgrid_file :225-308,
write_parcels_to_file :310-439), written in the classic 64-bit-offset format
and read back with scipy's independent NetCDF-3 reader: dimensions, variable
names, shapes and attributes of the reference's schema, and every value bit for
bit.  CPU: the host-array writers.  GPU: the context writers against the
binary dumps and the context's own parcel state.
"""
import math

import numpy as np
import pytest

scipy_netcdf = pytest.importorskip("scipy.io").netcdf_file

GRID_FIELDS = ["u", "v", "w", "p", "q", "r", "b", "hg", "hgliq", "vol"]
PARCEL_VARS = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt",
               "h", "b", "vol", "stetch", "tag"]
PROPS = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt",
         "h", "b", "vol", "stretch", "tag"]


def _read(path):
    f = scipy_netcdf(str(path), "r", mmap=False)
    return f, {k: v.data.copy() for k, v in f.variables.items()}


def check_grid_file(path, nx, ny, nz, lx, ly, lz, fields, time, timestep, dtm):
    f, v = _read(path)
    assert f.version_byte == 2
    assert f.dimensions == {"time": 1, "z": nz + 1, "y": ny, "x": nx}
    assert list(f.variables) == ["time", "z", "y", "x"] + GRID_FIELDS + ["timestep", "dtm"]
    assert f.title == b"MONC checkpoint file" and len(f.created) > 0
    for k in ["time", "z", "y", "x"] + GRID_FIELDS:
        assert f.variables[k].units == b"-", k
    assert f.variables["dtm"]._attributes == {} and f.variables["timestep"]._attributes == {}
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    np.testing.assert_array_equal(v["z"], dz * (np.arange(1, nz + 2, dtype=np.float32) - np.float32(1.0)).astype(np.float64))
    np.testing.assert_array_equal(v["y"], dy * (np.arange(1, ny + 1, dtype=np.float32) - np.float32(0.5)).astype(np.float64))
    np.testing.assert_array_equal(v["x"], dx * (np.arange(1, nx + 1, dtype=np.float32) - np.float32(0.5)).astype(np.float64))
    assert v["time"].tolist() == [time] and int(v["timestep"]) == timestep and float(v["dtm"]) == dtm
    for k in GRID_FIELDS:
        assert f.variables[k].dimensions == ("time", "x", "y", "z")
        np.testing.assert_array_equal(v[k][0], np.asarray(fields[k]).reshape(nx, ny, nz + 1), err_msg=k)
    f.close()


def check_parcel_file(path, nx, ny, nz, props, time, timestep, dtm):
    f, v = _read(path)
    n = len(props["x"])
    assert f.version_byte == 2
    assert f.dimensions == {"time": 1, "nparcel": None}  # nparcel is the unlimited dimension
    assert list(f.variables) == (["time", "parcel"] + PARCEL_VARS +
                                 ["x_start", "y_start", "z_start", "x_end", "y_end", "z_end", "timestep", "dtm"])
    np.testing.assert_array_equal(v["parcel"], np.arange(1, n + 1, dtype=np.float64))
    for var, prop in zip(PARCEL_VARS, PROPS):
        assert f.variables[var].dimensions == ("nparcel",)
        np.testing.assert_array_equal(v[var], props[prop], err_msg=var)
    bounds = [float(v[k]) for k in ["x_start", "y_start", "z_start", "x_end", "y_end", "z_end"]]
    assert bounds == [3.0, 3.0, 1.0, nx + 3.0, ny + 3.0, nz + 1.0]
    assert v["time"].tolist() == [time] and int(v["timestep"]) == timestep and float(v["dtm"]) == dtm
    f.close()


def test_grid_file_from_host_arrays(tmp_path):
    import pmpic_b200 as pm
    nx, ny, nz, lx, ly, lz = 12, 10, 8, 2 * math.pi, 5.0, math.pi
    rng = np.random.default_rng(3)
    fields = {k: rng.standard_normal((nz + 1) * ny * nx) for k in GRID_FIELDS}
    path = tmp_path / "grids_0007.nc"
    pm.netcdf_write_grids(path, nx, ny, nz, lx, ly, lz, fields, time=1.25, timestep=7, dtm=0.01)
    check_grid_file(path, nx, ny, nz, lx, ly, lz, fields, 1.25, 7, 0.01)


@pytest.mark.parametrize("n", [0, 1, 270001])  # one record; records across the writer's 2^18-record slabs
def test_parcel_file_from_host_arrays(tmp_path, n):
    import pmpic_b200 as pm
    rng = np.random.default_rng(n)
    props = {k: rng.standard_normal(n) for k in PROPS}
    path = tmp_path / "parcels_00000_0003.nc"
    pm.netcdf_write_parcels(path, 16, 12, 8, props, time=0.5, timestep=3, dtm=0.02)
    check_parcel_file(path, 16, 12, 8, props, 0.5, 3, 0.02)


def test_variable_beyond_the_format_limit_is_refused(tmp_path):
    # 1025 x 1024 x 1024 FP64 values per field exceed the 4 GiB a classic
    # 64-bit-offset variable may hold; the header check refuses the file before
    # any field value is read, so one-value arrays stand in for the fields
    import ctypes as C
    import pmpic_b200 as pm
    one = [np.zeros(1) for _ in range(10)]
    ptrs = (C.POINTER(C.c_double) * 10)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in one])
    rc = pm.lib().pmpic_netcdf_write_grids(str(tmp_path / "big.nc").encode(), 1024, 1024, 1024, 1.0, 1.0, 1.0,
                                           0.0, 0, 0.0, ptrs)
    assert rc != 0
    assert not (tmp_path / "big.nc").exists()


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_context_netcdf_files_match_the_dumps(pm, tmp_path, precision):
    nx, ny, nz = 16, 12, 8
    ic = pm.thermal_parcels(nx, ny, nz, seed=5)
    g = pm.Context(nx, ny, nz, 2 * math.pi, 2 * math.pi, math.pi, max_parcels=2 * len(ic["x"]), precision=precision)
    g.upload(**ic)
    g.step()
    g.write_grids(tmp_path / "grids.dat", time=0.75)
    g.write_grids_netcdf(tmp_path / "grids.nc", time=0.75, timestep=1)
    raw = np.fromfile(tmp_path / "grids.dat", dtype=np.uint8)
    vals = raw[7 * 8 + 3 * 4:].view(np.float64).reshape(10, -1)
    fields = dict(zip(GRID_FIELDS, vals))
    check_grid_file(tmp_path / "grids.nc", nx, ny, nz, 2 * math.pi, 2 * math.pi, math.pi, fields, 0.75, 1,
                    g.info().dtm)
    g.write_parcels_netcdf(tmp_path / "parcels.nc", time=0.75, timestep=1)
    check_parcel_file(tmp_path / "parcels.nc", nx, ny, nz, {k: g.get(k) for k in PROPS}, 0.75, 1, g.info().dtm)
    g.close()
