"""pmpic_b200 -- B200 implementation of the PMPIC per-timestep hot path.

A ctypes binding of ``libpmpic_gpu.so`` (the C ABI in ``include/pmpic_gpu.h``).
The library is built in-tree by ``pmpic_b200/Makefile`` (nvcc, sm_100a).  There
is no CPU fallback: if the library or a CUDA device is missing, creating a
``Context`` raises.

The context mirrors the reference's component interface: one method per
timestep callback of the integrator group (``vort2vel``,
``vorticity_tendency``, ``rk4_integrator``, ``parcel_splitting``,
``parcel_mixing``), each advancing the component's own iteration counter
exactly like the Fortran modules' ``iteration`` / ``rkstep`` variables, and
``step(n)`` for whole model steps (the RK group run four times per step).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpmpic_gpu.so")

PROPS = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt",
         "h", "b", "vol", "stretch", "tag", "btot",
         "xo", "yo", "zo", "xf", "yf", "zf", "po", "qo", "ro", "pf", "qf", "rf"]
PROP = {n: i for i, n in enumerate(PROPS)}
GRIDS = ["u", "v", "w", "p", "q", "r", "b", "dp", "dq", "dr", "vol", "hg"]
GRID = {n: i for i, n in enumerate(GRIDS)}
SPECS = ["u_s", "v_s", "w_s"]
SPEC = {n: i for i, n in enumerate(SPECS)}
IO_PROPS = ["x", "y", "z", "p", "q", "r", "b", "h", "vol", "stretch", "tag"]
PRECISIONS = {"fp64": 0, "mixed": 1}

ERRORS = {0: "ok", -1: "config", -2: "capacity", -3: "out of box", -4: "zero pivot",
          -5: "backfill", -6: "timeout", -7: "cuda", -8: "argument", -9: "state", -10: "too large"}


class Config(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
                ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
                ("dtm", C.c_double), ("dtmax", C.c_double), ("timestep_prefactor", C.c_double),
                ("max_parcels", C.c_int64), ("precision", C.c_int32), ("device", C.c_int32)]


class StepInfo(C.Structure):
    _fields_ = [("n_parcels", C.c_int64), ("dtm", C.c_double), ("limiter", C.c_int32),
                ("n_split", C.c_int64), ("n_removed", C.c_int64), ("n_added", C.c_int64),
                ("n_migrated", C.c_int64), ("vol_sum", C.c_double), ("hvol_sum", C.c_double),
                ("bvol_sum", C.c_double), ("error", C.c_int32), ("message", C.c_char * 160)]


class ThermalParams(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("sub", C.c_int32), ("jitter", C.c_double), ("seed", C.c_uint64),
                ("xc", C.c_double), ("yc", C.c_double), ("zc", C.c_double),
                ("radius", C.c_double), ("excess", C.c_double),
                ("h_in", C.c_double), ("h_env0", C.c_double),
                ("z_strat", C.c_double), ("n2", C.c_double)]


class PlumeParams(C.Structure):
    _fields_ = [("lam", C.c_double), ("H", C.c_double), ("z_c", C.c_double), ("mu", C.c_double),
                ("z_d", C.c_double), ("z_m", C.c_double), ("r_plume", C.c_double),
                ("e_values", C.c_double * 3)]


def thermal_params(nx, ny, nz, lx=2 * np.pi, ly=2 * np.pi, lz=np.pi, sub=2, jitter=0.25, seed=1,
                   xc=np.pi, yc=np.pi, zc=0.6, radius=0.4, excess=1.0, h_in=0.95, h_env0=0.3,
                   z_strat=1.2, n2=1.0) -> ThermalParams:
    return ThermalParams(nx, ny, nz, lx, ly, lz, sub, jitter, seed, xc, yc, zc, radius, excess,
                         h_in, h_env0, z_strat, n2)


class PmpicError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pmpic error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def build() -> None:
    """Compile libpmpic_gpu.so in-tree for sm_100a."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run pmpic_b200.build() (no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        P, D, I64 = C.c_void_p, C.POINTER(C.c_double), C.c_int64
        L.pmpic_create.argtypes = [C.POINTER(Config), C.POINTER(P)]
        L.pmpic_destroy.argtypes = [P]
        L.pmpic_last_error.restype = C.c_char_p
        L.pmpic_last_error.argtypes = [P]
        L.pmpic_upload_parcels.argtypes = [P, I64] + [D] * 11
        L.pmpic_download_parcels.argtypes = [P, I64, C.POINTER(I64)] + [D] * 11
        L.pmpic_set_property.argtypes = [P, C.c_int, I64, D]
        L.pmpic_get_property.argtypes = [P, C.c_int, I64, D]
        L.pmpic_set_count.argtypes = [P, I64]
        L.pmpic_get_count.argtypes = [P, C.POINTER(I64)]
        for n in ["pmpic_vort2vel", "pmpic_vorticity_tendency", "pmpic_rk4_integrator",
                  "pmpic_parcel_splitting", "pmpic_parcel_mixing", "pmpic_op_parcel_haloswap",
                  "pmpic_euler_integrator", "pmpic_prescribed_velocity_tag"]:
            getattr(L, n).argtypes = [P]
        L.pmpic_step.argtypes = [P, C.c_int]
        L.pmpic_prescribed_velocity.argtypes = [P, C.c_int]
        L.pmpic_get_step_info.argtypes = [P, C.POINTER(StepInfo)]
        L.pmpic_conserved_sums.argtypes = [P, C.POINTER(C.c_double)]
        L.pmpic_get_counters.argtypes = [P, C.POINTER(C.c_int32)]
        L.pmpic_set_counters.argtypes = [P, C.POINTER(C.c_int32)]
        L.pmpic_set_dtm.argtypes = [P, C.c_double]
        L.pmpic_download_grid.argtypes = [P, C.c_int, D]
        L.pmpic_upload_grid.argtypes = [P, C.c_int, D]
        L.pmpic_download_spectral.argtypes = [P, C.c_int, D]
        L.pmpic_op_cell_ids.argtypes = [P, C.POINTER(C.c_int32)]
        L.pmpic_op_par2grid.argtypes = [P, C.c_int, C.c_int]
        L.pmpic_op_grid2par.argtypes = [P, C.c_int, C.c_int]
        L.pmpic_op_fft_forward.argtypes = [P, D, D]
        L.pmpic_op_fft_backward.argtypes = [P, D, D]
        L.pmpic_op_diffx.argtypes = [P, D, D]
        L.pmpic_op_diffy.argtypes = [P, D, D]
        L.pmpic_op_filter.argtypes = [P, D, D]
        L.pmpic_op_diffz.argtypes = [P, D, D, D, D]
        L.pmpic_op_laplinv.argtypes = [P, D, C.c_int]
        IP = C.POINTER(C.c_int)
        L.pmpic_op_par2grid_multi.argtypes = [P, C.c_int, IP, IP]
        L.pmpic_op_grid2par_multi.argtypes = [P, C.c_int, IP, IP]
        L.pmpic_op_vort2vel_grids.argtypes = [P]
        L.pmpic_sort_parcels.argtypes = [P]
        L.pmpic_write_parcels.argtypes = [P, C.c_char_p, C.c_double]
        L.pmpic_read_parcels.argtypes = [P, C.c_char_p, C.c_int, C.POINTER(C.c_double)]
        L.pmpic_write_grids.argtypes = [P, C.c_char_p, C.c_double]
        L.pmpic_write_grids_netcdf.argtypes = [P, C.c_char_p, C.c_double, C.c_int32]
        L.pmpic_write_parcels_netcdf.argtypes = [P, C.c_char_p, C.c_double, C.c_int32]
        L.pmpic_netcdf_write_grids.argtypes = [C.c_char_p] + [C.c_int32] * 3 + [C.c_double] * 4 + \
            [C.c_int32, C.c_double, C.POINTER(D)]
        L.pmpic_netcdf_write_parcels.argtypes = [C.c_char_p] + [C.c_int32] * 3 + [I64, C.c_double, C.c_int32,
                                                                                 C.c_double, C.POINTER(D)]
        L.pmpic_ensemble_create.argtypes = [C.c_int, C.POINTER(Config), C.POINTER(P)]
        L.pmpic_ensemble_destroy.argtypes = [P]
        L.pmpic_ensemble_member.restype = P
        L.pmpic_ensemble_member.argtypes = [P, C.c_int]
        L.pmpic_ensemble_set_concurrency.argtypes = [P, C.c_int]
        L.pmpic_ensemble_autotune.argtypes = [P]
        L.pmpic_ensemble_step.argtypes = [P, C.c_int, C.POINTER(C.c_float)]
        L.pmpic_ensemble_tuning.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int32)]
        L.pmpic_set_p2g_segment.argtypes = [P, C.c_int]
        L.pmpic_timing.argtypes = [P, C.c_int]
        L.pmpic_timer_count.argtypes = []
        L.pmpic_timer_name.restype = C.c_char_p
        L.pmpic_timer_name.argtypes = [C.c_int]
        L.pmpic_timer_read.argtypes = [P, C.c_int, C.POINTER(C.c_double), C.POINTER(I64)]
        L.pmpic_launch_count.argtypes = [P, C.POINTER(I64)]
        L.pmpic_event_record.argtypes = [P, C.c_int]
        L.pmpic_event_elapsed.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.pmpic_pin_host.argtypes = [C.c_void_p, C.c_size_t]
        L.pmpic_unpin_host.argtypes = [C.c_void_p]
        # device pointers as plain integers (e.g. torch data_ptr()), stream as a handle
        L.pmpic_par2grid_static.argtypes = [C.c_int32] * 3 + [C.c_double] * 3 + [I64] + [C.c_void_p] * 7
        L.pmpic_setup_count.restype = I64
        L.pmpic_setup_count.argtypes = [C.POINTER(ThermalParams)]
        L.pmpic_setup_thermal.argtypes = [C.POINTER(ThermalParams), I64] + [D] * 11
        L.pmpic_setup_thermal_device.argtypes = [P, C.POINTER(ThermalParams)]
        L.pmpic_setup_plume.argtypes = [P, C.POINTER(PlumeParams), C.POINTER(I64)]
        L.pmpic_setup_basic.argtypes = [P, C.c_int32]
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def thermal_parcels(nx, ny, nz, lx=2 * np.pi, ly=2 * np.pi, lz=np.pi, sub=2, jitter=0.25, seed=1,
                    xc=np.pi, yc=np.pi, zc=0.6, radius=0.4, excess=1.0, h_in=0.95, h_env0=0.3,
                    z_strat=1.2, n2=1.0) -> dict:
    """Jittered-lattice thermal plume initial condition (host, Philox4x32-10)."""
    prm = thermal_params(nx, ny, nz, lx, ly, lz, sub, jitter, seed, xc, yc, zc, radius, excess,
                         h_in, h_env0, z_strat, n2)
    n = lib().pmpic_setup_count(C.byref(prm))
    out = {k: np.empty(n, np.float64) for k in IO_PROPS}
    rc = lib().pmpic_setup_thermal(C.byref(prm), n, *[_dp(out[k]) for k in IO_PROPS])
    if rc:
        raise PmpicError(rc, "pmpic_setup_thermal")
    return out


NETCDF_GRID_FIELDS = ["u", "v", "w", "p", "q", "r", "b", "hg", "hgliq", "vol"]
NETCDF_PARCEL_PROPS = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt",
                       "h", "b", "vol", "stretch", "tag"]


def netcdf_write_grids(path, nx, ny, nz, lx, ly, lz, fields, time=0.0, timestep=0, dtm=0.0):
    """The NetCDF grid file from host arrays: fields[name] of (nz+1)*ny*nx values, z fastest."""
    arrs = [np.ascontiguousarray(fields[k], dtype=np.float64).ravel() for k in NETCDF_GRID_FIELDS]
    if any(a.size != (nz + 1) * ny * nx for a in arrs):
        raise ValueError("each field needs (nz+1)*ny*nx values")
    ptrs = (C.POINTER(C.c_double) * 10)(*[_dp(a) for a in arrs])
    rc = lib().pmpic_netcdf_write_grids(os.fsencode(path), nx, ny, nz, lx, ly, lz, time, timestep, dtm, ptrs)
    if rc:
        raise PmpicError(rc, "pmpic_netcdf_write_grids")


def netcdf_write_parcels(path, nx, ny, nz, props, time=0.0, timestep=0, dtm=0.0):
    """The NetCDF parcel file from host arrays: props[name] for the 17 dumped properties."""
    arrs = [np.ascontiguousarray(props[k], dtype=np.float64) for k in NETCDF_PARCEL_PROPS]
    n = len(arrs[0])
    if any(len(a) != n for a in arrs):
        raise ValueError("all properties need the same length")
    ptrs = (C.POINTER(C.c_double) * 17)(*[_dp(a) for a in arrs])
    rc = lib().pmpic_netcdf_write_parcels(os.fsencode(path), nx, ny, nz, n, time, timestep, dtm, ptrs)
    if rc:
        raise PmpicError(rc, "pmpic_netcdf_write_parcels")


def random_vorticity(nx, ny, nz, lx=2 * np.pi, ly=2 * np.pi, lz=np.pi, kmax=64, seed=4, rms=1.0):
    """Divergence-free random vorticity on the (nz+1) x ny x nx grid (host set-up,
    not on the hot path): omega = curl B with B_x, B_y ~ cos(kz z) and B_z ~ sin(kz z),
    so omega_x, omega_y ~ sin(kz z) vanish at the walls z = 0, lz (free slip) and
    omega_z ~ cos(kz z).  Mode amplitudes N(0, 1) * |k|^(-11/6) for 0 < |k| <= kmax
    give an isotropic k^(-5/3) energy spectrum; the result is scaled to the given
    RMS over the grid.  Returns (p, q, r) = (omega_x, omega_y, omega_z)."""
    rng = np.random.default_rng(seed)
    a = np.fft.rfftfreq(nx, 1.0 / nx)               # x mode numbers 0..nx/2
    b = np.fft.fftfreq(ny, 1.0 / ny)                # y mode numbers
    mmax = int(min(kmax * lz / np.pi, nz))
    m = np.arange(mmax + 1)
    kx = (2 * np.pi / lx) * a[None, None, :]
    ky = (2 * np.pi / ly) * b[None, :, None]
    kz = (np.pi / lz) * m[:, None, None]
    kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    amp = np.where((kk > 0) & (kk <= kmax), np.power(np.where(kk > 0, kk, 1.0), -11.0 / 6.0), 0.0)
    shape = amp.shape

    def coef():
        return amp * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    cx, cy, cz = coef(), coef(), coef()
    # spectral coefficients of the vorticity per (m, ky, kx): curl of B
    wx = 1j * ky * cz + kz * cy      # times sin(kz z)
    wy = -kz * cx - 1j * kx * cz     # times sin(kz z)
    wz = 1j * kx * cy - 1j * ky * cx  # times cos(kz z)
    zk = np.arange(nz + 1) * (lz / nz)
    sin_t = np.sin(np.outer(zk, (np.pi / lz) * m))   # (nz+1, M)
    cos_t = np.cos(np.outer(zk, (np.pi / lz) * m))

    def synth(w, basis):
        planes = np.fft.irfft2(w, s=(ny, nx), axes=(1, 2)) * (nx * ny)  # (M, ny, nx)
        return (basis @ planes.reshape(len(m), -1)).reshape(nz + 1, ny, nx)
    p, q, r = synth(wx, sin_t), synth(wy, sin_t), synth(wz, cos_t)
    scale = rms / np.sqrt((p ** 2 + q ** 2 + r ** 2).mean() / 3.0)
    return p * scale, q * scale, r * scale


class Context:
    """One device-resident model state (the reference's model_state_type)."""

    def __init__(self, nx, ny, nz, lx, ly, lz, dtm=0.01, dtmax=0.01, prefactor=0.5,
                 max_parcels=1 << 20, device=0, precision="fp64"):
        """precision: "fp64" (the plain path) or "mixed" (FP32 fields, grids,
        transforms and RK4; positions as integer cell index + FP32 offset; FP64
        zero mode).  Transfers are FP64 on the host either way."""
        L = lib()
        self.nx, self.ny, self.nz = nx, ny, nz
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.precision = precision
        cfg = Config(nx, ny, nz, 0.0, lx, 0.0, ly, 0.0, lz, dtm, dtmax, prefactor,
                     int(max_parcels), PRECISIONS[precision], device)
        h = C.c_void_p()
        rc = L.pmpic_create(C.byref(cfg), C.byref(h))
        if rc:
            raise PmpicError(rc, "pmpic_create failed")
        self._h = h
        self.max_parcels = int(max_parcels)

    @classmethod
    def _member(cls, handle, nx, ny, nz, precision, max_parcels):
        """A view of an ensemble member's context (owned by the ensemble)."""
        self = cls.__new__(cls)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.precision = precision
        self.max_parcels = int(max_parcels)
        self._h = handle
        self._owned = False
        return self

    def close(self):
        if getattr(self, "_h", None) and getattr(self, "_owned", True):
            lib().pmpic_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise PmpicError(rc, lib().pmpic_last_error(self._h).decode())

    # -- parcels -----------------------------------------------------------------
    @property
    def n(self) -> int:
        v = C.c_int64()
        self._check(lib().pmpic_get_count(self._h, C.byref(v)))
        return int(v.value)

    def upload(self, **arrays):
        n = len(arrays["x"])
        ptrs = []
        keep = []
        for k in IO_PROPS:
            a = arrays.get(k)
            if a is not None:
                a = np.ascontiguousarray(a, np.float64)
                assert len(a) == n
                keep.append(a)
            ptrs.append(_dp(a))
        self._check(lib().pmpic_upload_parcels(self._h, n, *ptrs))

    def download(self) -> dict:
        n = self.n
        out = {k: np.empty(n, np.float64) for k in IO_PROPS}
        cnt = C.c_int64()
        self._check(lib().pmpic_download_parcels(self._h, n, C.byref(cnt),
                                                 *[_dp(out[k]) for k in IO_PROPS]))
        return out

    def set(self, name, arr, n=None):
        a = np.ascontiguousarray(arr, np.float64)
        self._check(lib().pmpic_set_property(self._h, PROP[name], len(a) if n is None else n, _dp(a)))

    def get(self, name, n=None) -> np.ndarray:
        n = self.n if n is None else n
        out = np.empty(n, np.float64)
        self._check(lib().pmpic_get_property(self._h, PROP[name], n, _dp(out)))
        return out

    def set_count(self, n):
        self._check(lib().pmpic_set_count(self._h, int(n)))

    def grid(self, name) -> np.ndarray:
        out = np.empty((self.nz + 1, self.ny, self.nx), np.float64)
        self._check(lib().pmpic_download_grid(self._h, GRID[name], _dp(out)))
        return out

    def set_grid(self, name, g):
        g = np.ascontiguousarray(g, np.float64)
        assert g.shape == (self.nz + 1, self.ny, self.nx)
        self._check(lib().pmpic_upload_grid(self._h, GRID[name], _dp(g)))

    def spec(self, name) -> np.ndarray:
        out = np.empty((self.nz + 1, self.ny + 2, self.nx + 2), np.float64)
        self._check(lib().pmpic_download_spectral(self._h, SPEC[name], _dp(out)))
        return out

    def info(self) -> StepInfo:
        s = StepInfo()
        self._check(lib().pmpic_get_step_info(self._h, C.byref(s)))
        return s

    def conserved_sums(self):
        """(sum vol, sum h vol, sum b vol) over the parcels now, compensated FP64."""
        out = (C.c_double * 3)()
        self._check(lib().pmpic_conserved_sums(self._h, out))
        return tuple(out)

    def counters(self):
        a = (C.c_int32 * 5)()
        self._check(lib().pmpic_get_counters(self._h, a))
        return list(a)

    def set_counters(self, v):
        a = (C.c_int32 * 5)(*v)
        self._check(lib().pmpic_set_counters(self._h, a))

    def set_dtm(self, dtm):
        self._check(lib().pmpic_set_dtm(self._h, float(dtm)))

    # -- components -----------------------------------------------------------------
    def vort2vel(self):
        self._check(lib().pmpic_vort2vel(self._h))

    def vorticity_tendency(self):
        self._check(lib().pmpic_vorticity_tendency(self._h))

    def rk4_integrator(self):
        self._check(lib().pmpic_rk4_integrator(self._h))

    # the reference's test components for the migration path (FP64 contexts)
    def euler_integrator(self):
        self._check(lib().pmpic_euler_integrator(self._h))

    def prescribed_velocity(self, profile):
        self._check(lib().pmpic_prescribed_velocity(self._h, int(profile)))

    def prescribed_velocity_tag(self):
        self._check(lib().pmpic_prescribed_velocity_tag(self._h))

    # -- set-up components written on the device ---------------------------------
    def setup_plume(self, lam=1.0, H=0.8, z_c=2.5, mu=0.9, z_d=4.0, z_m=5.0, r_plume=0.8,
                    e_values=(0.3, -0.4, 0.5)) -> int:
        """plume_parcelsetup (the reference's defaults in its config); replaces the
        parcels and returns the number of plume parcels (the first slots)."""
        prm = PlumeParams(lam, H, z_c, mu, z_d, z_m, r_plume, (C.c_double * 3)(*e_values))
        n_plume = C.c_int64(0)
        self._check(lib().pmpic_setup_plume(self._h, C.byref(prm), C.byref(n_plume)))
        return n_plume.value

    def setup_basic(self, parcels_per_cell_dir=2):
        """basic_parcelsetup: a regular sub-lattice of parcels_per_cell_dir^3 parcels
        per cell, vol = 1, written on the device."""
        self._check(lib().pmpic_setup_basic(self._h, int(parcels_per_cell_dir)))

    def setup_thermal(self, **kw):
        """The jittered thermal of thermal_parcels(**kw), written on the device."""
        prm = thermal_params(**kw)
        self._check(lib().pmpic_setup_thermal_device(self._h, C.byref(prm)))

    def parcel_splitting(self):
        self._check(lib().pmpic_parcel_splitting(self._h))

    def parcel_mixing(self):
        self._check(lib().pmpic_parcel_mixing(self._h))

    def step(self, nsteps=1):
        self._check(lib().pmpic_step(self._h, int(nsteps)))

    # -- model-core routines --------------------------------------------------------
    def cell_ids(self) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        self._check(lib().pmpic_op_cell_ids(self._h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def par2grid(self, prop, grid):
        self._check(lib().pmpic_op_par2grid(self._h, PROP[prop], GRID[grid]))

    def grid2par(self, grid, prop):
        self._check(lib().pmpic_op_grid2par(self._h, GRID[grid], PROP[prop]))

    def par2grid_multi(self, props, grids):
        """par2grid of 1, 3 or 4 properties into as many grids, one set of weights."""
        a = (C.c_int * len(props))(*[PROP[p] for p in props])
        b = (C.c_int * len(grids))(*[GRID[g] for g in grids])
        self._check(lib().pmpic_op_par2grid_multi(self._h, len(props), a, b))

    def grid2par_multi(self, grids, props):
        """grid2par of 1, 3 or 6 grids into as many properties."""
        a = (C.c_int * len(grids))(*[GRID[g] for g in grids])
        b = (C.c_int * len(props))(*[PROP[p] for p in props])
        self._check(lib().pmpic_op_grid2par_multi(self._h, len(grids), a, b))

    def vort2vel_grids(self):
        """vort2vel's inversion alone on the vorticity in grids p, q, r."""
        self._check(lib().pmpic_op_vort2vel_grids(self._h))

    def write_parcels(self, path, time=0.0):
        """Parcel dump in the reference's binary format (writebinary.F90)."""
        self._check(lib().pmpic_write_parcels(self._h, os.fsencode(path), float(time)))

    def read_parcels(self, path, append=False) -> float:
        """Restart from a parcel dump; returns the dump's time."""
        t = C.c_double()
        self._check(lib().pmpic_read_parcels(self._h, os.fsencode(path), 1 if append else 0, C.byref(t)))
        return float(t.value)

    def write_grids(self, path, time=0.0):
        """Grid dump in the reference's binary format (writebinary.F90)."""
        self._check(lib().pmpic_write_grids(self._h, os.fsencode(path), float(time)))

    def write_grids_netcdf(self, path, time=0.0, timestep=0):
        """NetCDF grid file of writenetcdf.F90:225-308 (classic 64-bit-offset format)."""
        self._check(lib().pmpic_write_grids_netcdf(self._h, os.fsencode(path), float(time), int(timestep)))

    def write_parcels_netcdf(self, path, time=0.0, timestep=0):
        """NetCDF parcel file of writenetcdf.F90:310-439 (classic 64-bit-offset format)."""
        self._check(lib().pmpic_write_parcels_netcdf(self._h, os.fsencode(path), float(time), int(timestep)))

    def sort_parcels(self):
        """Renumber slots into cell order (not a reference operation)."""
        self._check(lib().pmpic_sort_parcels(self._h))

    def parcel_haloswap(self):
        self._check(lib().pmpic_op_parcel_haloswap(self._h))

    def _sshape(self):
        return (self.nz + 1, self.ny + 2, self.nx + 2)

    def fft_forward(self, phys):
        phys = np.ascontiguousarray(phys, np.float64)
        out = np.empty(self._sshape())
        self._check(lib().pmpic_op_fft_forward(self._h, _dp(phys), _dp(out)))
        return out

    def fft_backward(self, spec):
        spec = np.ascontiguousarray(spec, np.float64)
        out = np.empty((self.nz + 1, self.ny, self.nx))
        self._check(lib().pmpic_op_fft_backward(self._h, _dp(spec), _dp(out)))
        return out

    def _unary(self, fn, a):
        a = np.ascontiguousarray(a, np.float64)
        out = np.empty_like(a)
        self._check(fn(self._h, _dp(a), _dp(out)))
        return out

    def diffx(self, a):
        return self._unary(lib().pmpic_op_diffx, a)

    def diffy(self, a):
        return self._unary(lib().pmpic_op_diffy, a)

    def filter(self, a):
        return self._unary(lib().pmpic_op_filter, a)

    def diffz(self, a, bot=None, top=None):
        a = np.ascontiguousarray(a, np.float64)
        out = np.empty_like(a)
        if bot is None:
            self._check(lib().pmpic_op_diffz(self._h, _dp(a), _dp(out), None, None))
        else:
            bot = np.ascontiguousarray(bot, np.float64)
            top = np.ascontiguousarray(top, np.float64)
            self._check(lib().pmpic_op_diffz(self._h, _dp(a), _dp(out), _dp(bot), _dp(top)))
        return out

    def laplinv(self, a, df_zero_on_boundary: bool):
        a = np.array(a, np.float64, copy=True, order="C")
        self._check(lib().pmpic_op_laplinv(self._h, _dp(a), 1 if df_zero_on_boundary else 0))
        return a


DUMP_PROPS = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt",
              "h", "b", "vol", "stretch", "tag"]
DUMP_GRIDS = ["u", "v", "w", "p", "q", "r", "b", "hg", "hgliq", "vol"]


def read_parcel_dump(path) -> dict:
    """Reads a parcel dump of the reference's format (writebinary.F90:149-199)."""
    with open(path, "rb") as f:
        hdr = np.fromfile(f, np.float64, 7)
        n = int(np.fromfile(f, np.int64, 1)[0])
        data = np.fromfile(f, np.float64, 17 * n).reshape(17, n)
    out = {k: data[i] for i, k in enumerate(DUMP_PROPS)}
    out["time"], out["bounds"], out["n"] = float(hdr[0]), hdr[1:], n
    return out


def read_grid_dump(path) -> dict:
    """Reads a grid dump of the reference's format (writebinary.F90:201-299);
    grids are returned as (nz+1, ny, nx) arrays, x fastest."""
    with open(path, "rb") as f:
        hdr = np.fromfile(f, np.float64, 7)
        nx, ny, nzp = (int(v) for v in np.fromfile(f, np.int32, 3))
        data = np.fromfile(f, np.float64, 10 * nx * ny * nzp).reshape(10, nx, ny, nzp)
    out = {k: np.ascontiguousarray(data[i].transpose(2, 1, 0)) for i, k in enumerate(DUMP_GRIDS)}
    out["time"], out["bounds"], out["sizes"] = float(hdr[0]), hdr[1:], (nx, ny, nzp)
    return out


def assign_members(costs, ranks):
    """Spreads ensemble members over `ranks` GPUs (one process each) by their
    estimated cost (parcels x steps): largest first, each to the least-loaded
    rank (ties to the lower rank), so that the ranks' loads differ by at most
    one member's cost.  Members are independent: no exchange between ranks.
    Returns per rank the member indices, ascending."""
    if ranks < 1:
        raise ValueError("ranks must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * ranks
    out = [[] for _ in range(ranks)]
    for i in order:
        r = min(range(ranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


class Ensemble:
    """Independent plumes of uneven sizes on one GPU, stepped concurrently
    (pmpic_ensemble_*; no counterpart in the reference).  members: a list of
    dicts with nx, ny, nz and optionally lx, ly, lz, dtm, dtmax, max_parcels,
    precision."""

    def __init__(self, members, device=0):
        L = lib()
        cfgs = (Config * len(members))()
        self._meta = []
        for i, m in enumerate(members):
            prec = m.get("precision", "fp64")
            dt = m.get("dtm", 0.01)
            cfgs[i] = Config(m["nx"], m["ny"], m["nz"], 0.0, m.get("lx", 2 * np.pi), 0.0, m.get("ly", 2 * np.pi),
                             0.0, m.get("lz", np.pi), dt, m.get("dtmax", dt), m.get("prefactor", 0.5),
                             int(m["max_parcels"]), PRECISIONS[prec], device)
            self._meta.append((m["nx"], m["ny"], m["nz"], prec, m["max_parcels"]))
        h = C.c_void_p()
        rc = L.pmpic_ensemble_create(len(members), cfgs, C.byref(h))
        if rc:
            raise PmpicError(rc, "pmpic_ensemble_create failed")
        self._h = h
        self.members = [Context._member(L.pmpic_ensemble_member(h, i), *self._meta[i])
                        for i in range(len(members))]

    def set_concurrency(self, threads):
        self._check(lib().pmpic_ensemble_set_concurrency(self._h, int(threads)))

    def autotune(self):
        self._check(lib().pmpic_ensemble_autotune(self._h))

    def step(self, nsteps=1) -> float:
        """Advance every member; returns the device time in ms."""
        ms = C.c_float()
        self._check(lib().pmpic_ensemble_step(self._h, int(nsteps), C.byref(ms)))
        return float(ms.value)

    def tuning(self):
        t = C.c_int()
        x = (C.c_int32 * len(self.members))()
        self._check(lib().pmpic_ensemble_tuning(self._h, C.byref(t), x))
        return int(t.value), list(x)

    def _check(self, rc):
        if rc:
            raise PmpicError(rc, "ensemble call failed")

    def close(self):
        if getattr(self, "_h", None):
            for m in self.members:
                m._h = None
            lib().pmpic_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
