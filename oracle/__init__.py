"""CPU oracle for the PMPIC hot path -- TEST INFRASTRUCTURE ONLY.

A ctypes binding of ``oracle/liboracle.so`` (built from ``pmpic_oracle.cpp`` by
``oracle/Makefile``), the C++ restatement of the reference Fortran hot path.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
``--impl reference`` legs may import this package; it is the checker, never the
thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

# property / grid / spectral ids (same numbering as include/pmpic_gpu.h)
PROPS = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt",
         "h", "b", "vol", "stretch", "tag", "btot",
         "xo", "yo", "zo", "xf", "yf", "zf", "po", "qo", "ro", "pf", "qf", "rf"]
PROP = {n: i for i, n in enumerate(PROPS)}
GRIDS = ["u", "v", "w", "p", "q", "r", "b", "dp", "dq", "dr", "vol", "hg"]
GRID = {n: i for i, n in enumerate(GRIDS)}
SPECS = ["u_s", "v_s", "w_s"]
SPEC = {n: i for i, n in enumerate(SPECS)}


class StepInfo(C.Structure):
    _fields_ = [("n_parcels", C.c_int64), ("dtm", C.c_double), ("limiter", C.c_int),
                ("n_split", C.c_int64), ("n_removed", C.c_int64), ("n_added", C.c_int64),
                ("n_migrated", C.c_int64), ("error", C.c_int), ("message", C.c_char * 160)]


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int] * 3 + [C.c_double] * 9 + [C.c_int64]
        L.orc_destroy.argtypes = [P]
        L.orc_error.argtypes = [P, C.c_char_p, C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_count.argtypes = [P, C.c_int64]
        L.orc_count.restype = C.c_int64
        L.orc_count.argtypes = [P]
        L.orc_set_prop.argtypes = [P, C.c_int, D, C.c_int64]
        L.orc_get_prop.argtypes = [P, C.c_int, D, C.c_int64]
        L.orc_get_grid.argtypes = [P, C.c_int, D]
        L.orc_set_grid.argtypes = [P, C.c_int, D]
        L.orc_get_spec.argtypes = [P, C.c_int, D]
        L.orc_get_step_info.argtypes = [P, C.POINTER(StepInfo)]
        L.orc_cache_weights.argtypes = [P, C.POINTER(C.c_int32)]
        L.orc_par2grid.argtypes = [P, C.c_int, C.c_int]
        L.orc_grid2par.argtypes = [P, C.c_int, C.c_int]
        L.orc_fft_forward.argtypes = [P, D, D]
        L.orc_fft_backward.argtypes = [P, D, D]
        L.orc_diffx.argtypes = [P, D, D]
        L.orc_diffy.argtypes = [P, D, D]
        L.orc_diffz.argtypes = [P, D, D, D, D]
        L.orc_laplinv.argtypes = [P, D, C.c_int]
        L.orc_filter.argtypes = [P, D, D]
        L.orc_kx_ky_k2.argtypes = [P, D, D, D, D]
        L.orc_prescribed_velocity.argtypes = [P, C.c_int]
        L.orc_plume_setup.argtypes = [P, D, C.POINTER(C.c_int64)]
        L.orc_basic_setup.argtypes = [P, C.c_int]
        L.orc_thermal_setup.argtypes = [P, D, C.c_uint64]
        L.orc_conserved_sums.argtypes = [P, D]
        for n in ["orc_parcel_haloswap", "orc_vort2vel", "orc_vort2vel_grids", "orc_vorticity_tendency",
                  "orc_rk4_integrator", "orc_parcel_splitting", "orc_parcel_mixing", "orc_step",
                  "orc_euler_integrator", "orc_prescribed_velocity_tag"]:
            getattr(L, n).argtypes = [P]
        L.orc_get_counters.argtypes = [P, C.POINTER(C.c_int)]
        L.orc_set_counters.argtypes = [P, C.POINTER(C.c_int)]
        L.orc_set_dtm.argtypes = [P, C.c_double]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleError(RuntimeError):
    pass


class Oracle:
    """One single-rank reference state (model_state_type + module save state)."""

    def __init__(self, nx, ny, nz, lx, ly, lz, dtm=0.01, dtmax=0.01, prefactor=0.5,
                 max_parcels=1 << 20, threads: int | None = None):
        L = lib()
        if threads is not None:
            L.orc_set_threads(int(threads))
        self.nx, self.ny, self.nz = nx, ny, nz
        self._h = L.orc_create(nx, ny, nz, 0.0, lx, 0.0, ly, 0.0, lz, dtm, dtmax, prefactor,
                               int(max_parcels))
        if not self._h:
            raise OracleError("orc_create rejected the configuration")
        self.max_parcels = int(max_parcels)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- errors ---------------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            buf = C.create_string_buffer(256)
            lib().orc_error(self._h, buf, 256)
            raise OracleError(f"oracle error {rc}: {buf.value.decode()}")

    # -- parcels --------------------------------------------------------------
    @property
    def n(self) -> int:
        return int(lib().orc_count(self._h))

    def set_parcels(self, **arrays):
        n = None
        for k, v in arrays.items():
            v = np.ascontiguousarray(v, dtype=np.float64)
            n = len(v) if n is None else n
            assert len(v) == n
            self._check(lib().orc_set_prop(self._h, PROP[k], _dp(v), n))
        self._check(lib().orc_set_count(self._h, n))

    def set_count(self, n):
        self._check(lib().orc_set_count(self._h, int(n)))

    def get(self, name, n=None) -> np.ndarray:
        n = self.n if n is None else n
        out = np.empty(n, np.float64)
        self._check(lib().orc_get_prop(self._h, PROP[name], _dp(out), n))
        return out

    def grid(self, name) -> np.ndarray:
        out = np.empty((self.nz + 1, self.ny, self.nx), np.float64)
        self._check(lib().orc_get_grid(self._h, GRID[name], _dp(out)))
        return out

    def set_grid(self, name, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        assert g.shape == (self.nz + 1, self.ny, self.nx)
        self._check(lib().orc_set_grid(self._h, GRID[name], _dp(g)))

    def spec(self, name) -> np.ndarray:
        out = np.empty((self.nz + 1, self.ny + 2, self.nx + 2), np.float64)
        self._check(lib().orc_get_spec(self._h, SPEC[name], _dp(out)))
        return out

    def info(self) -> StepInfo:
        s = StepInfo()
        lib().orc_get_step_info(self._h, C.byref(s))
        return s

    def conserved_sums(self):
        """(sum vol, sum h vol, sum b vol) over the parcels, compensated FP64."""
        out = np.zeros(3)
        self._check(lib().orc_conserved_sums(self._h, _dp(out)))
        return tuple(float(v) for v in out)

    def counters(self):
        a = (C.c_int * 5)()
        lib().orc_get_counters(self._h, a)
        return list(a)

    def set_counters(self, v):
        a = (C.c_int * 5)(*v)
        lib().orc_set_counters(self._h, a)

    def set_dtm(self, dtm):
        lib().orc_set_dtm(self._h, float(dtm))

    # -- kernels --------------------------------------------------------------
    def cache_weights(self) -> np.ndarray:
        cells = np.empty(self.n, np.int32)
        self._check(lib().orc_cache_weights(self._h, cells.ctypes.data_as(C.POINTER(C.c_int32))))
        return cells

    def par2grid(self, prop, grid):
        self._check(lib().orc_par2grid(self._h, PROP[prop], GRID[grid]))

    def grid2par(self, grid, prop):
        self._check(lib().orc_grid2par(self._h, GRID[grid], PROP[prop]))

    def _spec_shape(self):
        return (self.nz + 1, self.ny + 2, self.nx + 2)

    def fft_forward(self, phys):
        phys = np.ascontiguousarray(phys, np.float64)
        out = np.empty(self._spec_shape())
        self._check(lib().orc_fft_forward(self._h, _dp(phys), _dp(out)))
        return out

    def fft_backward(self, spec):
        spec = np.ascontiguousarray(spec, np.float64)
        out = np.empty((self.nz + 1, self.ny, self.nx))
        self._check(lib().orc_fft_backward(self._h, _dp(spec), _dp(out)))
        return out

    def diffx(self, a):
        a = np.ascontiguousarray(a, np.float64); out = np.empty_like(a)
        self._check(lib().orc_diffx(self._h, _dp(a), _dp(out))); return out

    def diffy(self, a):
        a = np.ascontiguousarray(a, np.float64); out = np.empty_like(a)
        self._check(lib().orc_diffy(self._h, _dp(a), _dp(out))); return out

    def filter(self, a):
        a = np.ascontiguousarray(a, np.float64); out = np.empty_like(a)
        self._check(lib().orc_filter(self._h, _dp(a), _dp(out))); return out

    def diffz(self, a, bot=None, top=None):
        a = np.ascontiguousarray(a, np.float64); out = np.empty_like(a)
        if bot is None:
            self._check(lib().orc_diffz(self._h, _dp(a), _dp(out), None, None))
        else:
            bot = np.ascontiguousarray(bot, np.float64); top = np.ascontiguousarray(top, np.float64)
            self._check(lib().orc_diffz(self._h, _dp(a), _dp(out), _dp(bot), _dp(top)))
        return out

    def laplinv(self, a, df_zero_on_boundary: bool):
        a = np.array(a, np.float64, copy=True, order="C")
        self._check(lib().orc_laplinv(self._h, _dp(a), 1 if df_zero_on_boundary else 0))
        return a

    def wavenumbers(self):
        s = (self.ny + 2, self.nx + 2)
        kx, ky, k2, f = (np.empty(s) for _ in range(4))
        lib().orc_kx_ky_k2(self._h, _dp(kx), _dp(ky), _dp(k2), _dp(f))
        return kx, ky, k2, f

    def parcel_haloswap(self):
        self._check(lib().orc_parcel_haloswap(self._h))

    # -- components -----------------------------------------------------------
    def vort2vel(self):
        self._check(lib().orc_vort2vel(self._h))

    def vort2vel_grids(self):
        """The inversion alone (vort2vel.F90:139-320) of grids p, q, r."""
        self._check(lib().orc_vort2vel_grids(self._h))

    def vorticity_tendency(self):
        self._check(lib().orc_vorticity_tendency(self._h))

    def rk4_integrator(self):
        self._check(lib().orc_rk4_integrator(self._h))

    def parcel_splitting(self):
        self._check(lib().orc_parcel_splitting(self._h))

    def parcel_mixing(self):
        self._check(lib().orc_parcel_mixing(self._h))

    def step(self):
        self._check(lib().orc_step(self._h))

    # -- test components (euler_integrator.F90, velocity.F90) ------------------
    def euler_integrator(self):
        self._check(lib().orc_euler_integrator(self._h))

    def prescribed_velocity(self, profile):
        self._check(lib().orc_prescribed_velocity(self._h, int(profile)))

    def prescribed_velocity_tag(self):
        self._check(lib().orc_prescribed_velocity_tag(self._h))

    # -- basic_parcelsetup.F90:22-134 ----------------------------------------
    def setup_basic(self, n_per_dir=2):
        """Replace the parcels with the reference's regular lattice set-up."""
        self._check(lib().orc_basic_setup(self._h, int(n_per_dir)))

    # -- the benchmark workloads' jittered thermal (no reference counterpart) --
    def setup_thermal(self, sub=2, jitter=0.25, seed=1, xc=3.141592653589793, yc=3.141592653589793, zc=0.6,
                      radius=0.4, excess=1.0, h_in=0.95, h_env0=0.3, z_strat=1.2, n2=1.0):
        """Replace the parcels with the jittered thermal, generated by the
        oracle itself (Philox4x32-10 keyed by seed and parcel index)."""
        prm = np.ascontiguousarray([sub, jitter, xc, yc, zc, radius, excess, h_in, h_env0, z_strat, n2],
                                   dtype=np.float64)
        self._check(lib().orc_thermal_setup(self._h, _dp(prm), int(seed)))

    # -- plume_parcelsetup.F90:58-334 -----------------------------------------
    def setup_plume(self, lam=1.0, H=0.8, z_c=2.5, mu=0.9, z_d=4.0, z_m=5.0, r_plume=0.8,
                    e_values=(0.3, -0.4, 0.5)) -> int:
        """Replace the parcels with the reference's plume initial condition;
        returns the number of plume parcels (they take the first slots)."""
        prm = np.ascontiguousarray([lam, H, z_c, mu, z_d, z_m, r_plume, *e_values], dtype=np.float64)
        n_plume = C.c_int64(0)
        self._check(lib().orc_plume_setup(self._h, _dp(prm), C.byref(n_plume)))
        return n_plume.value
