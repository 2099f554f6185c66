"""Host-side checks that need no GPU: the C ABI's symbol table, configuration
validation, the parcel set-up generator, the oracle's transforms against numpy,
and the multi-rank reduction of bench.py under gloo."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "pmpic_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pmpic_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import pmpic_b200 as pm
    lib = C.CDLL(pm.LIB_PATH)
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_configs_rejected_without_a_device():
    import pmpic_b200 as pm
    L = pm.lib()
    h = C.c_void_p()
    bad = [
        pm.Config(7, 8, 8, 0, 1, 0, 1, 0, 1, .01, .01, .5, 100, 0, 0),     # odd nx
        pm.Config(14, 8, 8, 0, 1, 0, 1, 0, 1, .01, .01, .5, 100, 0, 0),    # 7 is not 2^a 3^b 5^c
        pm.Config(8, 8, 8, 0.5, 1, 0, 1, 0, 1, .01, .01, .5, 100, 0, 0),   # non-zero origin
        pm.Config(8, 8, 8, 0, 1, 0, 1, 0, 1, .01, .01, .5, 0, 0, 0),       # no capacity
        pm.Config(8, 8, 8, 0, 1, 0, 1, 0, 1, .01, .01, .5, 100, 7, 0),     # unknown precision
    ]
    for cfg in bad:
        assert L.pmpic_create(C.byref(cfg), C.byref(h)) == -1  # PMPIC_ERR_CONFIG


def test_thermal_setup_is_deterministic_and_in_box():
    import pmpic_b200 as pm
    a = pm.thermal_parcels(8, 8, 8, seed=3)
    b = pm.thermal_parcels(8, 8, 8, seed=3)
    c = pm.thermal_parcels(8, 8, 8, seed=4)
    n = 8 ** 3 * 8
    assert len(a["x"]) == n
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert not np.array_equal(a["x"], c["x"])
    L, H = 2 * np.pi, np.pi
    assert a["x"].min() > 0 and a["x"].max() < L and a["z"].min() > 0 and a["z"].max() < H
    np.testing.assert_array_equal(a["tag"], np.arange(n))
    dx = L / 8
    # 2x2x2 jittered sub-lattice: each parcel stays within its quarter-cell window
    cell = np.floor(a["x"] / dx)
    centre = dx * (cell + np.floor((a["x"] / dx - cell) * 2) / 2 + 0.25)
    assert np.all(np.abs(a["x"] - centre) <= 0.125 * dx * (1 + 1e-12))  # jitter of 0.25 sub-spacings
    assert np.allclose(a["vol"], (L / 8) ** 2 * (H / 8) / 8)
    r = np.sqrt((a["x"] - np.pi) ** 2 + (a["y"] - np.pi) ** 2 + (a["z"] - 0.6) ** 2)
    assert np.all(a["h"][r < 0.4] == 0.95)
    assert a["b"][r < 0.4].max() > 0.3 and a["b"][(r > 0.4) & (a["z"] < 1.2)].max() == 0.0


@pytest.mark.parametrize("shape", [(32, 48, 16), (40, 24, 8), (30, 20, 6)])
def test_oracle_fft_matches_numpy(shape):
    from oracle import Oracle
    nx, ny, nz = shape
    o = Oracle(nx, ny, nz, 2 * np.pi, 2 * np.pi, np.pi, max_parcels=4)
    rng = np.random.default_rng(1)
    f = rng.standard_normal((nz + 1, ny, nx))
    s = o.fft_forward(f)
    Y = np.fft.rfft(f, axis=1)
    X1, X2 = np.fft.rfft(Y.real, axis=2), np.fft.rfft(Y.imag, axis=2)
    ref = np.empty_like(s)
    ref[:, 0::2, 0::2], ref[:, 0::2, 1::2] = X1.real, X1.imag
    ref[:, 1::2, 0::2], ref[:, 1::2, 1::2] = X2.real, X2.imag
    assert np.abs(s - ref).max() / np.abs(ref).max() < 1e-14
    assert np.abs(o.fft_backward(s) - f).max() < 1e-13


def test_oracle_c2r_ignores_zero_and_nyquist_imaginary_parts():
    """ffte_c2r (ffte_mod.F90:97-124) takes the real part of the inverse of the
    conjugate-symmetric extension, so Im of modes 0 and N/2 cannot matter."""
    from oracle import Oracle
    o = Oracle(16, 16, 4, 1.0, 1.0, 1.0, max_parcels=4)
    rng = np.random.default_rng(2)
    s = rng.standard_normal((5, 18, 18))
    a = o.fft_backward(s)
    s2 = s.copy()
    s2[:, :, 1] += 3.0      # Im of x-mode 0
    s2[:, :, 17] -= 2.0     # Im of x-mode N/2
    b = o.fft_backward(s2)
    np.testing.assert_allclose(a, b, atol=1e-13)


def _combine_worker(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t, w = bench.combine(1.0 + rank, 100 * (rank + 1), dist, "cpu")
    q.put((rank, t, w))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_combine_two_ranks_gloo():
    """Replica timing over 2 ranks: max of the device times, sum of the work."""
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_combine_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(2))
    for _, t, w in res:
        assert t == 2.0 and w == 300.0
