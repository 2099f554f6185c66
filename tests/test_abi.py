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


def _philox4x32_10(c, k0, k1):
    """Philox4x32-10 (Salmon et al., SC'11) on numpy uint64 lanes holding 32-bit words."""
    mask = np.uint64(0xFFFFFFFF)
    c = [np.asarray(x, dtype=np.uint64) for x in c]
    k0, k1 = np.uint64(k0), np.uint64(k1)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        c = [((p1 >> np.uint64(32)) ^ c[1] ^ k0) & mask, p1 & mask,
             ((p0 >> np.uint64(32)) ^ c[3] ^ k1) & mask, p0 & mask]
        k0 = (k0 + np.uint64(0x9E3779B9)) & mask
        k1 = (k1 + np.uint64(0xBB67AE85)) & mask
    return c


def test_philox_known_answers():
    """The generator's Philox4x32-10 against the known-answer vectors published
    with the Random123 library (counter, key -> output)."""
    cases = [([0, 0, 0, 0], (0, 0), [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
             ([0xffffffff] * 4, (0xffffffff, 0xffffffff), [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
             ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], (0xa4093822, 0x299f31d0),
              [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, want in cases:
        assert [int(x) for x in _philox4x32_10(ctr, *key)] == want


def test_thermal_generator_vs_numpy():
    """pmpic_setup_thermal (thermal.h) against an independent numpy statement of
    the same stream and formula, bit for bit (glibc cos through math.cos)."""
    import math
    import pmpic_b200 as pm
    nx, ny, nz, s, seed = 6, 5, 4, 2, (7 << 32) | 11
    lx, ly, lz = 2 * np.pi, 5.0, np.pi
    kw = dict(lx=lx, ly=ly, lz=lz, sub=s, jitter=0.25, seed=seed, xc=3.0, yc=2.4, zc=0.7, radius=0.9,
              excess=1.5, h_in=0.9, h_env0=0.3, z_strat=1.1, n2=1.2)
    got = pm.thermal_parcels(nx, ny, nz, **kw)
    idx = np.arange(nx * ny * nz * s ** 3, dtype=np.uint64)
    lo, hi = idx & np.uint64(0xFFFFFFFF), idx >> np.uint64(32)
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    zero, one = np.zeros_like(idx), np.ones_like(idx)
    c1 = _philox4x32_10([lo, hi, zero, zero], k0, k1)
    c2 = _philox4x32_10([lo, hi, one, zero], k0, k1)

    def u01(a, b):
        v = ((a << np.uint64(21)) ^ (b >> np.uint64(11))) & np.uint64((1 << 53) - 1)
        return v.astype(np.float64) * (1.0 / 9007199254740992.0)

    jx = (2.0 * u01(c1[0], c1[1]) - 1.0) * 0.25
    jy = (2.0 * u01(c1[2], c1[3]) - 1.0) * 0.25
    jz = (2.0 * u01(c2[0], c2[1]) - 1.0) * 0.25
    t = idx.astype(np.int64)
    cell, w = t // s ** 3, t % s ** 3
    i, j, k = cell // (ny * nz), (cell // nz) % ny, cell % nz
    a, b, c = w // (s * s), (w // s) % s, w % s
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    x = i * dx + (a + 0.5 + jx) * (dx / s)
    y = j * dy + (b + 0.5 + jy) * (dy / s)
    z = k * dz + (c + 0.5 + jz) * (dz / s)
    rr = np.sqrt((x - 3.0) * (x - 3.0) + (y - 2.4) * (y - 2.4) + (z - 0.7) * (z - 0.7))
    benv = np.where(z > 1.1, (z - 1.1) * 1.2, 0.0)
    bb, hh = benv.copy(), 0.3 * (1.0 - z / lz)
    pi = 4.0 * math.atan(1.0)
    for e in np.nonzero(rr < 0.9)[0]:
        cs = math.cos(pi * rr[e] / (2.0 * 0.9))
        bb[e] = benv[e] + 1.5 * cs * cs
        hh[e] = 0.9
    want = {"x": x, "y": y, "z": z, "b": bb, "h": hh, "vol": np.full(len(t), dx * dy * dz / float(s ** 3)),
            "tag": t.astype(np.float64)}
    assert 0 < int((rr < 0.9).sum()) < len(t)
    for key, v in want.items():
        np.testing.assert_array_equal(got[key], v, err_msg=key)


def test_oracle_thermal_generator_matches_host_generator():
    """The oracle's own thermal set-up (the CPU legs' initial condition) gives
    the same parcels as the library's host generator, bit for bit, so the CPU
    baseline and the GPU arm start from the same state without the CPU legs
    loading the library."""
    import pmpic_b200 as pm
    from oracle import Oracle
    cases = [(6, 5, 4, dict(lx=2 * np.pi, ly=5.0, lz=np.pi, sub=2, jitter=0.25, seed=(7 << 32) | 11, xc=3.0,
                            yc=2.4, zc=0.7, radius=0.9, excess=1.5, h_in=0.9, h_env0=0.3, z_strat=1.1, n2=1.2)),
             (16, 16, 16, dict(lx=2 * np.pi, ly=2 * np.pi, lz=np.pi)),
             (8, 8, 6, dict(lx=2 * np.pi, ly=2 * np.pi, lz=np.pi, sub=3, seed=5))]
    for nx, ny, nz, kw in cases:
        got = pm.thermal_parcels(nx, ny, nz, **kw)
        o = Oracle(nx, ny, nz, kw["lx"], kw["ly"], kw["lz"], max_parcels=len(got["x"]) + 5)
        o.setup_thermal(**{k: v for k, v in kw.items() if k not in ("lx", "ly", "lz")})
        assert o.n == len(got["x"])
        for key in ("x", "y", "z", "p", "q", "r", "b", "h", "vol", "stretch", "tag"):
            np.testing.assert_array_equal(o.get(key), got[key], err_msg=key)
        o.close()


def test_ensemble_members_spread_by_cost():
    """pmpic_b200.assign_members: every member on exactly one rank, the ranks'
    loads within one member's cost of each other, the same answer every time,
    and a rank without members when there are more ranks than members."""
    import pmpic_b200 as pm
    import bench
    spec = bench.ensemble_members(64)
    costs = [8 * m["G"] ** 3 * 50 for m in spec]
    for ranks in (1, 2, 3, 4, 8):
        parts = pm.assign_members(costs, ranks)
        assert len(parts) == ranks
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert parts == pm.assign_members(costs, ranks)
    parts = pm.assign_members([5.0, 3.0], 3)
    assert parts == [[0], [1], []]
