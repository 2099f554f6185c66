"""pmpic_par2grid_static: par2grid with its scratch in a static device array.

Collected last (file name) so that it also runs after every other GPU test in
the same process.  The result must equal pmpic_op_par2grid's on the same
parcels, bit for bit, on two calls in a row (the second call finds the scratch
as the first left it, so this also checks that the call clears its counters).
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import lattice_parcels

pytestmark = pytest.mark.gpu


def _static_call(L, shape, box, dev, out, stream=None):
    import torch

    nx, ny, nz = shape
    n = dev["x"].numel()
    ptr = [dev[k].data_ptr() for k in ("x", "y", "z", "vol", "b")]
    return L.pmpic_par2grid_static(nx, ny, nz, *box, n, *ptr, out.data_ptr(),
                                   None if stream is None else stream.cuda_stream)


def _case(seed, shape, box, per_dir):
    """Jittered sub-lattice parcels in shuffled slot order, random b and vol."""
    rng = np.random.default_rng(seed)
    p = lattice_parcels(*shape, *box, per_dir)
    n = len(p["x"])
    for k, L, m in (("x", box[0], shape[0]), ("y", box[1], shape[1]), ("z", box[2], shape[2])):
        h = L / m / per_dir
        p[k] = np.clip(p[k] + rng.uniform(-0.4, 0.4, n) * h, 0.0, np.nextafter(L, 0.0))
    perm = rng.permutation(n)
    p = {k: np.ascontiguousarray(v[perm]) for k, v in p.items()}
    p["b"] = rng.standard_normal(n)
    p["vol"] = p["vol"] * (0.5 + rng.random(n))
    return p


@pytest.mark.parametrize("shape,box,per_dir,seed", [
    ((16, 16, 8), (2 * np.pi, 2 * np.pi, np.pi), 2, 3),
    ((32, 32, 16), (1.0, 0.75, 0.5), 2, 7),       # 131072 parcels: the maximum
    ((32, 32, 32), (1.0, 1.0, 1.0), 1, 13),       # 32768 cells: the maximum
    ((20, 12, 6), (3.0, 2.0, 1.0), 2, 11),       # tiles cut by the domain edge
])
def test_static_par2grid_matches_context_twice(shape, box, per_dir, seed):
    import torch
    import pmpic_b200 as G

    nx, ny, nz = shape
    p = _case(seed, shape, box, per_dir)
    ctx = G.Context(nx, ny, nz, *box, max_parcels=len(p["x"]) + 16)
    ctx.upload(**{k: p[k] for k in ("x", "y", "z", "b", "vol")})
    ctx.par2grid("b", "b")
    want = ctx.grid("b")
    ctx.close()

    dev = {k: torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in ("x", "y", "z", "vol", "b")}
    L = G.lib()
    for call in range(2):
        out = torch.full(((nz + 1) * ny * nx,), np.nan, dtype=torch.float64, device="cuda")
        rc = _static_call(L, shape, box, dev, out)
        assert rc == 0, (call, rc)
        got = out.cpu().numpy().reshape(nz + 1, ny, nx)
        assert np.array_equal(got, want), (call, np.abs(got - want).max())


def test_static_par2grid_on_a_side_stream():
    import torch
    import pmpic_b200 as G

    shape, box = (16, 8, 8), (1.0, 1.0, 1.0)
    p = _case(5, shape, box, 2)
    dev = {k: torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in ("x", "y", "z", "vol", "b")}
    ref = torch.empty((9 * 8 * 16,), dtype=torch.float64, device="cuda")
    assert _static_call(G.lib(), shape, box, dev, ref) == 0
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    out = torch.empty_like(ref)
    assert _static_call(G.lib(), shape, box, dev, out, stream=s) == 0
    assert torch.equal(out, ref)


def test_static_par2grid_rejects_sizes_beyond_its_scratch():
    import torch
    import pmpic_b200 as G

    L = G.lib()
    x = torch.zeros(131073, dtype=torch.float64, device="cuda")
    out = torch.zeros(9 * 8 * 8, dtype=torch.float64, device="cuda")
    p = [x.data_ptr()] * 5
    # one parcel over the maximum: rejected before any launch
    assert L.pmpic_par2grid_static(8, 8, 8, 1.0, 1.0, 1.0, 131073, *p, out.data_ptr(), None) == -10
    # more cells than the scratch holds (64 x 32 x 32 = 65536 > 32768)
    big = torch.zeros(33 * 32 * 64, dtype=torch.float64, device="cuda")
    assert L.pmpic_par2grid_static(64, 32, 32, 1.0, 1.0, 1.0, 10, *p, big.data_ptr(), None) == -10
    # boxes below the smallest one pmpic_create accepts (4 x 4 x 3): argument errors
    for shape in ((1, 1, 1), (2, 3, 1), (3, 4, 3), (4, 4, 2)):
        assert L.pmpic_par2grid_static(*shape, 1.0, 1.0, 1.0, 10, *p, out.data_ptr(), None) == -8, shape
    assert torch.count_nonzero(out).item() == 0


def test_static_par2grid_reports_out_of_box():
    import torch
    import pmpic_b200 as G

    shape, box = (8, 8, 8), (1.0, 1.0, 1.0)
    p = _case(9, shape, box, 2)
    p["z"][17] = 1.5  # above the top wall
    dev = {k: torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in ("x", "y", "z", "vol", "b")}
    out = torch.empty((9 * 8 * 8,), dtype=torch.float64, device="cuda")
    assert _static_call(G.lib(), shape, box, dev, out) == -3
    # the error does not stick: a valid call afterwards succeeds
    p["z"][17] = 0.5
    dev["z"] = torch.from_numpy(p["z"]).cuda()
    assert _static_call(G.lib(), shape, box, dev, out) == 0
