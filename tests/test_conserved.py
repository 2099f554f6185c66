"""The compensated FP64 domain totals of vol, h*vol and b*vol on the GPU
(pmpic_conserved_sums, pmpic_step_info), against the oracle's, and the
reference's mixing invariant (report/report.tex:264; parcel_mixing.F90:87-103,
:409-418): total volume and h*vol conserved by mixing to 1e-13 on the FP64
path.  Needs a CUDA device."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi


@pytest.fixture(scope="module")
def pm():
    import pmpic_b200
    return pmpic_b200


def _shrunk_thermal(pm, N, seed=5):
    ic = pm.thermal_parcels(N, N, N)
    n = len(ic["x"])
    rng = np.random.default_rng(seed)
    vmin = (TWO_PI / N) ** 2 * (math.pi / N) / 216
    ic["vol"][rng.uniform(size=n) < 0.5] = 0.5 * vmin
    ic["h"] = ic["h"] * (1.0 + 0.1 * rng.standard_normal(n))
    return ic


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sums_match_oracle(pm, precision):
    from oracle import Oracle
    N = 32
    ic = _shrunk_thermal(pm, N)
    n = len(ic["x"])
    ctx = pm.Context(N, N, N, TWO_PI, TWO_PI, math.pi, max_parcels=2 * n, precision=precision)
    ctx.upload(**ic)
    got = ctx.conserved_sums()
    # the mixed form holds vol, h and b in FP32: the oracle sums the same rounded values
    ref_ic = dict(ic)
    if precision == "mixed":
        for k in ("vol", "h", "b"):
            ref_ic[k] = ic[k].astype(np.float32).astype(np.float64)
    o = Oracle(N, N, N, TWO_PI, TWO_PI, math.pi, max_parcels=2 * n)
    o.set_parcels(**ref_ic)
    want = o.conserved_sums()
    o.close()
    for g, w in zip(got, want):
        assert abs(g - w) <= 2e-16 * abs(w), (precision, g, w)
    # the same call twice gives the same bits; the step info carries them
    assert ctx.conserved_sums() == got
    info = ctx.info()
    assert (info.vol_sum, info.hvol_sum, info.bvol_sum) == got
    ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mixing_conserves_the_totals(pm, precision):
    """Half the parcels shrunk below vmin (report.tex:264's test): the totals
    after the mixing call, as its step info reports them, against the totals
    before it.  FP64: volume, h*vol and b*vol to 1e-13.  Mixed: FP32 fields,
    to 1e-6."""
    N = 32
    ic = _shrunk_thermal(pm, N)
    n = len(ic["x"])
    ctx = pm.Context(N, N, N, TWO_PI, TWO_PI, math.pi, max_parcels=2 * n, precision=precision)
    ctx.upload(**ic)
    before = ctx.conserved_sums()
    ctx.set_counters([0, 0, 1, 0, 3])  # mixing acts on the 4th RK substep
    ctx.parcel_mixing()
    info = ctx.info()
    assert info.n_removed > 0 and info.n_added > 0
    after = (info.vol_sum, info.hvol_sum, info.bvol_sum)
    assert after == ctx.conserved_sums()
    tol = 1e-13 if precision == "fp64" else 1e-6
    for a, b_ in zip(after, before):
        assert abs(a - b_) <= tol * abs(b_), (precision, a, b_)
    ctx.close()


def test_step_reports_the_totals(pm):
    """pmpic_step leaves the totals of the state after its last mixing call in
    the step info; on the FP64 path they equal the oracle's after the same step."""
    from oracle import Oracle
    N = 16
    ic = pm.thermal_parcels(N, N, N)
    n = len(ic["x"])
    ctx = pm.Context(N, N, N, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * n)
    ctx.upload(**ic)
    o = Oracle(N, N, N, TWO_PI, TWO_PI, math.pi, dtm=0.01, dtmax=0.01, max_parcels=2 * n)
    o.set_parcels(**ic)
    ctx.step(1)
    o.step()
    info = ctx.info()
    got = (info.vol_sum, info.hvol_sum, info.bvol_sum)
    want = o.conserved_sums()
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-14 * abs(w), (g, w)
    ctx.close()
    o.close()
