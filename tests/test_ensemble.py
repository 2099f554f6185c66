"""The batched ensemble (pmpic_ensemble_*): members stepped concurrently with
tuned tiles and concurrency give the same bits as the same plumes stepped alone
(members are independent, every sum runs in a fixed order, and the par2grid
column segment changes no summation order).  Needs a CUDA device."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi

MEMBERS = [  # uneven sizes, radix-2 and radix-3 grids, both precisions
    dict(nx=16, ny=16, nz=16, precision="mixed", radius=0.5, excess=1.2, seed=1000),
    dict(nx=24, ny=24, nz=24, precision="mixed", radius=0.3, excess=0.7, seed=1001),
    dict(nx=32, ny=16, nz=24, precision="fp64", radius=0.4, excess=1.0, seed=1002),
    dict(nx=32, ny=32, nz=32, precision="mixed", radius=0.45, excess=1.4, seed=1003),
]


def _ic(pm, m):
    return pm.thermal_parcels(m["nx"], m["ny"], m["nz"], radius=m["radius"], excess=m["excess"],
                              seed=m["seed"])


def _cfg(m, n):
    dt = 0.32 / max(m["nx"], m["ny"], m["nz"])
    return dict(nx=m["nx"], ny=m["ny"], nz=m["nz"], dtm=dt, dtmax=dt, max_parcels=2 * n,
                precision=m["precision"])


@pytest.mark.parametrize("threads", [0, 1])
def test_ensemble_matches_members_alone(threads):
    import pmpic_b200 as pm
    ics = [_ic(pm, m) for m in MEMBERS]
    cfgs = [_cfg(m, len(ic["x"])) for m, ic in zip(MEMBERS, ics)]
    ens = pm.Ensemble(cfgs)
    for mem, ic in zip(ens.members, ics):
        mem.upload(**ic)
    ens.autotune()
    ens.set_concurrency(threads)
    ms = ens.step(3)
    assert ms > 0
    t, xseg = ens.tuning()
    assert t >= 1 and all(s in (8, 16, 32, 64) for s in xseg)
    for i, (m, ic, cfg) in enumerate(zip(MEMBERS, ics, cfgs)):
        alone = pm.Context(cfg["nx"], cfg["ny"], cfg["nz"], TWO_PI, TWO_PI, math.pi, dtm=cfg["dtm"],
                           dtmax=cfg["dtmax"], max_parcels=cfg["max_parcels"], precision=cfg["precision"])
        alone.upload(**ic)
        alone.step(3)
        mem = ens.members[i]
        assert mem.n == alone.n, i
        for q in ["x", "y", "z", "p", "q", "r", "vol", "tag"]:
            np.testing.assert_array_equal(mem.get(q), alone.get(q), err_msg=f"member {i} {q}")
        for g in ["u", "v", "w"]:
            np.testing.assert_array_equal(mem.grid(g), alone.grid(g), err_msg=f"member {i} {g}")
        alone.close()
    ens.close()


def test_ensemble_members_vs_oracle():
    """Every member of a batched ensemble against the CPU oracle stepping the
    same plume: FP64 members' gridded u, v, w within 1e-10 and their parcel
    counts and tags identical; mixed members' within 1e-4 relative L2 with the
    oracle's parcel count."""
    import pmpic_b200 as pm
    from oracle import Oracle
    from helpers import rel, rel_l2
    ics = [_ic(pm, m) for m in MEMBERS]
    cfgs = [_cfg(m, len(ic["x"])) for m, ic in zip(MEMBERS, ics)]
    ens = pm.Ensemble(cfgs)
    for mem, ic in zip(ens.members, ics):
        mem.upload(**ic)
    ens.autotune()
    ens.set_concurrency(0)
    ens.step(3)
    for i, (ic, cfg) in enumerate(zip(ics, cfgs)):
        o = Oracle(cfg["nx"], cfg["ny"], cfg["nz"], TWO_PI, TWO_PI, math.pi, dtm=cfg["dtm"], dtmax=cfg["dtmax"],
                   max_parcels=cfg["max_parcels"])
        o.set_parcels(**ic)
        for _ in range(3):
            o.step()
        mem = ens.members[i]
        assert mem.n == o.n, i
        for g in ["u", "v", "w"]:
            a, b = mem.grid(g), o.grid(g)
            if cfg["precision"] == "fp64":
                assert rel(a, b) < 1e-10, (i, g, rel(a, b))
            else:
                assert rel_l2(a, b) < 1e-4, (i, g, rel_l2(a, b))
        if cfg["precision"] == "fp64":
            np.testing.assert_array_equal(mem.get("tag"), o.get("tag"))
        o.close()
    ens.close()
