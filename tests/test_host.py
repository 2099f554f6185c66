"""The MONC-style host (pmpic_b200/pmpic_monc): options database, registry and
timestepper, mirroring model_core/src/configuration/configurationfileparser.F90,
model_core/src/components/registry.F90 and timestepper.F90.

The CPU tests use the host's --dry-run mode, which builds the registry and runs
one step's callback order without a device; the GPU test runs the host for real
and compares its final state with the Python binding driving the same steps.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT

MONC = os.path.join(ROOT, "pmpic_b200", "pmpic_monc")
DATA = os.path.join(ROOT, "tests", "data")


def run(*args, check=True):
    p = subprocess.run([MONC, *args], capture_output=True, text=True, timeout=300)
    if check:
        assert p.returncode == 0, p.stdout + p.stderr
    return p


def dry(*extra):
    out = run(f"--config={os.path.join(DATA, 'monc_config.mcf')}", "--dry-run", *extra).stdout
    init = out.split("init:")[1].split("\n")[0].split()
    step = out.split("step:")[1].split("\n")[0].split()
    return init, step


def test_rk_group_runs_four_times_in_group_order():
    init, step = dry()
    # disabled parcel_mixing is skipped, euler_integrator is unknown/disabled
    body = ["vort2vel", "vorticity_tendency", "rk4_integrator", "parcel_splitting"]
    assert step == ["termination_check"] + body * 4 + ["model_synopsis"]


def test_plus_equals_appends_to_included_list():
    init, _ = dry()
    # initialisation_stage_ordering from the included file, += thermal_parcelsetup
    assert init == ["rk4_integrator", "thermal_parcelsetup"]


def test_command_line_override_wins_over_file():
    _, step = dry("--parcel_mixing_enabled=.true.")
    body = ["vort2vel", "vorticity_tendency", "rk4_integrator", "parcel_splitting", "parcel_mixing"]
    assert step == ["termination_check"] + body * 4 + ["model_synopsis"]


def test_missing_configuration_file_fails():
    p = run("--config=" + os.path.join(DATA, "no_such_file.mcf"), check=False)
    assert p.returncode != 0 and "cannot read" in p.stderr


def test_unsupported_group_type_fails():
    p = run(f"--config={os.path.join(DATA, 'monc_config.mcf')}", "--dry-run",
            "--last_group_type=sometimes", check=False)
    assert p.returncode != 0 and "not supported" in p.stderr


@pytest.mark.gpu
def test_host_run_matches_python_binding(tmp_path):
    import pmpic_b200 as G

    n, L = 16, 2 * np.pi
    steps, dtm = 3, 0.02
    cfg = tmp_path / "run.mcf"
    cfg.write_text(f"global_configuration={os.path.join(DATA, 'monc_global_config')}\n"
                   "rk4_integrator_enabled=.true.\nvort2vel_enabled=.true.\n"
                   "vorticity_tendency_enabled=.true.\nparcel_splitting_enabled=.true.\n"
                   "parcel_mixing_enabled=.true.\ninitialisation_stage_ordering+=thermal_parcelsetup\n"
                   f"nx={n}\nny={n}\nnz={n}\nxmin=0\nxmax={L!r}\nymin=0\nymax={L!r}\n"
                   f"zmin=0\nzmax={np.pi!r}\nmax_parcels=400000\ndtm={dtm!r}\ndtmax={dtm!r}\n"
                   f"termination_time=1000\nnn_timesteps={steps}\ndisplay_synopsis_frequency=1\n")
    out = run(f"--config={cfg}").stdout
    last = [l for l in out.splitlines() if l.startswith("step ")][-1]
    n_host = int(re.search(r"parcels (\d+)", last).group(1))
    dt_host = float(re.search(r" dt (\S+)", last).group(1))

    ic = G.thermal_parcels(n, n, n, L, L, np.pi)
    ctx = G.Context(n, n, n, L, L, np.pi, dtm=dtm, dtmax=dtm, max_parcels=400000)
    ctx.upload(**ic)
    for _ in range(steps):
        ctx.step(1)
    info = ctx.info()
    assert n_host == info.n_parcels
    assert dt_host == pytest.approx(info.dtm, rel=1e-5)
