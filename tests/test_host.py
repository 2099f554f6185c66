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


REF_SET = ("global_configuration={g}\n"
           "initialisation_stage_ordering=decomposition, setup_grid, parcelsetup_base, basic_parcelsetup,"
           "plume_parcelsetup, readfromfile_parcelsetup,termination_check, model_synopsis, halo_swapper, "
           "writebinary, writenetcdf, prescribed_parcel_velocity, euler_integrator,rk4_integrator,vort2vel,"
           "vorticity_tendency,parcel_mixing,parcel_splitting\n"
           "start_group_contents=writebinary,writenetcdf,termination_check, halo_swapper\n"
           "integrator_group_contents=prescribed_parcel_velocity,euler_integrator,rk4_integrator\n"
           "parcelsetup_base_enabled=.true.\nplume_parcelsetup_enabled=.true.\nthermal_parcelsetup_enabled=.false.\n"
           "euler_integrator_enabled=.true.\nprescribed_parcel_velocity_enabled=.true.\nvelocity_profile=2\n"
           "writebinary_enabled=.true.\nwritebinary_mode=step\nparcel_step_write_frequency=5\n"
           "grid_step_write_frequency=5\nwritenetcdf_enabled=.true.\nwritenetcdf_mode=none\n"
           "lambda=1\nH=0.8\nz_c=2.5\nmu=0.9\nz_d=4.\nz_m=5.\nr_plume=0.8\ne_values=0.3, -0.4 ,0.5\n"
           "nx=32\nny=32\nnz=32\nxmin=0\nxmax=6.28\nymin=0\nymax=6.28\nzmin=0\nzmax=6.28\n"
           "max_parcels=1000000\ndtm=0.1\ndtmax=0.1\n")


def _ref_set(tmp_path, extra=""):
    cfg = tmp_path / "ref_set.mcf"
    cfg.write_text(REF_SET.format(g=os.path.join(DATA, "monc_global_config")) + extra)
    return cfg


def test_reference_component_set_order(tmp_path):
    """The reference's set-up, test-integrator and writer components in its
    global_config orderings: parcelsetup_base allocates, plume_parcelsetup
    fills, the Euler integrator sets one stage per step (euler_integrator.F90:49)."""
    out = run(f"--config={_ref_set(tmp_path)}", "--dry-run").stdout
    init = out.split("init:")[1].split("\n")[0].split()
    step = out.split("step:")[1].split("\n")[0].split()
    assert init == ["parcelsetup_base", "plume_parcelsetup", "writebinary", "writenetcdf",
                    "prescribed_parcel_velocity", "euler_integrator"]
    assert step == ["writebinary", "writenetcdf", "termination_check", "prescribed_parcel_velocity",
                    "euler_integrator", "model_synopsis"]


def test_two_integrators_are_refused(tmp_path):
    p = run(f"--config={_ref_set(tmp_path, 'rk4_integrator_enabled=.true.\n')}", "--dry-run", check=False)
    assert p.returncode != 0 and "another integrator" in p.stderr


@pytest.mark.parametrize("extra,msg", [("e_values=0.3, -0.4\n", "e_values needs 3 values"),
                                       ("velocity_profile=11\n", "not one of 0..10")])
def test_bad_component_options_are_refused(tmp_path, extra, msg):
    p = run(f"--config={_ref_set(tmp_path, extra)}", "--dry-run", check=False)
    assert p.returncode != 0 and msg in p.stderr


def test_unknown_writer_mode_is_refused(tmp_path):
    p = run(f"--config={_ref_set(tmp_path, 'writenetcdf_mode=sometimes\n')}", "--dry-run", check=False)
    assert p.returncode != 0 and "not recognised" in p.stderr


def test_restart_counts_the_rank_files(tmp_path):
    """readfromfile_parcelsetup (readfromfile_parcelsetup.F90:50-68): the dumps of
    step restart_num are found rank by rank until one is missing; none is an error."""
    cfg = _ref_set(tmp_path, "plume_parcelsetup_enabled=.false.\nreadfromfile_parcelsetup_enabled=.true.\n"
                             "restart_num=7\n")

    def host():
        return subprocess.run([MONC, f"--config={cfg}", "--dry-run"], capture_output=True, text=True,
                              timeout=60, cwd=tmp_path)

    p = host()
    assert p.returncode != 0 and "no file to restart from" in p.stderr
    for rank in (0, 1):
        (tmp_path / f"parcels_{rank:05d}_00007.dat").write_bytes(b"")
    (tmp_path / "parcels_00003_00007.dat").write_bytes(b"")  # after a gap: not part of the dump
    p = host()
    assert p.returncode == 0, p.stderr
    assert "Found 2 files" in p.stdout
    init = p.stdout.split("init:")[1].split("\n")[0].split()
    assert init[:2] == ["parcelsetup_base", "readfromfile_parcelsetup"]


CONFIGS = os.path.join(ROOT, "pmpic_b200", "host", "configs")


def test_shipped_plume_configuration():
    """pmpic_b200/host/configs/plume.mcf: plume set-up, the full integrator group
    four times per step, both writers in the start group."""
    out = run(f"--config={os.path.join(CONFIGS, 'plume.mcf')}", "--dry-run").stdout
    init = out.split("init:")[1].split("\n")[0].split()
    step = out.split("step:")[1].split("\n")[0].split()
    assert init == ["parcelsetup_base", "plume_parcelsetup", "writebinary", "writenetcdf", "rk4_integrator"]
    body = ["vort2vel", "vorticity_tendency", "rk4_integrator", "parcel_splitting", "parcel_mixing"]
    assert step == ["writebinary", "writenetcdf", "termination_check"] + body * 4 + ["model_synopsis"]


def test_shipped_migration_configuration():
    """pmpic_b200/host/configs/migration.mcf: lattice set-up, prescribed velocity
    then Euler once per step (grid2par.mcf's group order)."""
    out = run(f"--config={os.path.join(CONFIGS, 'migration.mcf')}", "--dry-run").stdout
    init = out.split("init:")[1].split("\n")[0].split()
    step = out.split("step:")[1].split("\n")[0].split()
    assert init == ["parcelsetup_base", "basic_parcelsetup", "writebinary", "writenetcdf",
                    "prescribed_parcel_velocity", "euler_integrator"]
    assert step == ["writebinary", "writenetcdf", "termination_check", "prescribed_parcel_velocity",
                    "euler_integrator", "model_synopsis"]


def test_quoted_writer_modes_parse(tmp_path):
    """The reference's config.mcf quotes string options (writebinary_mode="time")."""
    extra = 'writebinary_mode="time"\nparcel_time_write_frequency=1.\ngrid_time_write_frequency=1.\n' \
            'writenetcdf_mode="step"\nparcel_step_write_netcdf_frequency=10\ngrid_step_write_netcdf_frequency=5\n'
    p = run(f"--config={_ref_set(tmp_path, extra)}", "--dry-run", check=False)
    assert p.returncode == 0, p.stderr
