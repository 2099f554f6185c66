#!/usr/bin/env python
"""Benchmark of the PMPIC hot path on B200: parcel-RK4-steps/s of the 256^3
thermal plume (one model step = four RK4 substeps of vort2vel,
vorticity_tendency, rk4_integrator, parcel_splitting, parcel_mixing).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One process per GPU (torchrun for N > 1); every rank runs an independent
replica of the plume (the path does not shard), value = all ranks' parcel
steps / the max over ranks of the device time.  ``--impl reference`` times the
CPU restatement of the reference on the host cores instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "parcel-RK4-steps/s at 256³: mixed-prec vs FP64 GPU, ≤1e-4 rel err vs FP64"
UNIT = "parcel-RK4-steps/s"
PEAKS_FILE = os.path.join(HERE, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0

# the 256^3 plume (thermal of radius 0.4 at (pi, pi, 0.6) in [0,2pi]^2 x [0,pi])
PLUME = dict(lx=2 * np.pi, ly=2 * np.pi, lz=np.pi, sub=2, jitter=0.25, seed=1, xc=np.pi, yc=np.pi,
             zc=0.6, radius=0.4, excess=1.0, h_in=0.95, h_env0=0.3, z_strat=1.2, n2=1.0)


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def combine(t_dev, work, pg, device):
    """Max of the device time and sum of the work over ranks (replicas)."""
    if pg is None:
        return float(t_dev), float(work)
    import torch
    t = torch.tensor([float(t_dev)], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    w = torch.tensor([float(work)], device=device, dtype=torch.float64)
    pg.all_reduce(w, op=pg.ReduceOp.SUM)
    return float(t.item()), float(w.item())


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference(grid, steps, warmup, threads):
    """The CPU restatement of the reference (oracle), timed on the host cores.
    The initial condition is the oracle's own thermal generator (the same
    parcels as the GPU path's, bit for bit), so nothing of the B200 library is
    loaded on this leg."""
    from oracle import Oracle
    n0 = PLUME["sub"] ** 3 * grid ** 3
    o = Oracle(grid, grid, grid, PLUME["lx"], PLUME["ly"], PLUME["lz"], dtm=0.0025, dtmax=0.0025,
               max_parcels=int(1.1 * n0), threads=threads)
    o.setup_thermal(**{k: PLUME[k] for k in ("sub", "jitter", "seed", "xc", "yc", "zc", "radius", "excess",
                                             "h_in", "h_env0", "z_strat", "n2")})
    assert o.n == n0
    for _ in range(warmup):
        o.step()
    work = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        work += o.n
        o.step()
    dt = time.perf_counter() - t0
    o.close()
    return work / dt, n0, dt


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    grid = args.ref_grid
    value, n0, dt = cpu_reference(grid, args.steps, args.warmup, threads)
    sample = (f"{grid}^3 plume ({n0} parcels, the same thermal and environment as the GPU arm), "
              f"{args.steps} timed steps after {args.warmup} warm-up; C++/OpenMP restatement of the "
              f"reference Fortran (no Fortran compiler or MPI here to build the reference itself)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"thermal plume {grid}^3, FP64, 8 parcels/cell; 4 RK4 substeps + "
                                   f"splitting + mixing per step",
                       "grid": grid, "parcels_initial": n0, "dt": 0.0025, "precision": "fp64"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def algorithmic_bytes(kernel, precision, n_avg, nphys, calls, steps):
    """Algorithmic bytes of all launches of one kernel in the timed region.

    par2grid (per launch, one field set): offsets, vol and the fields of every
      parcel, its sorted index, and the NQ grids written.  Per step: four
      vort2vel passes (p, q, r and btot from b, h, z, the btot property
      written back), the mixing kept class and, when any parcel is removed,
      the removed class (6 sums over b, h, p, q, r).
    rk4_kernel (per stage): the RK4 state it must read and write (x, y, z, p,
      q, r and their xo/xf copies, the six tendencies, the direction byte),
      the binning it gathers at (FP64: cell id + 3 offsets), and the six grids
      read once.  Stage 1 reads x, writes xo, xf, x; stages 2-3 read xo, xf,
      write xf, x; stage 4 reads xf, writes xf, x.  On the mixed form the
      current position is the cell id and three offsets (also the next
      binning), xf a displacement from xo, and every stage reads the current
      position for its gather (stages 2-4 read xo as well); its last stage
      advances the stretch of the split that follows (read + write).  Within
      pmpic_step stages 1-3 store no tendencies (dead until the next stage
      gathers them again).
    """
    w = 8 if precision == "fp64" else 4
    if kernel == "par2grid":
        if precision == "fp64":
            b0, b1 = 92.0, 76.0   # 3 del + vol + p,q,r + b,h,z + btot out (+4 index); 3 del + vol + b,h,p,q,r
        else:
            b0, b1 = 44.0, 40.0   # 3 offsets + vol + p,q,r + b,h + btot out (+4 index); 3 offsets + vol + b,h,p,q,r
        per_step = 4 * (b0 * n_avg + 4 * w * nphys) + (b1 * n_avg + 6 * w * nphys)
        extra = max(calls - 5 * steps, 0) * (b1 * n_avg + 6 * w * nphys)
        return per_step * steps + extra
    if kernel == "rk4_kernel":
        if precision == "fp64":
            st = [76 + 145, 124 + 97, 124 + 97, 76 + 145]
        else:
            # current position: cell id + 3 FP32 offsets (16 B, read at every
            # stage for the gather, written as the next binning); xo: 3 x
            # {int, FP32} (written at stage 1, read after); xf: 3 FP32
            # displacements; p, q, r and their po/pf copies FP32; the
            # direction byte; stage 4: the stretch and the six tendencies
            st = [28 + 89, 76 + 53, 76 + 53, 68 + 81]
        return steps * sum(s_ * n_avg + 6 * w * nphys for s_ in st)
    return None


# DRAM bytes per parcel of one launch, from ncu captures of the same kernels on
# the 128^3 plume (16.8 M parcels; these kernels stream the parcel state once, so
# traffic scales with parcels): RK4 stages 1-2 averaged, par2grid vort2vel pass.
TRAFFIC_PER_PARCEL = {("rk4_kernel", "fp64"): 235.9, ("rk4_kernel", "mixed"): 123.9,
                      ("par2grid", "fp64"): 108.6, ("par2grid", "mixed"): 55.7}


def run_form(precision, args, local, pg, headline):
    """One context of `precision`: W warm-up steps, K timed steps (CUDA events on
    the library's stream, clocks sampled), then untimed steps up to
    args.error_steps, and the gridded velocity downloaded for the error check."""
    import torch
    import pmpic_b200 as pm
    grid = args.grid
    ic = pm.thermal_parcels(grid, grid, grid, **PLUME)
    n0 = len(ic["x"])
    cap = int(args.capacity * n0)
    ctx = pm.Context(grid, grid, grid, PLUME["lx"], PLUME["ly"], PLUME["lz"], dtm=0.0025, dtmax=0.0025,
                     max_parcels=cap, device=local, precision=precision)
    ctx.upload(**ic)
    del ic
    L = pm.lib()
    h = ctx._h
    if args.p2g_segment:
        L.pmpic_set_p2g_segment(h, args.p2g_segment)

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        ctx.step(1)
    barrier()
    L.pmpic_timing(h, 1)
    l0 = C.c_int64()
    L.pmpic_launch_count(h, C.byref(l0))
    work = 0
    with ClockSampler(local) as clk:
        L.pmpic_event_record(h, 0)
        for _ in range(args.steps):
            work += ctx.n
            ctx.step(1)
        L.pmpic_event_record(h, 1)
        ms = C.c_float()
        L.pmpic_event_elapsed(h, 0, 1, C.byref(ms))
    l1 = C.c_int64()
    L.pmpic_launch_count(h, C.byref(l1))
    timers = {}
    for i in range(L.pmpic_timer_count()):
        tot, calls = C.c_double(), C.c_int64()
        L.pmpic_timer_read(h, i, C.byref(tot), C.byref(calls))
        timers[L.pmpic_timer_name(i).decode()] = (tot.value, calls.value)
    L.pmpic_timing(h, 0)
    barrier()
    t_max, work_all = combine(ms.value / 1e3, work, pg, "cuda")
    res = {"value": work_all / t_max, "ms_per_step": 1e3 * t_max / args.steps, "n0": n0, "cap": cap,
           "gpu_launches": int(l1.value - l0.value), "clocks": clk.summary(),
           "timers_ms": {k: round(v[0], 3) for k, v in timers.items() if v[1]}}

    # roofline of the dominant kernel of the two candidates
    peak, peak_kind = hbm_peak()
    nphys = (grid + 1) * grid * grid
    n_avg = work / max(args.steps, 1)
    best = max(["par2grid", "rk4_kernel"], key=lambda k: timers.get(k, (0.0, 0))[0])
    tot, calls = timers.get(best, (0.0, 0))
    step_ms = timers.get("step", (ms.value, args.steps))[0]
    total_bytes = algorithmic_bytes(best, precision, n_avg, nphys, calls, args.steps)
    achieved = total_bytes / (tot / 1e3) / 1e9 if calls and tot > 0 else None
    res["roofline"] = {
        "bound": "hbm", "kernel": best, "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None,
        "traffic": TRAFFIC_PER_PARCEL.get((best, precision), 0.0) * n_avg or None,
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per parcel at 128^3, scaled by parcels",
        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
        "share_of_step": tot / step_ms if step_ms else None, "launches": calls,
        "avg_launch_ms": tot / calls if calls else None,
        "algorithmic_bytes_per_launch": total_bytes / calls if calls else None}

    # the continuation to args.error_steps, timed as a second window (the
    # parcels have drifted from their set-up order and splitting has appended),
    # then the gridded velocity
    done = args.warmup + args.steps
    late_work, late_steps = 0, 0
    mixing_events = {"steps_with_removals": 0, "steps_with_new_parcels": 0, "split": 0, "removed": 0, "added": 0}
    L.pmpic_event_record(h, 6)
    while done < args.error_steps:
        late_work += ctx.n
        ctx.step(1)
        done += 1
        late_steps += 1
        inf = ctx.info()  # the step has synchronised already; this reads the counters it left
        mixing_events["steps_with_removals"] += int(inf.n_removed > 0)
        mixing_events["steps_with_new_parcels"] += int(inf.n_added > 0)
        mixing_events["split"] += int(inf.n_split)
        mixing_events["removed"] += int(inf.n_removed)
        mixing_events["added"] += int(inf.n_added)
    L.pmpic_event_record(h, 7)
    if late_steps:
        ms_late = C.c_float()
        L.pmpic_event_elapsed(h, 6, 7, C.byref(ms_late))
        t_late, late_all = combine(ms_late.value / 1e3, late_work, pg, "cuda")
        res["late_run"] = {"steps": f"{args.warmup + args.steps + 1}-{done}", "value": late_all / t_late,
                           "ms_per_step": 1e3 * t_late / late_steps, "unit": UNIT,
                           "events": mixing_events}
    res["steps_total"] = done
    res["n_final"] = ctx.n
    res["grids"] = {q: ctx.grid(q) for q in ("u", "v", "w")} if args.error_steps > 0 else None

    # end to end through the C ABI, host-owned state (headline form only; after
    # the error check, whose step count it would otherwise change)
    if headline and args.e2e_steps > 0:
        res["e2e"] = e2e_run(ctx, args, pg, barrier)
    ctx.close()
    return res


def e2e_run(ctx, args, pg, barrier):
    """The same step with the state on the host: each step uploads it from pinned
    host memory, runs through the C ABI and downloads the result."""
    import pmpic_b200 as pm
    L = pm.lib()
    h = ctx._h
    nb = ctx.n
    cap_h = int(nb * 1.02) + 1024
    host = {}
    for k in pm.IO_PROPS:
        a = np.empty(cap_h, np.float64)
        host[k] = a
        L.pmpic_pin_host(C.c_void_p(a.ctypes.data), C.c_size_t(a.nbytes))
    cur = ctx.download()
    for k in pm.IO_PROPS:
        host[k][:len(cur[k])] = cur[k]
    nh = len(cur["x"])
    del cur
    barrier()
    e2e_work, h2d, d2h, done = 0, 0, 0, 0
    cnt = C.c_int64()
    L.pmpic_event_record(h, 2)
    for _ in range(args.e2e_steps):
        ptrs = [host[k].ctypes.data_as(C.POINTER(C.c_double)) for k in pm.IO_PROPS]
        if L.pmpic_upload_parcels(h, nh, *ptrs):
            break
        e2e_work += nh
        h2d += 8 * 11 * nh
        L.pmpic_step(h, 1)
        if ctx.n > cap_h:
            break
        L.pmpic_download_parcels(h, cap_h, C.byref(cnt), *ptrs)
        nh = int(cnt.value)
        d2h += 8 * 11 * nh
        done += 1
    L.pmpic_event_record(h, 3)
    ms2 = C.c_float()
    L.pmpic_event_elapsed(h, 2, 3, C.byref(ms2))
    for k in pm.IO_PROPS:
        L.pmpic_unpin_host(C.c_void_p(host[k].ctypes.data))
    t_e2e, e2e_all = combine(ms2.value / 1e3, e2e_work, pg, "cuda")
    if not done:
        return None
    return {"value": e2e_all / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d // done,
            "d2h_bytes_per_step": d2h // done, "steps": done,
            "path": "pmpic_upload_parcels (pinned host, FP64) -> pmpic_step -> pmpic_download_parcels"}


def run_b200(args):
    rank, world, local = dist_env()
    import torch  # device selection and the multi-rank plumbing only
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    # the headline form first, on a device no other context of this process has
    # allocated and freed memory on yet; the FP64 form after it
    forms = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    headline = forms[0]
    res = {f: run_form(f, args, local, pg, f == headline) for f in forms}
    hr = res[headline]
    err = None
    if "fp64" in res and "mixed" in res and res["mixed"]["grids"] is not None:
        err = {"steps": res["mixed"]["steps_total"], "reference": "the plain FP64 GPU path, same plume"}
        for q in ("u", "v", "w"):
            a, b = res["mixed"]["grids"][q], res["fp64"]["grids"][q]
            err[q + "_rel_l2"] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
            err[q + "_max_abs"] = float(np.abs(a - b).max())
        err["n_parcels"] = {"mixed": res["mixed"]["n_final"], "fp64": res["fp64"]["n_final"]}

    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        threads = os.cpu_count() or 1
        v, n_s, dt = cpu_reference(args.ref_grid, 1, 1, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{args.ref_grid}^3 plume ({n_s} parcels, the GPU arm's initial state), 1 timed "
                         f"step after 1 warm-up step ({dt:.1f} s), C++/OpenMP restatement of the reference"}
    if pg:
        pg.barrier()
    if rank == 0:
        grid = args.grid
        label = {"mixed": "mixed-precision form (FP32 fields/grids/RK4, int cell + FP32 offset positions, "
                          "FP64 zero mode)", "fp64": "plain FP64 path"}
        line = {"metric": METRIC, "value": hr["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": hr["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (f64 zero mode)" if headline == "mixed" else "f64",
                "data": "synthetic (seeded jittered-lattice thermal plume, 8 parcels/cell)",
                "config": {"workload": f"thermal plume {grid}^3, {label[headline]}; 4 RK4 substeps + "
                                       f"splitting + mixing per step",
                           "grid": grid, "parcels_initial": hr["n0"], "max_parcels": hr["cap"], "dt": 0.0025,
                           "precision": headline, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2 (parcel state {:.0f} GB)".format(hr["n0"] * 30 * 8 / 1e9)},
                "roofline": hr["roofline"], "cpu_baseline": cpu, "e2e": hr.get("e2e"),
                "gpu_launches": hr["gpu_launches"], "clocks": hr["clocks"], "timers_ms": hr["timers_ms"],
                "late_run": hr.get("late_run")}
        if "fp64" in res and headline != "fp64":
            f = res["fp64"]
            line["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "roofline": f["roofline"],
                            "gpu_launches": f["gpu_launches"], "clocks": f["clocks"], "timers_ms": f["timers_ms"],
                            "late_run": f.get("late_run")}
            line["mixed_over_fp64"] = hr["value"] / f["value"]
        line["error_vs_fp64"] = err
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


def fourier_field(x, y, z, nmodes, kmax, rng, lx=2 * np.pi, ly=2 * np.pi, lz=np.pi):
    """Sum of nmodes random Fourier modes with |k| <= kmax and N(0, 1) amplitudes:
    periodic in x and y, cos(m pi z / lz) in z (the walls' natural condition)."""
    out = np.zeros(np.broadcast(x, y, z).shape)
    done = 0
    while done < nmodes:
        a, b, m = rng.integers(-kmax, kmax + 1), rng.integers(-kmax, kmax + 1), rng.integers(0, kmax + 1)
        kx, ky, kz = 2 * np.pi * a / lx, 2 * np.pi * b / ly, np.pi * m / lz
        if not (0 < kx * kx + ky * ky + kz * kz <= kmax * kmax):
            continue
        amp, ph = rng.standard_normal(), rng.uniform(0, 2 * np.pi)
        out += amp * np.cos(kx * x + ky * y + ph) * np.cos(kz * z)
        done += 1
    return out


def event_ms(L, h, fn, reps):
    """Mean device time of fn() over reps calls, CUDA events on the context's stream."""
    L.pmpic_event_record(h, 4)
    for _ in range(reps):
        fn()
    L.pmpic_event_record(h, 5)
    ms = C.c_float()
    L.pmpic_event_elapsed(h, 4, 5, C.byref(ms))
    return ms.value / reps


def run_interp(args):
    """Interpolation microbenchmark: 128^3 grid, 8 parcels per cell at seeded
    uniform-random positions; par2grid of 4 fields and grid2par of 6 fields,
    FP64 vs the mixed form, in the given (random) slot order and after the
    parcels are renumbered into cell order; binning checked against the oracle."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    import pmpic_b200 as pm
    from oracle import Oracle
    G = args.grid if args.grid != 256 else 128
    P = 8 * G ** 3
    rng = np.random.default_rng(2)
    x = rng.uniform(0, 2 * np.pi, P)
    y = rng.uniform(0, 2 * np.pi, P)
    z = rng.uniform(0, np.pi, P)
    vol = np.full(P, (2 * np.pi / G) ** 2 * (np.pi / G) / 8)
    frng = np.random.default_rng(3)
    fields = {q: fourier_field(x, y, z, 16, 8, frng) for q in ("p", "q", "r", "b")}
    zg, yg, xg = np.meshgrid(np.arange(G + 1) * (np.pi / G), np.arange(G) * (2 * np.pi / G),
                             np.arange(G) * (2 * np.pi / G), indexing="ij")
    grids = {g: fourier_field(xg, yg, zg, 16, 8, frng) for g in ("u", "v", "w", "dp", "dq", "dr")}
    o = Oracle(G, G, G, 2 * np.pi, 2 * np.pi, np.pi, max_parcels=P, threads=os.cpu_count() or 1)
    o.set_parcels(x=x, y=y, z=z, vol=vol)
    ref_cells = o.cache_weights()
    o.close()
    p4, g6 = ["p", "q", "r", "b"], ["u", "v", "w", "dp", "dq", "dr"]
    props6 = ["dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt"]
    res, outs = {}, {}
    for prec in ("fp64", "mixed"):
        ctx = pm.Context(G, G, G, 2 * np.pi, 2 * np.pi, np.pi, max_parcels=P, device=local, precision=prec)
        ctx.upload(x=x, y=y, z=z, vol=vol, **fields, tag=np.arange(P, dtype=np.float64))
        for g in g6:
            ctx.set_grid(g, grids[g])
        L, h = pm.lib(), ctx._h
        mism = int(np.count_nonzero(ctx.cell_ids() != ref_cells))
        r = {"binning_mismatches_vs_oracle": mism}
        for order in ("random", "cell"):
            if order == "cell":
                ctx.sort_parcels()
            ctx.par2grid_multi(p4, p4)
            ctx.grid2par_multi(g6, props6)
            t_p = event_ms(L, h, lambda: ctx.par2grid_multi(p4, p4), args.steps)
            t_g = event_ms(L, h, lambda: ctx.grid2par_multi(g6, props6), args.steps)
            r[order] = {"par2grid4_ms": t_p, "grid2par6_ms": t_g, "pair_parcels_per_s": P / ((t_p + t_g) / 1e3)}
            if order == "random":
                outs[prec] = {"grids": {q: ctx.grid(q) for q in p4}, "gath": {q: ctx.get(q) for q in props6}}
        res[prec] = r
        ctx.close()
    err = {}
    for q in p4:
        a, b = outs["mixed"]["grids"][q], outs["fp64"]["grids"][q]
        err["par2grid_" + q + "_rel_l2"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    for q in props6:
        a, b = outs["mixed"]["gath"][q], outs["fp64"]["gath"][q]
        err["grid2par_" + q + "_rel_l2"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    peak, peak_kind = hbm_peak()
    # algorithmic bytes of the pair per parcel: par2grid reads positions (FP64 24 B; mixed: 3 int + 3 float
    # cell slots, 24 B) + vol + 4 fields, writes the cell and (FP64) 3 offsets; grid2par reads the cell /
    # positions and writes 6 values; plus 4 grids written and 6 read
    bp = {"fp64": 24 + 28 + 8 + 32 + 28 + 48, "mixed": 24 + 4 + 4 + 16 + 24 + 24}
    nph = (G + 1) * G * G
    line = {"workload": "interp", "metric": "interpolation pairs (par2grid 4 fields + grid2par 6 fields), parcels/s",
            "unit": "parcels/s", "higher_is_better": True, "value": res["mixed"]["cell"]["pair_parcels_per_s"],
            "config": {"grid": G, "parcels": P, "positions": "uniform random, seed 2",
                       "fields": "16 random Fourier modes |k|<=8, N(0,1) amplitudes, seed 3",
                       "timing": f"CUDA events, mean of {args.steps} calls after one warm-up; par2grid includes the binning and cell sort"},
            "fp64": res["fp64"], "mixed": res["mixed"], "mixed_vs_fp64": err,
            "roofline": {prec: {order: {"achieved_gbs": (bp[prec] * P + (10 * nph * (8 if prec == "fp64" else 4)))
                                        / ((res[prec][order]["par2grid4_ms"] + res[prec][order]["grid2par6_ms"]) / 1e3) / 1e9,
                                        "peak_gbs": peak}
                                for order in ("random", "cell")} for prec in ("fp64", "mixed")},
            "peak_source": peak_kind}
    print(json.dumps(line), flush=True)
    return 0


def run_vort2vel(args):
    """vort2vel's inversion alone at 256^3 on a random divergence-free vorticity
    (k^-5/3 spectrum cut at k = 64, unit RMS, wall conditions): FP64 vs the mixed
    form (FP32 transforms, FP64 zero mode), errors against the FP64 oracle."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    import pmpic_b200 as pm
    from oracle import Oracle
    G = args.grid
    p, q, r = pm.random_vorticity(G, G, G, kmax=64, seed=4)
    res, vel = {}, {}
    for prec in ("fp64", "mixed"):
        ctx = pm.Context(G, G, G, 2 * np.pi, 2 * np.pi, np.pi, max_parcels=16, device=local, precision=prec)
        L, h = pm.lib(), ctx._h

        def load():
            ctx.set_grid("p", p)
            ctx.set_grid("q", q)
            ctx.set_grid("r", r)
        load()
        ctx.vort2vel_grids()
        vel[prec] = {k: ctx.grid(k) for k in ("u", "v", "w")}
        load()
        ctx.vort2vel_grids()  # warm-up
        res[prec] = {"ms_per_call": event_ms(L, h, ctx.vort2vel_grids, args.steps)}
        ctx.close()
    o = Oracle(G, G, G, 2 * np.pi, 2 * np.pi, np.pi, max_parcels=16, threads=os.cpu_count() or 1)
    o.set_grid("p", p)
    o.set_grid("q", q)
    o.set_grid("r", r)
    t0 = time.perf_counter()
    o.vort2vel_grids()
    t_cpu = time.perf_counter() - t0
    ref = {k: o.grid(k) for k in ("u", "v", "w")}
    o.close()
    err = {}
    for prec in ("fp64", "mixed"):
        for k in ("u", "v", "w"):
            d = vel[prec][k] - ref[k]
            err[f"{prec}_{k}_rel_l2"] = float(np.linalg.norm(d) / np.linalg.norm(ref[k]))
            err[f"{prec}_{k}_max_abs"] = float(np.abs(d).max())
    nspec = (G + 1) * (G + 2) * (G + 2)
    nph = (G + 1) * G * G
    peak, peak_kind = hbm_peak()
    roof = {}
    for prec in ("fp64", "mixed"):
        w = 8 if prec == "fp64" else 4
        alg = w * 12 * nph  # 3 grids in, 9 out (corrected p, q, r; u, v, w; u_s, v_s, w_s)
        passes = w * 9 * 4 * nspec  # 9 transforms x 2 passes x (read + write)
        t = res[prec]["ms_per_call"] / 1e3
        roof[prec] = {"algorithmic_gbs": alg / t / 1e9, "pass_model_gbs": passes / t / 1e9, "peak_gbs": peak}
    line = {"workload": "vort2vel", "metric": "vort2vel inversion at 256^3, ms per call", "unit": "ms",
            "higher_is_better": False, "value": res["mixed"]["ms_per_call"],
            "config": {"grid": G, "vorticity": "divergence-free, k^-5/3 energy spectrum, |k|<=64, unit RMS, seed 4",
                       "timing": f"CUDA events, mean of {args.steps} calls after one warm-up"},
            "fp64": res["fp64"], "mixed": res["mixed"], "error_vs_oracle": err, "roofline": roof,
            "peak_source": peak_kind,
            "cpu_baseline": {"value": 1e3 * t_cpu, "unit": "ms", "cores": os.cpu_count() or 1, "kind": "port",
                             "sample": "one call of the C++ restatement (oracle) at the same size"}}
    print(json.dumps(line), flush=True)
    return 0


def ensemble_members(n, seed=999):
    """The config-4 ensemble: per member a grid drawn from {32, 48, 64, 96, 128}^3,
    thermal radius U[0.25, 0.5], excess U[0.5, 1.5], humidity fraction
    U[0.8, 1.0] of the surface saturation, own seed 1000+m, 8 parcels per cell."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        G = int(rng.choice([32, 48, 64, 96, 128]))
        out.append(dict(G=G, radius=float(rng.uniform(0.25, 0.5)), excess=float(rng.uniform(0.5, 1.5)),
                        h_in=float(rng.uniform(0.8, 1.0)), seed=1000 + m, dt=0.32 / G))
    return out


def run_ensemble(args):
    """Batched ensemble of independent plumes in the mixed form: the members run
    one after another (concurrency 1, default tiles) and then batched (tuned
    tiles, concurrent members), each from the same initial state for the same
    number of steps; then every member against the same plume on the FP64 path.
    Under torchrun the members are spread over the ranks by cost
    (pmpic_b200.assign_members; no exchange between ranks): each rank runs its
    share both ways, and the aggregate is all work over the max device time."""
    rank, world, local = dist_env()
    # 64 member streams: let the device give them more hardware work queues
    # than the default 8, so independent streams do not wait on one another
    # (read once, when this process creates its CUDA context, which is below)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    import torch
    torch.cuda.set_device(local)
    import pmpic_b200 as pm
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
        pg = dist
    spec_all = ensemble_members(args.members)
    steps = args.ens_steps
    mine = pm.assign_members([8 * m["G"] ** 3 * steps for m in spec_all], world)[rank]
    spec = [spec_all[i] for i in mine]

    def ic(m):
        return pm.thermal_parcels(m["G"], m["G"], m["G"], radius=m["radius"], excess=m["excess"],
                                  h_in=m["h_in"], seed=m["seed"])
    counts = [8 * m["G"] ** 3 for m in spec]
    cfgs = [dict(nx=m["G"], ny=m["G"], nz=m["G"], dtm=m["dt"], dtmax=m["dt"], max_parcels=int(1.15 * c),
                 precision="mixed") for m, c in zip(spec, counts)]
    ens = pm.Ensemble(cfgs, device=local) if spec else None
    members = ens.members if ens else []

    def load():
        for mem, m in zip(members, spec):
            mem.upload(**ic(m))
        torch.cuda.synchronize()

    def work(n_before):
        n_after = [mem.n for mem in members]
        return sum(0.5 * (a + b) for a, b in zip(n_before, n_after)) * steps

    ms_seq = ms_bat = ms_tune = 0.0
    w_seq = w_bat = 0.0
    threads, xseg = 0, []
    errs = []
    if ens:
        load()
        ens.set_concurrency(1)
        n0 = [mem.n for mem in members]
        ms_seq = ens.step(steps)
        w_seq = work(n0)
        load()
        for mem in members:
            pm.lib().pmpic_set_p2g_segment(mem._h, 64)
        ens.autotune()
        # the host concurrency is tuned online (one step per candidate); those steps
        # run before the timed window, then the initial state is loaded again
        ens.set_concurrency(0)
        ms_tune = ens.step(6)
        load()
        n0 = [mem.n for mem in members]
        ms_bat = ens.step(steps)
        w_bat = work(n0)
        threads, xseg = ens.tuning()
        grids = [{g: mem.grid(g) for g in ("u", "v", "w")} for mem in members[:args.error_members]]
        n_mixed = [mem.n for mem in members]
        ens.close()
        for i, m in enumerate(spec[:args.error_members]):
            G = m["G"]
            c = pm.Context(G, G, G, 2 * np.pi, 2 * np.pi, np.pi, dtm=m["dt"], dtmax=m["dt"],
                           max_parcels=int(1.15 * counts[i]), device=local)
            c.upload(**ic(m))
            c.step(steps)
            e = {"member": mine[i], "grid": G, "n_mixed": n_mixed[i], "n_fp64": c.n}
            for g in ("u", "v", "w"):
                ref = c.grid(g)
                e[g + "_rel_l2"] = float(np.linalg.norm(grids[i][g] - ref) / max(np.linalg.norm(ref), 1e-300))
            errs.append(e)
            c.close()
    # every rank takes the same collective steps, members or not
    t_seq, w_seq_all = combine(ms_seq / 1e3, w_seq, pg, "cuda")
    t_bat, w_bat_all = combine(ms_bat / 1e3, w_bat, pg, "cuda")
    emax_local = max((max(e["u_rel_l2"], e["v_rel_l2"], e["w_rel_l2"]) for e in errs), default=0.0)
    emax, _ = combine(emax_local, 0.0, pg, "cuda")
    if pg:
        pg.barrier()
    if rank == 0:
        seq_v, bat_v = w_seq_all / t_seq, w_bat_all / t_bat
        sizes = {}
        for m, s_ in zip(spec, xseg):
            sizes.setdefault(str(m["G"]), s_)
        line = {"workload": "ensemble", "metric": "aggregate parcel-RK4-steps/s of the batched ensemble",
                "unit": UNIT, "higher_is_better": True, "value": bat_v, "n_gpus": world,
                "config": {"members": len(spec_all), "steps": steps, "precision": "mixed",
                           "grids": {str(G): sum(1 for m in spec_all if m["G"] == G) for G in (32, 48, 64, 96, 128)},
                           "parcels_initial": int(sum(8 * m["G"] ** 3 for m in spec_all)), "dt": "0.32 / grid size",
                           "members_per_rank": "by cost (parcels x steps), largest first to the least-loaded rank",
                           "timing": "device time from the first member's start to the last member's end "
                                     "(events across all member streams; max over ranks); the batched run is "
                                     "timed after its tuning (row-pass segments per grid size, then six steps "
                                     "trying 2-64 host threads, then the initial state loaded again)"},
                "cuda_device_max_connections": os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS"),
                "sequential": {"value": seq_v, "ms": 1e3 * t_seq, "concurrency": 1, "par2grid_segment": 64},
                "batched": {"value": bat_v, "ms": 1e3 * t_bat, "concurrency": threads,
                            "par2grid_segment_by_grid": sizes, "tuning_ms": ms_tune},
                "batched_over_sequential": bat_v / seq_v,
                "error_vs_fp64": {"members_rank0": errs, "max_rel_l2_all_ranks": emax}}
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--capacity", type=float, default=2.25, help="max_parcels / initial parcels")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-grid", type=int, default=256,
                    help="grid of the CPU legs (the reference arm and cpu_baseline)")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--p2g-segment", type=int, default=0,
                    help="columns per x segment of the par2grid row pass (0: the library's default)")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: time FP64 then the mixed form (the headline value), and compare them")
    ap.add_argument("--error-steps", type=int, default=100,
                    help="total steps per form before the gridded velocities are compared (0: no check)")
    ap.add_argument("--members", type=int, default=64, help="ensemble workload: members")
    ap.add_argument("--ens-steps", type=int, default=50, help="ensemble workload: steps per member")
    ap.add_argument("--error-members", type=int, default=64,
                    help="ensemble workload: members compared with the FP64 path")
    ap.add_argument("--workload", default="plume", choices=["plume", "interp", "vort2vel", "ensemble"],
                    help="plume: the headline step; interp: the interpolation microbenchmark (128^3); "
                         "vort2vel: the inversion alone (256^3); ensemble: 64 plumes of uneven sizes")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "interp":
        return run_interp(args)
    if args.workload == "vort2vel":
        return run_vort2vel(args)
    if args.workload == "ensemble":
        return run_ensemble(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
