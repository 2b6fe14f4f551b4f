#!/usr/bin/env python
"""Benchmark: particle-steps/s of the B200 ROMSPath particle step.

Workload (the plain-method-at-scale configuration): one ROMS grid of
512 x 384 rho points x 30 s-levels (Vtransform 2 / Vstretching 4), 8 %
seeded island land mask, analytic double gyre + M2 tide fields supplied in
FP32 with a 0.05 m/s surface Stokes drift (e-folding 5 m) added on upload,
horizontal diffusivity Kh = 1 m^2/s, the vertical random displacement model
on a 30 s sub-step, 1,048,576 particles released uniformly in (x, y, s),
idt = 300 s, hourly frames.  Inputs are synthetic (no ocean-model output on
this machine).

Three forms of the step are timed on it, one after the other:
  mixed  (headline) FP16 u/v/w/AKs with per-level scales, FP32 positions
         with Kahan compensation, FP64 age and smoothing spline;
  f32    FP64 arithmetic on FP32-stored fields (bit-identical to the oracle);
  f64    plain FP64 (FP64-stored fields; bit-identical to the oracle).

One benchmark step = one hydrodynamic frame interval = 12 internal steps
(update_particles calls) over all particles.

  value   device-resident: frames already in the ring, particles in HBM;
          CUDA events on the library's compute stream.
  e2e     through the C ABI with page-locked host buffers: every step
          uploads one frame (FP32 + Stokes) and reads the particle state
          back (the dataOutput columns), host clock between device syncs;
          the next frame's upload overlaps the current interval's steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  python bench.py --error-study [--workload cfg3 --days 10 --deterministic]

For N > 1 (torchrun), each rank advances its own 1,048,576 particles
(replicas of the fields, no collective on the data path: weak scaling);
the reported time is the max over ranks.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from romspath_b200 import schedule, synth  # noqa: E402

WORKLOAD_DESC = ("cfg2: 512x384x30 ROMS grid, 8% islands, FP32 u/v/w/AKs/zeta frames + Stokes, "
                 "Kh=1 m^2/s, VTurb dt_turb=30 s, RK4 idt=300 s")
WORKLOAD_DESCS = {
    "cfg2": WORKLOAD_DESC,
    "cfg1": "cfg1: 130x98x20 ROMS grid, land corner, FP64 frames, HTurb off, VTurb dt_turb=30 s, RK4 idt=300 s",
    "cfg3": "cfg3: config 1's 130x98x20 grid (FP64 frames; FP16 in the mixed form), HTurb off, VTurb dt_turb=30 s, "
            "RK4 idt=300 s, 4,194,304 particles",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2")
    ap.add_argument("--particles", type=int, default=None)
    ap.add_argument("--scale", type=float, default=1.0, help="--batched: fraction of the particle counts")
    ap.add_argument("--cpu-sample", type=int, default=32768, help="particles in the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--form", default="mixed", choices=["mixed", "exact"],
                    help="headline form: mixed precision (default) or exact FP64 arithmetic on the workload's "
                         "field storage; the other forms are timed beside it")
    ap.add_argument("--resort", type=int, default=12,
                    help="re-sort the particle state by grid and cell every this many internal steps "
                         "(0: never; results are unchanged)")
    ap.add_argument("--error-study", action="store_true",
                    help="instead of timing: run the exact and the mixed form in lockstep on the same "
                         "frames and noise and report the mixed form's position / profile error")
    ap.add_argument("--days", type=float, default=10.0, help="error study length")
    ap.add_argument("--kernel-form", default="fused", choices=["fused", "split", "smem", "fused-noprefetch"],
                    help="kernel form of the timed forms (rp_set_kernel_form; smem and fused-noprefetch: mixed "
                         "forms only, the exact forms run those fused)")
    ap.add_argument("--param", action="append", default=[], metavar="KEY=VALUE",
                    help="override one of the workload's run parameters in the timed forms (e.g. vturb_on=0, "
                         "sub=2, deltat=300) to time parts of the step; the line's config lists the overrides")
    ap.add_argument("--error-days", type=float, default=1.0,
                    help="length of the headline line's lockstep error check of the mixed forms (0: none)")
    ap.add_argument("--error-particles", type=int, default=65536,
                    help="particles of the headline line's lockstep error check")
    ap.add_argument("--batched", action="store_true",
                    help="instead of the single-grid workload: batched nested grids (400x300x30 parent, 3x and 5x "
                         "children; 3M / 800k / 200k particles + 16 release ensembles), one launch per internal "
                         "step over all grids, frame intervals as CUDA graphs, launch settings autotuned")
    ap.add_argument("--config1", action="store_true",
                    help="instead of timing: the reference's CPU-runnable case end to end (130x98x20 grid, "
                         "10,000 particles, 2 days), the exact GPU form against the CPU restatement of the "
                         "reference on the host cores, final states compared bit for bit")
    ap.add_argument("--adjoint", action="store_true",
                    help="instead of timing the step: the adjoint pair on the 130x98x20 grid (262,144 particles, "
                         "3 days, checkpoints every 48 steps): forward / backward / tangent times and the "
                         "finite-difference agreement")
    ap.add_argument("--features", action="store_true",
                    help="cost of the diagnostics, WETDRY, behave and the output record on the exact step, "
                         "and the init lookup (LL2ij, nest maps) against the oracle")
    ap.add_argument("--variants", default=None,
                    help="--features: comma-separated step variants to run (default all); 'none' skips the steps")
    ap.add_argument("--no-init", action="store_true", help="--features: skip the LL2ij and nest-map timings")
    ap.add_argument("--deterministic", action="store_true", help="error study with turbulence off")
    ap.add_argument("--mixed-kind", default="mixed", choices=["mixed", "mixed-i16"],
                    help="16-bit field storage of the mixed form: FP16 (default) or int16 fixed point")
    ap.add_argument("--perturb", type=float, default=0.0,
                    help="error study of the exact form against itself with initial x, y moved by up to "
                         "this many grid cells (the flow's own sensitivity)")
    return ap.parse_args()


def measured_peaks(path=None):
    """HBM copy bandwidth (GB/s) for the roofline: `hbm_gbs` of the measured
    peaks file (top level, or in nested objects and lists; a positive number,
    not a boolean), else the pool's earlier measurement of 6.65 TB/s."""
    p = path or os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
        except Exception:
            d = None
        stack = [d]
        while stack:
            x = stack.pop()
            if isinstance(x, dict):
                v = x.get("hbm_gbs")
                if isinstance(v, (int, float)) and not isinstance(v, bool) and v > 0:
                    return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
                stack.extend(reversed(list(x.values())))
            elif isinstance(x, list):
                stack.extend(reversed(x))
    return 6650.0, "fallback (6.65 TB/s)"


def parse_params(items, params):
    """--param KEY=VALUE overrides of the workload's run parameters; KEY must
    be one of them and VALUE is read as a number (int where it is one)."""
    out = {}
    for it in items:
        if "=" not in it:
            raise SystemExit(f"--param wants KEY=VALUE, got {it!r}")
        k, v = it.split("=", 1)
        if k not in params:
            raise SystemExit(f"--param: unknown parameter {k!r} (one of {sorted(params)})")
        try:
            val = int(v)
        except ValueError:
            val = float(v)
        out[k] = val
    return out


def profile_traffic(workload, kernel, key="dram_bytes_per_launch"):
    """DRAM (or, with key="lts_bytes_per_launch", L2) bytes per launch of
    `kernel` from the committed ncu summary of the same workload, or None
    when no summary covers that kernel."""
    p = os.path.join(ROOT, "profiles", f"step_{workload}_traffic.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
        except Exception:
            return None
        k = d.get("kernels", {}).get(kernel)
        if k:
            return k.get(key)
    return None


def profile_fp64(workload, kernel):
    """FP64 arithmetic of one launch of `kernel` from the committed ncu
    counts of the same workload (DADD + DMUL + 2 DFMA thread instructions,
    fp64 pipe activity), or None when no summary covers that kernel."""
    p = os.path.join(ROOT, "profiles", f"step_{workload}_fp64.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
        except Exception:
            return None
        return d.get("kernels", {}).get(kernel)
    return None


# B200 FP64 (vector and tensor core) nominal peak: 296 TFLOP/s per 8-GPU
# DGX B200 system; no measured FP64 peak exists for this pool
FP64_PEAK_NOMINAL_TFLOPS = 37.0


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # the timed region starts once sampling runs (first line written;
        # at most 3 s)
        t0 = time.time()
        while time.time() - t0 < 3.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def pinned_like(a: np.ndarray):
    """A Fortran-ordered copy of ``a`` in page-locked host memory."""
    import torch
    t = torch.empty(a.size, dtype={np.float32: torch.float32, np.float64: torch.float64}[a.dtype.type],
                    pin_memory=True)
    buf = t.numpy()
    buf[:] = np.asfortranarray(a).ravel(order="F")
    out = buf.reshape(a.shape, order="F")
    return out, t


def pinned_empty(n, dtype):
    import torch
    tdt = {np.float64: torch.float64, np.int32: torch.int32, np.uint32: torch.int32}[dtype]
    t = torch.empty(n, dtype=tdt, pin_memory=True)
    return t.numpy().view(dtype), t


# ------------------------------------------------------------------ CPU arm

def cpu_timing(workload, npart, steps, warmup, threads):
    """The CPU restatement of the reference step (oracle) on the host cores:
    `steps` frame intervals of 12 internal steps over `npart` particles."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import oracle as O
    spec = synth.config_spec(workload)[0]
    grid = synth.make_grid(spec)
    params = synth.config_params(workload)
    frames = {k: synth.stored_frame(synth.make_frame(spec, grid, (k - 1) * 3600.0), spec.field_dtype, spec.stokes)
              for k in (1, 2, 3)}
    m = O.OracleModel([spec], [grid], params)
    for slot, k in ((1, 1), (2, 2), (3, 3)):
        m.set_frame(1, slot, frames[k])
    rel = synth.uniform_release(spec, grid, synth.make_frame(spec, grid, 0.0), npart, seed=0)
    m.init_particles(rel)
    ext = list(schedule.external_steps(2.0, 3600, 300))[2]      # ets = 3 pattern
    t_total, n_steps = 0.0, 0
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        for it in ext.internal:
            m.step(it.ex, it.ix, it.ets, 1, 2, 3, noise="philox", seed=7, step_index=s * 12 + it.its,
                   nthreads=threads)
        dt = time.perf_counter() - t0
        if s >= warmup:
            t_total += dt
            n_steps += 1
    return npart * 12 * n_steps / t_total, t_total / max(n_steps, 1)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    npart = min(args.cpu_sample, 16384)
    val, per = cpu_timing(args.workload, npart, args.steps, args.warmup, threads)
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": val, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD_DESCS.get(args.workload, args.workload),
                                        "step": "one frame interval = 12 internal steps",
                                        "sample_particles": npart},
        "cpu_baseline": {"value": val, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{args.workload} grid, {npart} particles x 12 internal steps per step, "
                                   f"Philox noise, {threads} OpenMP threads (oracle restatement; the "
                                   f"Fortran reference cannot be built here)"},
        "e2e": {"value": val, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ error study

MOVED = (1.0, float(np.float32(1.1)), float(np.float32(1.2)))


def error_stats(ref, mix, spec):
    """Mixed-form error against the exact form: horizontal position (grid
    cells) and depth (m) over particles active in both, the vertical
    concentration profile (20 bins of the water-column fraction) and the
    horizontal one (cells of 8 x 8 rho points), as L1 distances of the
    normalised histograms."""
    ok = np.isin(ref["status"], MOVED) & np.isin(mix["status"], MOVED)
    dh = np.hypot(mix["x"] - ref["x"], mix["y"] - ref["y"])[ok]
    dz = (mix["z"] - ref["z"])[ok]
    depth = (ref["bath"] + ref["zeta"])[ok]
    frac = lambda st: ((st["z"] + st["bath"]) / (st["bath"] + st["zeta"]))[ok]
    hv = [np.histogram(frac(st), bins=20, range=(0.0, 1.0))[0] for st in (ref, mix)]
    bx, by = np.arange(0, spec.xi_rho + 8, 8), np.arange(0, spec.eta_rho + 8, 8)
    hh = [np.histogram2d(st["x"][ok], st["y"][ok], bins=(bx, by))[0] for st in (ref, mix)]
    n = max(int(ok.sum()), 1)
    return {"particles_compared": int(ok.sum()), "status_agreement": float(np.mean(ref["status"] == mix["status"])),
            "rms_position_cells": float(np.sqrt(np.mean(dh ** 2))) if dh.size else None,
            "median_position_cells": float(np.median(dh)) if dh.size else None,
            "p99_position_cells": float(np.percentile(dh, 99)) if dh.size else None,
            "max_position_cells": float(dh.max()) if dh.size else None,
            "rms_depth_m": float(np.sqrt(np.mean(dz ** 2))) if dz.size else None,
            "rms_depth_frac_of_column": float(np.sqrt(np.mean((dz / depth) ** 2))) if dz.size else None,
            "vertical_profile_L1": float(np.abs(hv[0] - hv[1]).sum() / n),
            "horizontal_profile_L1": float(np.abs(hh[0] - hh[1]).sum() / n)}


def lockstep_error(wl, kinds, days, npart, deterministic=False):
    """The mixed forms `kinds` and the exact form stepped in lockstep on one
    GPU for `days` (same grid, hourly frames, release and Philox noise),
    error_stats of each against the exact form at the end."""
    from romspath_b200 import Tracker
    spec = synth.config_spec(wl)[0]
    grid = synth.make_grid(spec)
    params = dict(synth.config_params(wl))
    if deterministic:
        params.update(vturb_on=0, hturb_on=0)
    cache = {}

    def frame(k):
        if k not in cache:
            cache[k] = synth.make_frame(spec, grid, (k - 1) * float(params["dt"]))
            for old in [j for j in cache if j < k - 3]:
                del cache[old]
        return cache[k]

    rel = synth.uniform_release(spec, grid, frame(1), npart, seed=0)
    forms = {"exact": spec.field_dtype, **{k: k for k in kinds}}
    T = {f: Tracker([spec], [grid], params, numpar=npart, field_dtype=d, stokes=spec.stokes, seed=7, resort=12)
         for f, d in forms.items()}
    for (k, slot) in schedule.initial_loads():
        for t in T.values():
            t.upload_frame(1, slot, frame(k))
    for t in T.values():
        t.locate(rel, t_b=1)
    for ext in schedule.external_steps(days, int(params["dt"]), int(params["idt"])):
        for (k, slot) in ext.loads:
            for t in T.values():
                t.upload_frame(1, slot, frame(k))
        for t in T.values():
            t.step_n(ext.internal)
    st = {f: t.get_particles() for f, t in T.items()}
    for t in T.values():
        t.close()
    return {k: error_stats(st["exact"], st[k], spec) for k in kinds}


def error_study(args):
    """The mixed form against the exact FP64 form (bit-identical to the CPU
    restatement of the reference, by the parity tests) on one GPU: same
    grid, frames, release and Philox noise, stepped in lockstep."""
    from romspath_b200 import Tracker
    wl = args.workload
    spec = synth.config_spec(wl)[0]
    grid = synth.make_grid(spec)
    params = dict(synth.config_params(wl))
    if args.deterministic:
        params.update(vturb_on=0, hturb_on=0)
    npart = args.particles or 65536
    cache = {}

    def frame(k):
        if k not in cache:
            cache[k] = synth.make_frame(spec, grid, (k - 1) * float(params["dt"]))
            for old in [j for j in cache if j < k - 3]:
                del cache[old]
        return cache[k]

    rel = synth.uniform_release(spec, grid, frame(1), npart, seed=0)
    forms = {"exact": spec.field_dtype, "mixed": spec.field_dtype if args.perturb > 0 else args.mixed_kind}
    T = {f: Tracker([spec], [grid], params, numpar=npart, field_dtype=d, stokes=spec.stokes, seed=7)
         for f, d in forms.items()}
    for (k, slot) in schedule.initial_loads():
        for t in T.values():
            t.upload_frame(1, slot, frame(k))
    for t in T.values():
        t.locate(rel, t_b=1)
    if args.perturb > 0:
        st = T["mixed"].get_particles()
        rng = np.random.default_rng(1)
        dx, dy = rng.uniform(-args.perturb, args.perturb, (2, npart))
        T["mixed"].set_particles(st["x"] + dx, st["y"] + dy, st["z"], rel.dob, st["age"], st["status"], st["gid"],
                                 st["isin"])
    out = {"mode": "error-study", "workload": wl, "days": args.days, "particles": npart,
           "compared_form": (f"exact, initial x/y perturbed by U(-{args.perturb}, {args.perturb}) cells"
                             if args.perturb > 0 else args.mixed_kind),
           "turbulence": "off" if args.deterministic else "as configured (same Philox noise in both forms)",
           "reference_form": f"exact FP64 arithmetic on {spec.field_dtype}-stored fields", "checkpoints": []}
    t0 = time.time()
    day_steps = 86400 // int(params["idt"])
    done = 0
    for ext in schedule.external_steps(args.days, int(params["dt"]), int(params["idt"])):
        for (k, slot) in ext.loads:
            for t in T.values():
                t.upload_frame(1, slot, frame(k))
        for it in ext.internal:
            for t in T.values():
                t.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            done += 1
            if done % day_steps == 0:
                st = {f: t.get_particles() for f, t in T.items()}
                e = error_stats(st["exact"], st["mixed"], spec)
                e["day"] = done / day_steps
                out["checkpoints"].append(e)
    out["wall_s"] = time.time() - t0
    for t in T.values():
        t.close()
    print(json.dumps(out), flush=True)


# ----------------------------------------------------- batched nested grids

def batched_run(args):
    """Config 4: every grid and ensemble advanced by one launch per internal
    step (particles carry their grid id; hand-off moves them between
    grids), each frame interval's 12 steps captured as one CUDA graph, the
    kernel form, re-sort interval and particles per thread autotuned on the
    run (the tuner's figures are ns per active particle-step)."""
    import torch
    from romspath_b200 import Tracker
    from romspath_b200.autotune import tune
    torch.cuda.set_device(0)
    specs = synth.config_spec("cfg4")
    grids = [synth.make_grid(sp) for sp in specs]
    params = synth.config_params("cfg4")
    scl, off = synth.nest_maps(specs)
    counts = [max(1, int(c * args.scale)) for c in synth.CONFIG4_COUNTS]
    rel = synth.batched_release(specs, grids, counts, n_ensembles=16, ens_min=max(1, int(1000 * args.scale)),
                                ens_max=max(2, int(500_000 * args.scale)), seed=0)
    n = rel.z.shape[0]
    nframes = 4
    frames = [[synth.make_frame(sp, gr, k * 3600.0) for k in range(nframes)] for sp, gr in zip(specs, grids)]
    exts = list(schedule.external_steps(30.0, int(params["dt"]), int(params["idt"])))
    out = {"mode": "batched", "workload": "cfg4: parent 400x300x30 (8% islands) + child A 240x180x30 (3x) + child "
                                         "B 300x250x30 (5x), children with a 0.1 m/s eddy field; FP32 frames + "
                                         "Stokes; Kh = 1 m^2/s; VTurb dt_turb = 30 s",
           "particles": n, "released_over": {"child_B": counts[0], "child_A": counts[1], "parent": counts[2],
                                             "ensembles": int(n - sum(counts))}}
    forms = {}
    for form in (args.mixed_kind, "f32"):
        T = Tracker(specs, grids, params, numpar=n, field_dtype=form, stokes=True, seed=7, scl=scl, off=off,
                    resort=12)
        for k, slot in enumerate((1, 2, 3)):
            for ng in range(1, len(specs) + 1):
                T.upload_frame(ng, slot, frames[ng - 1][k])
        T.locate(rel, t_b=1)
        st0 = T.get_particles()
        pos = [2]

        def interval(graph=True):
            e = exts[pos[0]]
            for (k, slot) in e.loads:
                for ng in range(1, len(specs) + 1):
                    T.upload_frame(ng, slot, frames[ng - 1][(k - 1) % nframes])
            if graph:
                T.step_n(e.internal)
                ms, _ = T.last_step_stats()
            else:
                ms = 0.0
                for it in e.internal:
                    T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
                    ms += T.last_step_stats()[0]
            active = int(sum(np.sum(rel.dob < it.ix[2]) for it in e.internal))
            pos[0] += 1
            return ms, active

        r = {}
        if form == args.mixed_kind:
            # ns per active particle-step: releases make the active count
            # grow from one interval to the next
            r["autotune"] = tune(T, lambda: (lambda m, a: 1e6 * m / max(a, 1))(*interval()))
        interval()
        ms_g, act, ms_p = [], 0, []
        for _ in range(args.steps):
            m, a = interval(graph=True)
            ms_g.append(m)
            act += a
        for _ in range(2):
            ms_p.append(interval(graph=False)[0])
        st = T.get_particles()
        T.close()
        own0 = np.bincount(st0["gid"].astype(int), minlength=len(specs) + 1)[1:]
        own = np.bincount(st["gid"].astype(int), minlength=len(specs) + 1)[1:]
        r.update({"ms_per_interval_graph": float(np.median(ms_g)), "ms_per_interval_stepwise": float(np.median(ms_p)),
                  "active_particle_steps_per_s": act / (sum(ms_g) / 1e3),
                  "owned_by_grid_at_start": {"child_B": int(own0[0]), "child_A": int(own0[1]), "parent": int(own0[2])},
                  "owned_by_grid_at_end": {"child_B": int(own[0]), "child_A": int(own[1]), "parent": int(own[2])},
                  "grid_changes": int(np.sum(st["gid"] != st0["gid"]))})
        forms[form] = r
    out["forms"] = forms
    out["speedup_mixed_over_exact"] = forms[args.mixed_kind]["active_particle_steps_per_s"] / \
        forms["f32"]["active_particle_steps_per_s"]
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------- config 1

def config1_run(args):
    """Config 1 end to end: hourly frames uploaded as the driver reads them,
    576 internal steps of 10,000 particles; the exact GPU form (FP64) and
    the oracle (FP64 C restatement of the reference, OpenMP over particles,
    same Philox noise) from the same release; then the serial form of the
    reference's noise (one MT19937 stream) on the oracle, single-threaded,
    on a 1,000-particle sample."""
    import torch
    from romspath_b200 import Tracker
    from oracle import oracle as O
    torch.cuda.set_device(0)
    spec = synth.config_spec("cfg1")[0]
    grid = synth.make_grid(spec)
    params = synth.config_params("cfg1")
    npart = args.particles or synth.CONFIG_PARTICLES["cfg1"]
    days = synth.CONFIG_DAYS["cfg1"]
    frames = {}

    def frame(k):
        if k not in frames:
            frames[k] = synth.make_frame(spec, grid, (k - 1) * float(params["dt"]))
        return frames[k]

    rel = synth.uniform_release(spec, grid, frame(1), npart, seed=0)
    exts = list(schedule.external_steps(days, int(params["dt"]), int(params["idt"])))
    for e in exts:                                   # frames made before the timed runs
        for (k, _) in e.loads:
            frame(k)
    for k in (1, 2, 3):
        frame(k)
    T = Tracker([spec], [grid], params, numpar=npart, field_dtype="f64", seed=7)
    T.synchronize()
    t0 = time.perf_counter()
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, frame(k))
    T.locate(rel, t_b=1)
    nsteps = 0
    for e in exts:
        for (k, slot) in e.loads:
            T.upload_frame(1, slot, frame(k))
        for it in e.internal:
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            nsteps += 1
    g = T.get_particles()
    t_gpu = time.perf_counter() - t0
    T.close()
    threads = os.cpu_count() or 1

    def oracle_run(n, noise, nthreads):
        m = O.OracleModel([spec], [grid], params)
        r = synth.Release(ipos=rel.ipos[:, :n], jpos=rel.jpos[:, :n], z=rel.z[:n], dob=rel.dob[:n])
        mt = O.MT19937(7) if noise == "mt" else None
        t0 = time.perf_counter()
        for (k, slot) in schedule.initial_loads():
            m.set_frame(1, slot, frame(k))
        m.init_particles(r, tb=1)
        for e in exts:
            for (k, slot) in e.loads:
                m.set_frame(1, slot, frame(k))
            for it in e.internal:
                m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise=noise, seed=7, step_index=it.step_index,
                       mt=mt, nthreads=nthreads)
        return m.state(), time.perf_counter() - t0

    o, t_cpu = oracle_run(npart, "philox", threads)
    nser = min(1000, npart)
    _, t_ser = oracle_run(nser, "mt", 1)
    same = {}
    for k in ("x", "y", "z", "age", "status"):
        a, b = np.asarray(g[k]), np.asarray(o[k]).astype(np.float64)
        same[k] = int(np.sum(a.view(np.uint64) != b.view(np.uint64)))
    out = {"mode": "config1", "workload": "cfg1: 130x98x20 grid, 10x10 land corner, VTurb on, HTurb off, 2 days",
           "particles": npart, "internal_steps": nsteps,
           "seconds": {"gpu_end_to_end": t_gpu, "cpu_oracle_openmp": t_cpu,
                       f"cpu_oracle_serial_mt19937_{nser}_particles": t_ser},
           "particle_steps_per_s": {"gpu_end_to_end": npart * nsteps / t_gpu,
                                    "cpu_oracle_openmp": npart * nsteps / t_cpu,
                                    "cpu_oracle_serial_mt19937": nser * nsteps / t_ser},
           "cpu_threads": threads, "particles_differing_from_oracle": same,
           "note": "GPU time includes every frame upload from host arrays, the initial lookup and the final "
                   "read-back; the frames are made before either run"}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------- features

def features_run(args):
    """The rows beyond the step on config 2's grid and 1,048,576 particles,
    exact FP32-field form: the step with the diagnostics (SaltTempOn,
    SaltTempMean, WriteBottom), WETDRY, behave 10 (Process_VA and _WA) and
    all of them, device time per internal step (CUDA events on the
    library's stream, median of K after W); one output record (device pack,
    read-back into page-locked arrays); LL2ij of every particle from lon/lat
    (rp_locate_lonlat, end to end) against the oracle's LL2ij on a
    single-threaded sample; InitGrid's nest maps hashed against the
    reference's search on a parent 400x300 / child 240x180 pair.  The
    "mixed/" variants run the mixed-precision form instead."""
    import torch
    from romspath_b200 import Tracker
    from romspath_b200.tracker import nest_maps
    from oracle import oracle as O
    torch.cuda.set_device(0)
    npart = args.particles or synth.CONFIG_PARTICLES["cfg2"]
    base = synth.config_spec("cfg2")[0]
    spec = dataclasses.replace(base, diag=True, wetdry=True, behave=True)
    grid = synth.make_grid(spec)
    params0 = synth.config_params("cfg2")
    frames = [synth.make_frame(spec, grid, k * 3600.0) for k in range(4)]
    rel = synth.uniform_release(spec, grid, frames[0], npart, seed=0)
    exts = list(schedule.external_steps(2.0, int(params0["dt"]), int(params0["idt"])))
    its = [it for e in exts for it in e.internal]
    synth_diag = {"salttemp_on": 1, "salttemp_mean": 1, "write_bottom": 1}
    variants = [
        ("passive", {}),
        ("diagnostics", dict(synth_diag)),
        ("wetdry", {"wetdry": 1}),
        ("behave10", dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0)),
        ("diagnostics+behave10", dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0, **synth_diag)),
        ("diagnostics+wetdry", dict(wetdry=1, **synth_diag)),
        ("behave10+wetdry", dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0, wetdry=1)),
        ("all", dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0, wetdry=1, **synth_diag)),
    ]
    variants += [("passive/split", {}), ("all/split", variants[-1][1]),
                 ("mixed/passive", {}), ("mixed/diagnostics", dict(synth_diag)),
                 ("mixed/behave10", dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0)),
                 ("mixed/wetdry", {"wetdry": 1}),
                 ("mixed/all", dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0, wetdry=1, **synth_diag))]
    if args.variants:
        keep = set(args.variants.split(","))
        variants = [v for v in variants if v[0] in keep]
    steps = {}
    for name, pov in variants:
        params = dict(params0, **pov)
        form = "mixed" if name.startswith("mixed/") else spec.field_dtype
        T = Tracker([spec], [grid], params, numpar=npart, field_dtype=form, stokes=spec.stokes,
                    seed=7, resort=args.resort, variant="split" if name.endswith("/split") else "fused")
        for k, slot in enumerate((1, 2, 3)):
            T.upload_frame(1, slot, frames[k])
        T.locate(rel, t_b=1)
        ms = []
        for i in range(args.warmup + args.steps):
            it = its[i % 12]
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            T.synchronize()
            if i >= args.warmup:
                ms.append(T.last_step_stats()[0])
        rec_ms = None
        if name == "all":
            pins = {k: pinned_empty(npart, np.float64) for k in Tracker.RECORD}   # (array, owning tensor)
            out = {k: v[0] for k, v in pins.items()}
            T.synchronize()
            t0 = time.perf_counter()
            T.output_record(13, out=out)
            rec_ms = (time.perf_counter() - t0) * 1e3
        T.close()
        steps[name] = {"ms_per_step": float(np.median(ms)), "particle_steps_per_s": npart / (np.median(ms) * 1e-3)}
        if rec_ms is not None:
            steps[name]["output_record_ms"] = rec_ms
    for name in steps:
        ref = "mixed/passive" if name.startswith("mixed/") else "passive"
        if ref in steps:
            steps[name]["vs_passive"] = steps[name]["ms_per_step"] / steps[ref]["ms_per_step"]
    if args.no_init:
        print(json.dumps({"mode": "features", "step": steps}), flush=True)
        return

    # LL2ij from lon/lat: every particle, end to end through the C ABI
    lon = np.ascontiguousarray(synth_bilinear(grid["lon_rho"], rel.ipos[0], rel.jpos[0]))
    lat = np.ascontiguousarray(synth_bilinear(grid["lat_rho"], rel.ipos[0], rel.jpos[0]))
    T = Tracker([spec], [grid], params0, numpar=npart, field_dtype=spec.field_dtype, stokes=spec.stokes, seed=7)
    for k, slot in enumerate((1, 2, 3)):
        T.upload_frame(1, slot, frames[k])
    T.locate_lonlat(lon[:4096], lat[:4096], rel.z[:4096], rel.dob[:4096])    # warm-up
    T.synchronize()
    t0 = time.perf_counter()
    gi, gj = T.locate_lonlat(lon, lat, rel.z, rel.dob)
    t_gpu = time.perf_counter() - t0
    T.close()
    m = O.OracleModel([spec], [grid], params0)
    ns = min(args.cpu_sample, npart)
    t0 = time.perf_counter()
    oi, oj = m.ll2ij(1, lon[:ns], lat[:ns], spherical=1)
    t_cpu = time.perf_counter() - t0
    same = int(np.sum(oi.view(np.uint64) != gi[0, :ns].view(np.uint64)) +
               np.sum(oj.view(np.uint64) != gj[0, :ns].view(np.uint64)))
    ll2ij = {"particles": npart, "grid": f"{spec.xi_rho}x{spec.eta_rho}",
             "gpu_end_to_end_s": t_gpu, "gpu_particles_per_s": npart / t_gpu,
             "cpu_oracle_sample": ns, "cpu_oracle_s": t_cpu, "cpu_particles_per_s": ns / t_cpu, "cpu_threads": 1,
             "sample_indices_differing": same,
             "max_index_error_cells": float(max(np.max(np.abs(gi[0] - rel.ipos[0])),
                                                np.max(np.abs(gj[0] - rel.jpos[0]))))}

    # nest maps: a parent 400x300 at 1 km and a child 240x180 at 250 m whose
    # rho point (1,1) sits on parent point (101, 76)
    px, py = np.meshgrid(np.arange(400) * 1000.0, np.arange(300) * 1000.0, indexing="ij")
    cx, cy = np.meshgrid(100000.0 + np.arange(240) * 250.0, 75000.0 + np.arange(180) * 250.0, indexing="ij")
    specs = [synth.GridSpec(240, 180, 4), synth.GridSpec(400, 300, 4)]
    grids = [synth.make_grid(s) for s in specs]
    grids[0]["lon_rho"], grids[0]["lat_rho"] = np.asfortranarray(cx), np.asfortranarray(cy)
    grids[1]["lon_rho"], grids[1]["lat_rho"] = np.asfortranarray(px), np.asfortranarray(py)
    t0 = time.perf_counter()
    sh, oh = nest_maps(grids, [4.0])
    t_hash = time.perf_counter() - t0
    mo = O.OracleModel(specs, grids, params0)
    t0 = time.perf_counter()
    so, oo = mo.nest_maps([4.0])
    t_search = time.perf_counter() - t0
    nest = {"grids": "child 240x180 (250 m) in parent 400x300 (1 km)", "hashed_s": t_hash,
            "reference_search_s": t_search, "maps_equal": bool(np.array_equal(sh, so) and np.array_equal(oh, oo)),
            "child_to_parent": {"scl": sh[0][1].tolist(), "off": oh[0][1].tolist()}}
    print(json.dumps({"mode": "features", "workload": "cfg2 grid 512x384x30, FP32 fields, 1,048,576 particles",
                      "step": steps, "ll2ij": ll2ij, "nest_maps": nest,
                      "timing": f"median of {args.steps} steps after {args.warmup}, CUDA events"}), flush=True)


def synth_bilinear(a, ip, jp):
    I, J = np.floor(ip).astype(int), np.floor(jp).astype(int)
    X, Y = ip - I, jp - J
    return ((1 - X) * (1 - Y) * a[I - 1, J - 1] + X * (1 - Y) * a[I, J - 1] + X * Y * a[I, J]
            + (1 - X) * Y * a[I - 1, J])


# ---------------------------------------------------------------- adjoint

def adjoint_run(args):
    """Release attribution on the 130x98x20 grid: L = sum_p exp(-d_p^2 /
    (2 sigma^2)), d_p the distance (cells) of particle p at day 3 from the
    centroid of a target box, sigma = 5 cells; gradients with respect to the
    initial positions and to the diffusivity multiplier, checked against
    the tangent-linear reference and central differences."""
    import torch
    from romspath_b200 import Tracker
    from romspath_b200.adjoint import Adjoint, attribution_loss, step_table
    torch.cuda.set_device(0)
    wl = "cfg5"
    spec = synth.config_spec(wl)[0]
    grid = synth.make_grid(spec)
    params = synth.config_params(wl)
    npart = args.particles or synth.CONFIG_PARTICLES[wl]
    days = synth.CONFIG_DAYS[wl]
    frames = {}

    def frame(k):
        if k not in frames:
            frames[k] = synth.make_frame(spec, grid, (k - 1) * float(params["dt"]))
        return frames[k]

    rel = synth.uniform_release(spec, grid, frame(1), npart, seed=0)
    T = Tracker([spec], [grid], params, numpar=npart, field_dtype="f64", seed=7)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, frame(k))
    T.locate(rel, t_b=1)
    st0 = T.get_particles()
    steps, kmax = step_table(days, int(params["dt"]), int(params["idt"]))
    adj = Adjoint(T)
    adj.load_frames(kmax, lambda ng, k: frame(k))
    target = (0.5 * (40 + 90), 0.5 * (30 + 70))          # centroid of the box i 40..90, j 30..70
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn):
        T.synchronize()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        T.synchronize()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    _, t_fwd = timed(lambda: adj.forward(steps, kappa=1.0, checkpoint_every=48))
    fin = T.get_particles()
    L, gx, gy = attribution_loss(fin["x"], fin["y"], target)
    (ax, ay, az, ak), t_bwd = timed(lambda: adj.backward(gx, gy, np.zeros(npart)))
    J, t_tan = timed(lambda: adj.tangent())
    _, t_rep = timed(lambda: adj.replay())
    tx = gx * J[:, 0, 0] + gy * J[:, 1, 0]
    tk = float((gx * J[:, 0, 3] + gy * J[:, 1, 3]).sum())
    moved = np.isin(fin["status"], [1.0, np.float32(1.1), np.float32(1.2)])
    sig = moved & (np.abs(ax) > 1e-3 * np.abs(ax).max())       # particles that carry the gradient
    agree_tan = float(np.max(np.abs(ax - tx)) / max(np.abs(tx).max(), 1e-300))

    def fd_rel(eps):
        xp, yp, _ = adj.replay(x0=st0["x"] + eps)
        xm, ym, _ = adj.replay(x0=st0["x"] - eps)
        term = lambda x, y: np.exp(-((x - target[0]) ** 2 + (y - target[1]) ** 2) / 50.0)
        fd = (term(xp, yp) - term(xm, ym)) / (2 * eps)
        r = np.abs(fd - ax) / np.abs(ax)
        return r[sig]

    r6, r3 = fd_rel(1e-6), fd_rel(1e-3)
    fdk = {}
    term = lambda x, y: np.exp(-((x - target[0]) ** 2 + (y - target[1]) ** 2) / 50.0)
    tkp = gx * J[:, 0, 3] + gy * J[:, 1, 3]                     # each particle's share of dL/dkappa
    sigk = moved & (np.abs(tkp) > 1e-3 * np.abs(tkp).max())
    kfrac = {}
    for ke in (1e-4, 1e-6):
        xp, yp, _ = adj.replay(kappa=1.0 + ke)
        xm, ym, _ = adj.replay(kappa=1.0 - ke)
        fdk[ke] = (attribution_loss(xp, yp, target)[0] - attribution_loss(xm, ym, target)[0]) / (2 * ke)
        fdp = (term(xp, yp) - term(xm, ym)) / (2 * ke)
        kfrac[ke] = float(np.mean((np.abs(fdp - tkp) / np.abs(tkp))[sigk] < 1e-4))
    out = {"mode": "adjoint", "workload": "cfg5: 130x98x20 grid, VTurb on, HTurb off, 3 days = 864 steps",
           "particles": npart, "steps": len(steps), "checkpoint_every": 48, "loss": L,
           "seconds": {"forward": t_fwd, "backward": t_bwd, "tangent": t_tan, "replay": t_rep},
           "backward_over_forward": t_bwd / t_fwd, "tangent_over_forward": t_tan / t_fwd,
           "backward_over_replay": t_bwd / t_rep,
           "particle_steps_per_s": {"forward": npart * len(steps) / t_fwd, "backward": npart * len(steps) / t_bwd},
           "dL_dkappa": {"adjoint": ak, "tangent": tk,
                         "central_difference_eps_1e-4": fdk[1e-4], "rel_diff_eps_1e-4": abs(fdk[1e-4] - ak) / abs(ak),
                         "central_difference_eps_1e-6": fdk[1e-6], "rel_diff_eps_1e-6": abs(fdk[1e-6] - ak) / abs(ak),
                         "per_particle_share_within_1e-4_eps_1e-4": kfrac[1e-4],
                         "per_particle_share_within_1e-4_eps_1e-6": kfrac[1e-6],
                         "per_particle_compared": int(sigk.sum()),
                         "note": "the summed central difference includes the jumps of the few particles whose "
                                 "+-eps runs straddle a discontinuity of the model (cell-edge zeta, land "
                                 "rejection); per particle the shares agree"},
           "dL_dx0_vs_tangent_max_rel": agree_tan,
           "dL_dx0_vs_central_difference": {
               "particles_compared": int(sig.sum()),
               "selection": "moved particles whose |dL/dx0| exceeds 1e-3 of the largest",
               "eps_1e-6_fraction_within_1e-4": float(np.mean(r6 < 1e-4)), "eps_1e-6_median_rel": float(np.median(r6)),
               "eps_1e-3_fraction_within_1e-4": float(np.mean(r3 < 1e-4)), "eps_1e-3_median_rel": float(np.median(r3))},
           "note": "times include the host loop over steps; backward = recompute of each 48-step segment from its "
                   "checkpoint + reverse steps (per-step Jacobians by 4-direction dual numbers)"}
    T.close()
    del ev
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ GPU arm

FORM_DESC = {
    "mixed": "mixed precision: FP16 u/v/w/AKs with per-level power-of-two scales, FP32 zeta, FP32 positions with "
             "Kahan compensation, FP32 interpolation/RK4, FP64 age, secant search and sub-steps, smoothing-spline "
             "factor rows in FP64 and substitution sweeps in FP32",
    "mixed-i16": "mixed precision with int16 fixed-point u/v/w/AKs (scale = level max / 32767)",
    "f32": "exact: FP64 arithmetic on FP32-stored fields (bit-identical to the CPU oracle)",
    "f64": "plain FP64: FP64-stored fields, FP64 arithmetic (bit-identical to the CPU oracle)",
}
KERNEL = {"mixed": "k_step_mixed", "mixed-i16": "k_step_mixed", "f32": "k_step_fused", "f64": "k_step_fused"}
# algorithmic bytes per particle-step of each form on the cfg2 / cfg3 grids
B_ALG_FORM = {("cfg2", "mixed"): 1872, ("cfg2", "mixed-i16"): 1872, ("cfg2", "f32"): 3192, ("cfg2", "f64"): 6248,
              ("cfg3", "mixed"): 1632, ("cfg3", "mixed-i16"): 1632, ("cfg3", "f64"): 5288, ("cfg1", "f64"): 5288}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.error_study:
        error_study(args)
        return
    if args.adjoint:
        adjoint_run(args)
        return
    if args.batched:
        batched_run(args)
        return
    if args.config1:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        config1_run(args)
        return
    if args.features:
        features_run(args)
        return
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    from romspath_b200 import Tracker

    wl = args.workload
    spec = synth.config_spec(wl)[0]
    grid = synth.make_grid(spec)
    params = dict(synth.config_params(wl))
    overrides = parse_params(args.param, params)
    params.update(overrides)
    npart = args.particles or synth.CONFIG_PARTICLES[wl]
    nframes = 4
    frames = [synth.make_frame(spec, grid, k * 3600.0) for k in range(nframes)]
    rel = synth.uniform_release(spec, grid, frames[0], npart, seed=rank)
    exts = list(schedule.external_steps(30.0, int(params["dt"]), int(params["idt"])))
    head = args.mixed_kind if args.form == "mixed" else spec.field_dtype
    others = ("mixed-i16" if head == "mixed" else "mixed",) if head.startswith("mixed") else ()
    forms = [head] + [f for f in others + (spec.field_dtype, "f64") if f != head]

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def make_tracker(form):
        T = Tracker([spec], [grid], params, numpar=npart, field_dtype=form, stokes=spec.stokes, seed=7,
                    device=local, resort=args.resort)
        T.set_id_base(rank * npart)     # global particle ids: rank r holds [r*npart, (r+1)*npart)
        T.set_kernel_form(args.kernel_form)
        for k, slot in enumerate((1, 2, 3)):
            T.upload_frame(1, slot, frames[k])
        T.locate(rel, t_b=1)
        T.synchronize()
        return T

    def time_resident(T, clocks_on):
        """W untimed + K timed frame intervals (12 internal steps each) on
        device-resident frames and particles; CUDA events on the library's
        compute stream."""
        st = T.device_state()
        stream = torch.cuda.ExternalStream(st.stream, device=torch.device("cuda", local))

        def run(e0, n_ext, record):
            evs = []
            for e in exts[e0:e0 + n_ext]:
                for it in e.internal:
                    if record:
                        a = torch.cuda.Event(enable_timing=True)
                        b = torch.cuda.Event(enable_timing=True)
                        a.record(stream)
                    T.step(it.ex, it.ix, it.ets, 1, 2, 3)
                    if record:
                        b.record(stream)
                        evs.append((a, b))
            return evs

        run(2, args.warmup, False)
        T.synchronize()
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if clocks_on else None
        if sampler:
            sampler.start()
        l0 = T.kernel_launches()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        evs = run(2 + args.warmup, args.steps, True)
        t1.record(stream)
        T.synchronize()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        region_ms = max_over_ranks(t0.elapsed_time(t1))
        kern = max_over_ranks(float(np.mean([a.elapsed_time(b) for a, b in evs])))
        return {"region_ms": region_ms, "avg_launch_ms": kern, "launches": T.kernel_launches() - l0,
                "clocks": clocks}

    def spline_counts(T):
        """One frame interval after the timed region, with VTurb's
        smoothing-spline fits and their chol1d passes counted (outside every
        timed region; counting changes no result)."""
        T.count_spline_passes(True)
        for it in exts[1].internal:
            T.step(it.ex, it.ix, it.ets, 1, 2, 3)
        f, p = T.spline_pass_counts()
        T.count_spline_passes(False)
        return f, p

    results = {}
    e2e = None
    head_T = None
    for form in forms:
        T = make_tracker(form)
        r = time_resident(T, form == head)
        r["spline_fits"], r["spline_passes"] = spline_counts(T)
        r["value"] = npart * 12 * args.steps * world / (r["region_ms"] / 1e3)
        r["ms_per_step"] = r["region_ms"] / args.steps
        results[form] = r
        if form == head:
            head_T = T
        else:
            T.close()

    # ---------------- e2e of the headline form: frames up, particles back
    T = head_T
    if not args.no_e2e:
        keep = []
        pframes = []
        for f in frames:
            d = {}
            for k, a in f.items():
                arr, t = pinned_like(a)
                keep.append(t)
                d[k] = arr
            pframes.append(d)
        # the dataOutput record (ROMSPath.f90:1012-1024, 1924-1995): lon,
        # lat, zp, age, status, GID, double-buffered page-locked arrays
        outs = []
        for _ in range(2):
            o = {}
            for k in ("lon", "lat", "zp", "age", "status", "gid"):
                o[k], t = pinned_empty(npart, np.float64)
                keep.append(t)
            outs.append(o)
        h2d = sum(pframes[0][k].nbytes for k in ("zeta", "u", "v", "w", "aks", "su", "sv") if k in pframes[0])
        d2h = sum(v.nbytes for v in outs[0].values())

        def e2e_run(es, f0):
            """The driver's frame intervals, pipelined: interval j's steps are
            enqueued (one graph) with its output record behind them, then
            interval j+1's frame is uploaded into the ring's spare slot while
            they run; each record is copied into page-locked arrays while the
            next interval runs (double-buffered; a record may be read after
            rp_output_wait).  Each frame and each record crosses PCIe once,
            and the results equal the unpipelined order's (a step binds its
            ring slots when it is enqueued)."""
            for (kf, slot) in es[0].loads:
                T.upload_frame(1, slot, pframes[f0 % nframes])
            for j, e in enumerate(es):
                T.step_n(e.internal)
                T.output_record_async(1, outs[j % 2])
                if j + 1 < len(es):
                    for (kf, slot) in es[j + 1].loads:
                        T.upload_frame(1, slot, pframes[(f0 + j + 1) % nframes])
            T.output_wait()

        base = 2 + args.warmup + args.steps
        # warm-up intervals (untimed) with the fit's passes counted: the
        # frames change every interval here, unlike the resident leg's
        T.count_spline_passes(True)
        e2e_run(exts[base:base + args.warmup], 0)
        T.synchronize()
        e2e_fits, e2e_passes = T.spline_pass_counts()
        T.count_spline_passes(False)
        barrier()
        l0 = T.kernel_launches()
        t0 = time.perf_counter()
        e2e_run(exts[base + args.warmup:base + args.warmup + args.steps], 1)
        T.synchronize()
        t1 = time.perf_counter()
        e2e_s = max_over_ranks(t1 - t0)
        e2e = {"value": npart * 12 * args.steps * world / e2e_s, "unit": "particle-steps/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e2e_s * 1e3 / args.steps, "gpu_launches": T.kernel_launches() - l0,
               "chol1d_passes_per_fit": (e2e_passes / e2e_fits) if e2e_fits else None,
               "form": head,
               "timing": "host clock between device synchronizations; every step uploads one frame "
                         "(quantised on the device in the mixed form) and reads its dataOutput record "
                         "(lon, lat, zp, age, status, GID) back into page-locked host memory; the next "
                         "interval's frame is uploaded and each record copied back while the next "
                         "steps run (one CUDA graph per interval)"}
    T.close()

    # ---------------- roofline of the headline step kernel (algorithmic bytes)
    hr = results[head]
    peak, peak_src = measured_peaks()
    balg = B_ALG_FORM.get((wl, head), 1872)
    achieved = balg * npart / (hr["avg_launch_ms"] / 1e3) / 1e9
    traffic = profile_traffic(wl, KERNEL[head])
    l2_traffic = profile_traffic(wl, KERNEL[head], "lts_bytes_per_launch")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                "dram_gbs_from_traffic": (traffic / (hr["avg_launch_ms"] / 1e3) / 1e9) if traffic else None,
                "l2_traffic": l2_traffic,
                "l2_gbs_from_traffic": (l2_traffic / (hr["avg_launch_ms"] / 1e3) / 1e9) if l2_traffic else None,
                "note": "achieved counts the field and particle bytes the reference arithmetic consumes at the "
                        "form's storage widths; DRAM traffic is dominated by the smoothing-spline workspace in "
                        "local memory (see profiles/)",
                "kernel": f"{KERNEL[head]} (one launch per internal step)",
                "avg_launch_ms": hr["avg_launch_ms"],
                "algorithmic_bytes": f"{balg} B/particle-step x {npart} particles per launch"}

    # ---------------- the smoothing-spline fit: passes per fit, FP64 rate
    np_fit = int((spec.N + 1) * params["sub"])

    def spline_of(form):
        r = results[form]
        f, p = r["spline_fits"], r["spline_passes"]
        d = {"fits_per_particle_step": f / (npart * 12), "chol1d_passes_per_fit": (p / f) if f else None,
             "np": np_fit}
        prof = profile_fp64(wl, KERNEL[form])
        if prof and prof.get("form") == form:
            fl = prof["fp64_flop_per_launch"] / prof["particles"]
            d.update({"fp64_flop_per_particle_step": fl,
                      "fp64_tflops": fl * npart / (r["avg_launch_ms"] / 1e3) / 1e12,
                      "fp64_pipe_active_pct": prof.get("fp64_pipe_active_pct"),
                      "fp64_source": prof.get("source")})
        return d

    spline = {"form": head, **spline_of(head),
              "forms": {f: spline_of(f) for f in results if f != head},
              "fp64_peak_tflops": FP64_PEAK_NOMINAL_TFLOPS, "fp64_peak_source": "nominal (296 TFLOP/s per DGX B200 / 8)",
              "note": "fits and chol1d passes counted on the device over one frame interval after the timed region "
                      "(rp_count_spline_passes); FP64 flops = DADD + DMUL + 2 DFMA per launch from ncu counts of the "
                      "same workload, scaled per particle-step, over the live-timed launch"}
    if "fp64_tflops" in spline:
        spline["fp64_frac"] = spline["fp64_tflops"] / FP64_PEAK_NOMINAL_TFLOPS

    # ---------------- error of the mixed forms at this speed (lockstep)
    err = None
    if rank == 0 and head.startswith("mixed") and args.error_days > 0:
        t0 = time.time()
        kinds = [head] + [k for k in ("mixed", "mixed-i16") if k != head]
        err = {"vs": f"the exact form (FP64 arithmetic on {spec.field_dtype}-stored fields, bit-identical to the "
                     f"CPU restatement of the reference), stepped in lockstep on the same grid, hourly frames, "
                     f"release and Philox noise; positions in grid cells over particles moved in both forms",
               "days": args.error_days, "particles": args.error_particles,
               **lockstep_error(wl, kinds, args.error_days, args.error_particles)}
        err["wall_s"] = time.time() - t0

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cval, _ = cpu_timing(wl, args.cpu_sample, 1, 0, threads)
        cpu = {"value": cval, "unit": "particle-steps/s", "cores": threads, "kind": "port",
               "sample": f"{wl} grid, {args.cpu_sample} particles x 12 internal steps, Philox noise, "
                         f"{threads} OpenMP threads (FP64 C restatement of the reference; the Fortran "
                         f"reference cannot be built here)"}

    if rank == 0:
        plain = results.get("f64")
        line = {
            "metric": "particle-steps/s", "value": hr["value"], "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": hr["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16/f32/f64 (mixed)" if head.startswith("mixed") else "f64",
            "data": "synthetic (analytic ROMS-shaped fields, seeded release)",
            "config": {"workload": WORKLOAD_DESCS.get(wl, wl), "particles_per_gpu": npart,
                       "step": "one hydro frame interval = 12 internal steps (idt=300 s)",
                       "form": FORM_DESC[head], "kernel_form": args.kernel_form,
                       **({"param_overrides": overrides} if overrides else {}),
                       "l2": ("inputs larger than L2 (frame ring 390 MB FP32 / 195 MB FP16, particle state "
                              "~80 MB, spline workspace in local memory ~0.5-1 GB)") if wl == "cfg2" else
                             ("frames L2-resident (8.4 MB per FP64 frame), particle state and spline workspace "
                              "larger than L2"),
                       "parallelism": f"replicas x{world}: particles split per rank, no data-path collective",
                       "resort": f"particle state re-sorted by grid and cell every {args.resort} internal steps "
                                 f"(inside the timed region)" if args.resort else "off"},
            "forms": {f: {"value": r["value"], "ms_per_step": r["ms_per_step"],
                          "avg_launch_ms": r["avg_launch_ms"], "desc": FORM_DESC[f],
                          "speedup_vs_plain_fp64": (r["value"] / plain["value"]) if plain else None}
                      for f, r in results.items()},
            "roofline": roofline, "spline": spline, "error": err, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": hr["clocks"],
            "gpu_launches": int(hr["launches"]),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
