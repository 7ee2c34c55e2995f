#!/usr/bin/env python
"""Throughput of the B200 Godunov level step (RAMSES-CPP HydroSolver::godunov_fine)
on the metric's own configuration: the 3D Sedov blast with octree AMR.

Workload (the headline `value`): reference levelmin 7, levelmax 10 (a 64^3
base grid refined to 512^3 effective; the Fortran numbering's levelmin 6 /
levelmax 9), refinement on relative density and pressure gradients > 0.1,
nexpand 1, sub-cycling 2, MonCen slopes, HLLC, gamma 1.4, Courant factor
0.25, FP64, periodic.  The tree and the state are resident on the GPU: the
run is initialised on the device (rg_amr.initialize: the reference's
Simulation::initialize rounds with the device tree kernels) and every coarse
step is one rg_amr_coarse_step call (Simulation::amr_step with flag_fine,
make_grid_fine, remove_grid_fine, restrict_fine, the CFL step, set_unew,
godunov_fine and set_uold all on the device).  One bench step = one coarse
step; W warm-up coarse steps, then K timed ones (the window is coarse steps
W+1..W+K of the run).  Cell updates = son == 0 cells processed by every
godunov_fine call of the window, sub-cycled ones included.

The reference's own scheme collapses on this run after about 40 coarse steps
at Courant 0.25 (6 at the 0.8 of the other configs): refluxes that reach a
cell after its own clamp drive coarse cells next to the refined region to
negative density, the density floor then gives sound speeds of 1e4 and dt
falls to 1e-13.  The default window (W=5, K=20) lies before that; the line
reports the window's time span and its last finest-level dt.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  N > 1 runs one independent replica of the
AMR run per GPU (replicas only: the single grid is not partitioned), so the
ranks exchange nothing but the final timing maximum.

Keys besides the contract's:
- `roofline`: the dominant kernel of the AMR step (the face kernel, summed
  over every level step of two coarse steps with CUDA events) against the
  measured HBM copy bandwidth; `traffic` and the FP64 counts come from the
  machine-readable ncu record profiles/roofline_inputs.json, checked against
  the hash of the kernel sources it was captured at (`stale` if they moved);
- `e2e`: the same coarse steps with the state in page-locked host memory,
  uploaded before and downloaded after every coarse step;
- `cpu_baseline`: the reference compiled here, one core, on coarse steps of
  the same window;
- `parity`: the GPU run's uold and son after W+2 coarse steps against the
  reference's (SHA-1 digest, computed in the CPU baseline's process);
- `sedov128` (config 2: the uniform 128^3 level, brick face kernel, its own
  rooflines), `newton` (config 5), `ensemble` (config 4), `amr_dropin`
  (the reference's own AmrGrid/TreeUpdater step with the GPU hydro drop-in),
  `sod1d` (config 1).
"""
import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "ramses-cpp_b200"))

METRIC = "cell-updates/s 3D Sedov AMR FP64, %HBM roofline; Newton iters learned vs plain"
UNIT = "cell-updates/s"
AMR = dict(lmin=7, lmax=10, ngridmax=48000, cfl=0.25, ed=0.1, ep=0.1, gamma=1.4)
WORKLOAD = ("3D Sedov blast with octree AMR, reference levelmin 7 / levelmax 10 (64^3 base, 512^3 effective), "
            "err_grad_d = err_grad_p = 0.1, nexpand 1, sub-cycled, MonCen + HLLC, gamma 1.4, courant 0.25, FP64, "
            "tree and state resident on the GPU")
BYTES_PER_CELL_UPDATE = 80  # uold read once + unew written once, 5 FP64 variables each
FACE_SOURCES = ("rg_face.cuh", "rg_face_brick.cuh", "rg_face_pipe.cuh", "rg_physics.cuh", "rg_face.cu",
                "rg_face_1d.cu", "rg_face_3d.cu", "rg_internal.cuh", "rg_nav.cuh")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def face_source_sha():
    """SHA-256 (16 hex digits) of the face kernels' sources, the key of the
    ncu record in profiles/roofline_inputs.json."""
    h = hashlib.sha256()
    for name in FACE_SOURCES:
        h.update((ROOT / "ramses-cpp_b200" / "csrc" / name).read_bytes())
    return h.hexdigest()[:16]


def roofline_inputs(key):
    """The ncu record of a face kernel (profiles/roofline_inputs.json): DRAM
    bytes, FP64 FLOPs and FP64 instructions per cell update, and whether the
    sources have changed since the capture."""
    f = ROOT / "profiles" / "roofline_inputs.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text()).get(key)
    if not d:
        return None
    d = dict(d)
    d["current_source_sha"] = face_source_sha()
    d["stale"] = d.get("source_sha") != d["current_source_sha"]
    return d


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.rows = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "10", "-i", str(gpu_index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, line in self.rows:
            if not (t0 - 0.05 <= t <= t1 + 0.1):
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU side
def amr_cpu_window(warmup, steps, parity_after=None):
    """The reference on the headline's AMR window, single-threaded: its own
    initialisation and coarse steps (AmrGrid / TreeUpdater / HydroSolver
    compiled here from its sources, driven through refsupport.AmrRun, which
    replays Simulation::initialize and Simulation::amr_step with the CFL step
    of the reference formula), `warmup` untimed coarse steps, then `steps`
    timed ones.  Runs in its own process (the reference prints a line per
    flagged cell).  parity_after = k: also the SHA-1 of uold and son after
    coarse step k (1-based)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from refsupport import AmrRun, RefHarness, namelist, sedov_ic
    # the reference's flag_fine prints a line per flagged cell: to /dev/null,
    # at the descriptor level (it writes through the C++ runtime)
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        return _amr_cpu_window(warmup, steps, parity_after, AmrRun, RefHarness, namelist, sedov_ic)
    finally:
        import ctypes
        ctypes.CDLL(None).fflush(None)  # printf's buffer still belongs to /dev/null
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


def _amr_cpu_window(warmup, steps, parity_after, AmrRun, RefHarness, namelist, sedov_ic):
    A = AMR
    nml = namelist(slope_type=2, riemann="hllc", levelmin=A["lmin"], levelmax=A["lmax"], err_grad_d=A["ed"],
                   err_grad_p=A["ep"])
    h = RefHarness(3).create(nml, ngridmax=A["ngridmax"], levelmin=A["lmin"], nlevelmax=A["lmax"], gamma=A["gamma"])
    r = AmrRun(h, A["lmin"], A["lmax"], A["gamma"], cfl=A["cfl"], ed=A["ed"], ep=A["ep"])
    t0 = time.perf_counter()
    r.initialize(sedov_ic(3, A["lmin"]))
    init_s = time.perf_counter() - t0
    digest = None
    done = 0
    for _ in range(warmup):
        r.coarse_step()
        done += 1
        if parity_after == done:
            a = h.arrays()
            digest = hashlib.sha1(a["uold"].tobytes() + a["son"].tobytes()).hexdigest()
    cu0 = r.cell_updates
    el = 0.0
    for _ in range(steps):
        t = time.perf_counter()
        r.coarse_step()
        el += time.perf_counter() - t
        done += 1
        if parity_after == done:
            a = h.arrays()
            digest = hashlib.sha1(a["uold"].tobytes() + a["son"].tobytes()).hexdigest()
    out = {"kind": "reference", "seconds": el, "cells": r.cell_updates - cu0, "steps": steps, "warmup": warmup,
           "init_s": init_s, "t_end": r.t, "digest": digest,
           "octs_per_level": [h.count_grids(il) for il in range(A["lmin"], A["lmax"] + 1)]}
    h.close()
    return out


def run_cpu_window(warmup, steps, parity_after=None, timeout=1800):
    cmd = [sys.executable, str(Path(__file__).resolve()), "--amr-cpu-window", str(warmup), str(steps),
           str(parity_after or 0)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    for line in reversed(r.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("CPU window failed: " + r.stderr[-2000:])


def reference_arm(args, rank, world):
    """The reference's own CPU implementation on the same AMR window, on all
    host cores: one independent process per core, each running the reference's
    initialisation, W untimed and K timed coarse steps (the reference is
    single-threaded); value = all processes' cell updates over the slowest
    process's timed seconds."""
    if rank != 0:
        return None
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.starmap(amr_cpu_window, [(args.warmup, args.steps)] * cores)
    wall = time.perf_counter() - t0
    el = max(r["seconds"] for r in res)
    cells = sum(r["cells"] for r in res)
    value = cells / el
    sample = (f"{cores} processes (one per host core, no shared-memory parallelism in the reference), each the "
              f"whole window: the reference's initialisation, {args.warmup} untimed and {args.steps} timed coarse "
              f"steps of the Sedov AMR run")
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD.replace(", tree and state resident on the GPU", ""),
                       "window": f"coarse steps {args.warmup + 1}..{args.warmup + args.steps}",
                       "cells_per_step": res[0]["cells"] / args.steps, "parallelism": f"{cores} processes"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "t_end": res[0]["t_end"], "octs_per_level": res[0]["octs_per_level"], "wall_s": wall}


# ---------------------------------------------------------------- GPU arm
def amr_params(rgpu):
    return rgpu.make_params(3, slope_type=2, riemann="hllc", interpol_type=1, interpol_var=0, gamma=AMR["gamma"],
                            courant_factor=AMR["cfl"])


def amr_run(ctx):
    """A fresh Sedov AMR run resident on ctx, initialised on the device."""
    import rg_amr
    A = AMR
    rg_amr.initialize(ctx, 3, A["lmin"], A["lmax"], A["ngridmax"], rg_amr.sedov_primitives(3, A["lmin"], A["gamma"]),
                      A["gamma"], ed=A["ed"], ep=A["ep"])
    return rg_amr.DeviceAmrRun(ctx, nx=1, levelmin=A["lmin"], nlevelmax=A["lmax"], cfl=A["cfl"], ed=A["ed"],
                               ep=A["ep"])


def count_launches(torch, run, steps=2):
    """This library's kernels launched per coarse step, counted by the CUDA
    profiler interface (torch.profiler / CUPTI) over `steps` coarse steps."""
    try:
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            for _ in range(steps):
                run.coarse_step()
            torch.cuda.synchronize()
        n = sum(1 for e in prof.events() if e.device_type.name == "CUDA" and "rg::" in e.name)
        return n / steps
    except Exception:  # no profiler on this build: the count stays unreported
        return None


def amr_headline(args, rank, world, local_rank):
    """The headline: K coarse steps of the resident Sedov AMR run after W
    warm-up steps, CUDA events on the library's stream around each coarse step,
    a 256 MB write between steps (outside the events) so every step starts
    with a cold L2; max over ranks."""
    import numpy as np
    import torch
    import rgpu

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream()
    ctx = rgpu.Context(amr_params(rgpu), local_rank)
    ctx.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    run = amr_run(ctx)
    ctx.synchronize()
    init_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        run.coarse_step()
    ctx.synchronize()
    t_start, cu0 = run.t, run.cell_updates
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB of L2
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(local_rank) if rank == 0 else None
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    tw0 = time.time()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        ev[k][0].record(stream)
        run.coarse_step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    tw1 = time.time()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    cells = run.cell_updates - cu0
    if dist:
        dist.barrier()
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clocks = sampler.summary(tw0, tw1) if sampler else None
    if sampler:
        sampler.stop()
    value = world * cells / (ms / 1e3)
    window = {"coarse_steps": f"{args.warmup + 1}..{args.warmup + args.steps}", "t_start": t_start, "t_end": run.t,
              "finest_dt_end": run.clock.dtnew[AMR["lmax"]], "init_s": init_s,
              "octs_per_level": [ctx.count_grids(il) for il in range(AMR["lmin"], AMR["lmax"] + 1)],
              "cells_per_step": cells / args.steps}

    # the dominant kernel: the face kernel of every level step, two coarse steps
    ctx.set_timing("accumulate")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(2):
        run.coarse_step()
    e1.record(stream)
    kms, face_cells, level_steps = ctx.kernel_ms_totals()
    step2_ms = e0.elapsed_time(e1)
    ctx.set_timing(False)
    launches = count_launches(torch, run)

    # end to end: the state in page-locked host memory, uploaded before and
    # downloaded after every coarse step (uold, nvar x ncell FP64 each way)
    ngm, ncell = ctx.tree_sizes()
    host = torch.empty(5 * ncell, dtype=torch.float64, pin_memory=True)
    ctx.download_state_ptr(uold_ptr=host.data_ptr())
    ne = min(args.steps, 10)
    ee = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ne)]
    cu1 = run.cell_updates
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(ne):
        ee[k][0].record(stream)
        ctx.upload_state_ptr(uold_ptr=host.data_ptr())
        run.coarse_step()
        ctx.download_state_ptr(uold_ptr=host.data_ptr())
        ee[k][1].record(stream)
    torch.cuda.synchronize()
    ms_e2e = sum(a.elapsed_time(b) for a, b in ee)
    cells_e2e = run.cell_updates - cu1
    if dist:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = world * cells_e2e / (ms_e2e / 1e3)
    fp64_peak = ctx.measure_fp64_peak() if rank == 0 else None
    ctx.close()
    del flush
    torch.cuda.empty_cache()
    if rank != 0:
        return None

    # a fresh run to coarse step W+2 for the parity digest against the reference
    pctx = rgpu.Context(amr_params(rgpu), local_rank)
    prun = amr_run(pctx)
    for _ in range(args.warmup + 2):
        prun.coarse_step()
    got = pctx.tree_fetch({k: np.zeros(AMR["lmax"] + 1, np.int32) for k in ("headl", "taill", "numbl")})
    digest = hashlib.sha1(got["uold"].tobytes() + got["son"].tobytes()).hexdigest()
    pctx.close()

    peak, peak_kind = peaks()
    face_s = kms[1] / 1e3
    achieved = BYTES_PER_CELL_UPDATE * face_cells / face_s / 1e9
    rin = roofline_inputs("k_face_tiles_amr")
    per_launch_cells = face_cells / max(level_steps, 1)
    traffic = rin["dram_bytes_per_cell_update"] * per_launch_cells if rin else None
    fp64 = None
    if rin and fp64_peak:
        fl = rin["fp64_flops_per_cell_update"] * face_cells / face_s / 1e12
        ops = rin["fp64_ops_per_cell_update"] * face_cells / face_s / 1e12
        fp64 = {"bound": "fp64", "achieved": fl, "peak": fp64_peak, "unit": "TFLOP/s", "frac": fl / fp64_peak,
                "op_frac": ops / (fp64_peak / 2), "kernel": "k_face_tiles",
                "flops_per_cell_update": rin["fp64_flops_per_cell_update"],
                "peak_source": "rg_measure_fp64_peak: independent DFMA chains on every SM (measured here)",
                "flops_source": "profiles/roofline_inputs.json k_face_tiles_amr (ncu)", "stale": rin["stale"]}
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "window": window, "riemann": "hllc", "slope_type": 2,
                   "cfl": "reference compute_courant_step formula without its p <= 100 rho cap, courant_factor 0.25",
                   "l2": "flushed between timed coarse steps (a 256 MB write outside the timed events)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "k_face_tiles (every level step of the coarse step)",
                     "algorithmic_bytes_per_launch": BYTES_PER_CELL_UPDATE * per_launch_cells,
                     "launches": level_steps, "face_share_of_step": kms[1] / step2_ms,
                     "kernel_ms_per_coarse_step": {"prim": kms[0] / 2, "face": kms[1] / 2, "fold": kms[2] / 2,
                                                   "whole_step": step2_ms / 2},
                     "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})",
                     "traffic_source": ("profiles/roofline_inputs.json k_face_tiles_amr (ncu), scaled to the average "
                                        "launch" if rin else None),
                     "traffic_stale": rin["stale"] if rin else None,
                     "step_hbm_frac": (BYTES_PER_CELL_UPDATE * value / world / 1e9) / peak},
        "roofline_fp64": fp64,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * 5 * ncell, "d2h_bytes_per_step": 8 * 5 * ncell,
                "ms_per_step": ms_e2e / ne, "steps": ne,
                "path": "rg_upload_state (page-locked uold) + rg_amr_coarse_step + rg_download_state per coarse step"},
        "gpu_launches": round(launches * args.steps) if launches else None,
        "gpu_launches_per_step": launches,
        "clocks": clocks,
        "parity_digest": {"after_coarse_step": args.warmup + 2, "sha1_uold_son": digest},
    }


def uniform_report(local_rank, steps, warmup, face_variant=None):
    """Config 2: the uniform 128^3 Sedov level (reference levelmin = levelmax
    = 8), MonCen + HLLC, courant 0.8, one substep per step in a CUDA graph
    (dt finalize, brick face kernel, fold that prepares the next substep);
    inputs larger than L2 (state, primitives and flux scratch 0.8 GB)."""
    import numpy as np
    import torch
    import rg_tree
    import rgpu
    L = 8
    g = rg_tree.build_uniform(3, L)
    u0 = rg_tree.sedov_state(g, L)
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", interpol_type=1, gamma=1.4,
                                        courant_factor=0.8), local_rank)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.sync_topology(g)
    ctx.upload_state(u0, u0)
    if face_variant is not None:  # a fixed face-kernel shape instead of the autotuner's pick
        ctx.set_face_config(L, face_variant, 1)
    dx = 1.0 / 2 ** L
    for _ in range(warmup):
        ctx.level_substep(L, dx, pressure_cap=False, use_graph=True)
    ctx.synchronize()
    cells = ctx.cell_updates(L)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ctx.level_substep(L, dx, pressure_cap=False, use_graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    variant = ctx.face_config(L)[0]
    face_kernel = "k_face_brick" if variant >= 9 else ("k_face_pipe" if variant >= 7 else "k_face_tiles")
    ctx.set_timing(True)
    nk = min(steps, 40)
    acc = np.zeros(3)
    for _ in range(nk):
        ctx.level_substep(L, dx, pressure_cap=False, use_graph=False)
        ctx.synchronize()
        acc += np.array(ctx.kernel_ms())
    ctx.set_timing(False)
    kms = acc / nk
    n = g.nvar * g.ncell
    host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    ctx.download_state_ptr(uold_ptr=host.data_ptr())
    ne = min(steps, 40)
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(ne):
        ctx.level_substep_host_ptr(L, dx, host.data_ptr(), want_dt=False)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    fp64_peak = ctx.measure_fp64_peak()
    link = pinned_copy_gbs(torch, stream, 8 * g.nvar * cells)
    ctx.close()
    peak, peak_kind = peaks()
    face_s = kms[1] / 1e3
    achieved = BYTES_PER_CELL_UPDATE * cells / face_s / 1e9
    rin = roofline_inputs(f"{face_kernel}_sedov128")
    return {"workload": "3D Sedov blast, uniform 128^3 (reference levelmin=levelmax=8), MonCen + HLLC, gamma 1.4, "
                        "courant 0.8 without the p <= 100 rho cap, FP64",
            "value": cells * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "cells_per_step": cells, "kernel_ms": {"prim": kms[0], "face": kms[1], "fold": kms[2]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": rin["dram_bytes_per_cell_update"] * cells if rin else None,
                         "traffic_stale": rin["stale"] if rin else None, "kernel": face_kernel, "variant": variant,
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})"},
            "roofline_fp64": fp64_roofline(rin, face_kernel, cells, face_s, fp64_peak),
            "e2e": {"value": cells * ne / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": 8 * g.nvar * cells,
                    "d2h_bytes_per_step": 8 * g.nvar * cells, "ms_per_step": ms_e2e / ne,
                    "path": "rg_level_substep_host on pinned host memory: the level's cells up, substep, its cells down",
                    "bound": e2e_bound(link, 8 * g.nvar * cells, ms / steps, ms_e2e / ne)}}


def pinned_copy_gbs(torch, stream, nbytes, reps=5):
    """This box's host<->device copy bandwidth for one level's state: a
    page-locked buffer of the e2e step's size copied up and down, best of
    `reps`, CUDA events on the bench stream."""
    n = nbytes // 8
    h = torch.empty(n, dtype=torch.float64, pin_memory=True)
    d = torch.empty(n, dtype=torch.float64, device="cuda")
    out = {}
    for name, (dst, src) in (("h2d_gbs", (d, h)), ("d2h_gbs", (h, d))):
        best = 1e30
        with torch.cuda.stream(stream):
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                dst.copy_(src, non_blocking=True)
                b.record(stream)
                b.synchronize()
                best = min(best, a.elapsed_time(b))
        out[name] = nbytes / (best / 1e3) / 1e9
    return out


def e2e_bound(link, nbytes, ms_device, ms_e2e):
    """Lower bound of the e2e step on this box: the level's cells up and down
    at the measured copy bandwidths, plus the device-resident step."""
    if not link:
        return None
    ms_copy = nbytes / (link["h2d_gbs"] * 1e9) * 1e3 + nbytes / (link["d2h_gbs"] * 1e9) * 1e3
    return {"h2d_gbs": link["h2d_gbs"], "d2h_gbs": link["d2h_gbs"], "copy_ms": ms_copy,
            "bound_ms": ms_copy + ms_device, "frac": (ms_copy + ms_device) / ms_e2e,
            "note": "copies at the measured pinned bandwidth plus the device step, serial (a step's input is the "
                    "previous step's output)"}


def fp64_roofline(rin, face_kernel, cells, face_s, peak_tflops):
    """The face kernel against the FP64 pipe, its real bound: executed FP64
    FLOPs per cell update (ncu instruction counts, a DFMA counted as 2, from
    profiles/roofline_inputs.json) over its CUDA-event time, against the FP64
    throughput measured on this GPU."""
    if not rin or not peak_tflops:
        return None
    achieved = rin["fp64_flops_per_cell_update"] * cells / face_s / 1e12
    ops = rin["fp64_ops_per_cell_update"] * cells / face_s / 1e12
    # instruction throughput: DMUL and DADD take an issue slot of the FP64 pipe
    # like a DFMA but carry one FLOP, so the FLOP fraction understates it
    return {"bound": "fp64", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
            "frac": achieved / peak_tflops, "op_frac": ops / (peak_tflops / 2),
            "flops_per_cell_update": rin["fp64_flops_per_cell_update"],
            "ops_per_cell_update": rin["fp64_ops_per_cell_update"], "kernel": face_kernel, "stale": rin["stale"],
            "peak_source": "rg_measure_fp64_peak: independent DFMA chains on every SM, best of 5 (measured here)",
            "flops_source": f"profiles/roofline_inputs.json {face_kernel}_sedov128 (ncu)"}


def newton_report(local_rank, stream, steps):
    """Exact solver, plain vs learned Newton start (converged mode |dp|/p < 1e-14)."""
    import numpy as np
    import torch
    import rg_tree
    import rgpu
    out = {"tolerance": 1e-14, "iteration_cap": 100}
    ctx = rgpu.Context(rgpu.make_params(3, riemann="exact"), local_rank)
    ctx.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    loss = ctx.mlp_train()
    ctx.synchronize()
    out["training"] = {"samples": 10_000_000, "epochs": 30, "loss": loss, "seconds": time.perf_counter() - t0,
                       "precision": "BF16 tensor-core products, FP32 master weights, Adam"}
    w = ctx.mlp_get()
    n = 256 ** 3
    dev = torch.device("cuda", local_rank)
    ql = torch.empty(5 * n, dtype=torch.float64, device=dev)
    qr = torch.empty_like(ql)
    gam = torch.empty(n, dtype=torch.float64, device=dev)
    ctx.stress_states(n, 20261203, ql.data_ptr(), qr.data_ptr(), gam.data_ptr())
    res = {}
    for learned in (False, True):
        f = torch.empty(5 * n, dtype=torch.float64, device=dev)
        ps = torch.empty(n, dtype=torch.float64, device=dev)
        it = torch.empty(n, dtype=torch.int32, device=dev)
        call = lambda: ctx.exact_batch(n, ql.data_ptr(), qr.data_ptr(), gam.data_ptr(), f.data_ptr(), ps.data_ptr(),
                                       it.data_ptr(), learned=learned, niter=100, tol=1e-14)
        call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(5):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 5
        hist = torch.bincount(it.long(), minlength=101).cpu().numpy()
        cdf = np.cumsum(hist) / n
        res[learned] = (f, ps, {"mean_iters": float((hist * np.arange(len(hist))).sum() / n),
                                "p99_iters": int(np.searchsorted(cdf, 0.99)),
                                "at_cap_count": int(hist[100:].sum()), "max_iters": int(np.flatnonzero(hist).max()),
                                "ms": ms,
                                "interfaces_per_s": n / (ms / 1e3)})
    (f0, p0, a), (f1, p1, b) = res[False], res[True]
    rel = ((p1 - p0).abs() / p0.abs().clamp_min(1e-300))
    frel = ((f1 - f0).abs() / f0.abs().clamp_min(1e-300))
    out["stress"] = {"workload": "256^3 independent interface pairs: rho ratio to 1e4, p ratio to 1e6, "
                                 "30% strong double rarefactions, gamma 5/3 or 1.4, seed 20261203",
                     "interfaces": n, "plain": a, "learned": b,
                     "iteration_ratio": a["mean_iters"] / b["mean_iters"],
                     "polish_updates_per_interface": 2,
                     "iteration_ratio_with_polish": (a["mean_iters"] + 2) / (b["mean_iters"] + 2),
                     "pstar_rel_max": float(rel.max()), "pstar_rel_gt_1e-13_count": int((rel > 1e-13).sum().item()),
                     "pstar_bits_differ_count": int((p1 != p0).sum().item()),
                     "flux_rel_gt_1e-12_count": int((frel > 1e-12).sum().item()),
                     "note": "converged mode: bracketed Newton-bisection to |dp|/p < 1e-14, then 2 polish updates "
                             "from the root's 30 leading bits (counted apart: the same for both starts)"}
    # reference mode (10 updates, 1e-6: RiemannSolver.cpp:220-235) on a strided
    # sample of the same pairs against the reference's own solve_godunov_nr
    m = 65536
    idx = torch.arange(0, n, n // m, device=dev)[:m]
    fr = torch.empty(5 * n, dtype=torch.float64, device=dev)
    ctx.exact_batch(n, ql.data_ptr(), qr.data_ptr(), gam.data_ptr(), fr.data_ptr(), 0, 0, learned=False, niter=10,
                    tol=1e-6)
    torch.cuda.synchronize()
    import tempfile
    tmp = Path(tempfile.mkdtemp()) / "stress_sample.npz"
    np.savez(tmp, ql=ql.view(5, n)[:, idx].cpu().numpy(), qr=qr.view(5, n)[:, idx].cpu().numpy(),
             gam=gam[idx].cpu().numpy(), flux=fr.view(5, n)[:, idx].cpu().numpy())
    del ql, qr, gam, f0, f1, p0, p1, res, rel, frel, fr
    ctx.close()
    torch.cuda.empty_cache()
    try:
        out["stress"]["reference_mode_vs_reference"] = run_sample("--stress-ref", str(tmp))
    finally:
        tmp.unlink(missing_ok=True)

    L = 8
    g = rg_tree.build_uniform(3, L)
    u0 = rg_tree.sedov_state(g, L)
    dx = 1.0 / 2 ** L
    sed = {}
    for learned in (False, True):
        c = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="exact", interpol_type=1, gamma=1.4,
                                          courant_factor=0.8, exact_niter=100, exact_tol=1e-14,
                                          exact_guess=1 if learned else 0), local_rank)
        c.set_stream(stream.cuda_stream)
        if learned:
            c.mlp_set(w)
        c.sync_topology(g)
        c.upload_state(u0, u0)
        for _ in range(3):
            c.level_substep(L, dx, pressure_cap=False, use_graph=True)
        c.synchronize()
        c.exact_stats(reset=True)
        cells = c.cell_updates(L)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            c.level_substep(L, dx, pressure_cap=False, use_graph=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        iters, calls = c.exact_stats()
        sed["learned" if learned else "plain"] = {"cell_updates_per_s": cells / (ms / 1e3), "ms_per_step": ms,
                                                   "iters_per_interface": iters / max(calls, 1)}
        c.close()
    sed["workload"] = ("3D Sedov blast, uniform 128^3, MonCen + exact solver (converged mode), gamma 1.4, courant "
                       f"0.8, {steps} substeps after 3")
    out["sedov_exact"] = sed
    return out


def ensemble_report(rank, world, local_rank, steps):
    """Config 4: 512 independent periodic boxes (edges 16..64, nx 1 and 3,
    planar Riemann problems, gamma 5/3) in one launch sequence per substep,
    each box with its own CFL step.  N > 1: the boxes are partitioned over the
    ranks by cell count and each rank steps its shard (no exchange)."""
    import torch
    import rg_ensemble as ens
    import rgpu
    dist = None
    if world > 1:
        import torch.distributed as dist
    t0 = time.perf_counter()
    specs = ens.box_specs(512)
    f = ens.Forest(ens.shard_boxes(specs, world)[rank])
    u0 = f.initial_state()
    build_s = time.perf_counter() - t0
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", gamma=5.0 / 3.0, courant_factor=0.8),
                       local_rank)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.sync_topology(f.grid)
    ctx.upload_state(u0, u0)
    ctx.set_level_boxes(f.level, f.first_oct, f.dx)
    ctx.set_level_lattices(f.level, *f.lattices())
    for _ in range(3):
        ctx.level_substep(f.level, 0.0, pressure_cap=False, use_graph=True)
    ctx.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ctx.level_substep(f.level, 0.0, pressure_cap=False, use_graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cells = f.cells
    if dist:
        t = torch.tensor([ms, float(cells)], device="cuda", dtype=torch.float64)
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        ms, cells = float(mx[0].item()), int(t[1].item())
    variant = ctx.face_config(f.level)
    ctx.close()
    if rank != 0:
        return None
    return {"workload": "512 periodic boxes, edges uniform in {16,24,32,48,64} (24, 48: nx=3), planar Riemann "
                        "problem with random normal, rho log-U[1e-3,1e3], p log-U[1e-4,1e4], u_n U[-3,3], gamma 5/3, "
                        "MonCen + HLLC, per-box CFL, seed 20261203",
            "boxes": 512, "cells_per_step": cells, "steps": steps, "ms_per_step": ms / steps,
            "value": cells * steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "sharding": "boxes partitioned over ranks by cell count, no exchange" if world > 1 else "one GPU",
            "face_variant": list(variant), "host_build_s": build_s}


def stress_ref(path):
    """The exact solver in reference mode on GPU against the reference's own
    RiemannSolver::solve_godunov_nr (compiled here) on a sample of the stress
    pairs: per flux entry, relative differences (3e-12 is the tolerance the
    ulp-level pow() differences between CUDA and glibc stay inside)."""
    import numpy as np
    sys.path.insert(0, str(ROOT / "tests"))
    from refsupport import RefHarness
    d = np.load(path)
    ql, qr, gam, got = d["ql"], d["qr"], d["gam"], d["flux"]
    h = RefHarness(3)
    sys.stdout.flush()
    saved, devnull = os.dup(1), os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # the reference prints its first solves
    try:
        want = np.array([h.riemann("exact", ql[:, i], qr[:, i], float(gam[i]))[:5] for i in range(ql.shape[1])]).T
    finally:
        import ctypes
        ctypes.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    return {"pairs": int(ql.shape[1]), "flux_entries": int(rel.size), "identical_frac": float(np.mean(got == want)),
            "within_3e-12_frac": float(np.mean(rel <= 3e-12)), "rel_max": float(rel.max()),
            "check": "GPU reference mode (10 updates, 1e-6) against the reference's solve_godunov_nr, compiled here"}


def _ensemble_box_oracle(index, steps):
    """One ensemble box alone, `steps` substeps with its own CFL step, by the C
    oracle (the CPU side of the ensemble parity check)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import numpy as np
    import rg_ensemble as ens
    from refsupport import GridArrays, Oracle, make_params
    spec = next(s for s in ens.box_specs(512) if s.index == index)
    f = ens.Forest([spec])
    b, g = f.boxes[0], f.gamma
    ga = GridArrays(ncoarse=b.ncoarse, ngridmax=b.ngridmax, ncell=b.ncell, nvar=b.nvar, nx=b.nx, ny=b.ny, nz=b.nz,
                    ncpu=1, nboundary=0, nlevelmax=b.nlevelmax, son=b.son, father=b.father, nbor=b.nbor, next=b.next,
                    headl=b.headl)
    orc = Oracle()
    params = make_params(3, slope_type=2, riemann="hllc", gamma=g)
    uold = f.box_state(0)
    unew = uold.copy()
    dts = []
    for _ in range(steps):
        dt = orc.courant(ga, 3, 5, spec.level, spec.dx, g, 0.8, uold, pressure_cap=False)
        dts.append(dt)
        orc.set_unew(ga, 3, 5, spec.level, uold, unew)
        orc.godunov_fine(ga, params, spec.level, dt, spec.dx, uold, unew)
        orc.set_uold(ga, 3, 5, spec.level, uold, unew)
    want = np.ascontiguousarray(uold.reshape(5, b.ncell)[:, b.cell_ids(spec.level) - 1])
    return index, hashlib.sha1(want.tobytes()).hexdigest(), dts


def ensemble_parity(local_rank, nbox=32, steps=3):
    """Config 4's parity check on a seeded, edge-stratified subset of the 512
    boxes (about the same number of boxes of every edge): the subset stepped
    together on the GPU (per-box CFL, brick face kernel over the boxes'
    lattices) against each box stepped alone by the C oracle, per-box state
    digests and dt bits compared."""
    import multiprocessing as mp

    import numpy as np
    import rg_ensemble as ens
    import rgpu
    specs = ens.box_specs(512)
    edges = sorted({s.edge for s in specs})
    per = {e: [s for s in specs if s.edge == e] for e in edges}
    subset = []
    k = 0
    while len(subset) < nbox:
        for e in edges:
            if len(subset) < nbox and k < len(per[e]):
                subset.append(per[e][k])
        k += 1
    f = ens.Forest(subset)
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", gamma=f.gamma, courant_factor=0.8), local_rank)
    try:
        ctx.sync_topology(f.grid)
        u0 = f.initial_state()
        ctx.upload_state(u0, u0)
        ctx.set_level_boxes(f.level, f.first_oct, f.dx)
        ctx.set_level_lattices(f.level, *f.lattices())
        dts = []
        for k in range(steps):
            ctx.level_substep(f.level, 0.0, pressure_cap=False, use_graph=k > 0)
            dts.append(ctx.level_box_dt(f.level, f.nbox))
        got = np.empty_like(u0)
        ctx.download_state(uold=got)
    finally:
        ctx.close()
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        res = pool.starmap(_ensemble_box_oracle, [(s.index, steps) for s in subset])
    want = {i: (d, t) for i, d, t in res}
    same_state = same_dt = 0
    for i, s in enumerate(f.specs):
        d = hashlib.sha1(np.ascontiguousarray(f.extract(got, i)).tobytes()).hexdigest()
        same_state += d == want[s.index][0]
        same_dt += all(float(dts[k][i]) == want[s.index][1][k] for k in range(steps))
    return {"boxes": nbox, "edges": {str(e): sum(1 for s in subset if s.edge == e) for e in edges},
            "substeps": steps, "cells": int(f.cells), "bit_identical_boxes": same_state, "same_dt_boxes": same_dt,
            "check": "GPU forest of the subset (brick face kernel, per-box CFL) against each box alone by the C oracle"}


def amr_sample(variant, steps, lmin=7, lmax=10, ngridmax=400000):
    """Config 3 through the reference's own AmrGrid / TreeUpdater / HydroSolver
    (the CPU reference, or the reference with the GPU drop-in); runs in its own
    process: the reference prints a line per flagged cell."""
    import hashlib
    sys.path.insert(0, str(ROOT / "tests"))
    from refsupport import AmrRun, RefHarness, namelist, sedov_ic
    nml = namelist(slope_type=2, riemann="hllc", levelmin=lmin, levelmax=lmax, err_grad_d=0.1, err_grad_p=0.1)
    h = RefHarness(3, variant).create(nml, ngridmax=ngridmax, levelmin=lmin, nlevelmax=lmax, gamma=1.4)
    hyd = [0.0]

    def on_g(run, il, dt, dx):
        t = time.perf_counter()
        run.h.godunov_fine(il, dt, dx)
        hyd[0] += time.perf_counter() - t

    # the hydro time covers every HydroSolver call of the step: with the GPU
    # drop-in the level's cells move in set_unew and set_uold
    for name in ("set_unew", "set_uold"):
        def timed(il, _f=getattr(h, name)):
            t = time.perf_counter()
            _f(il)
            hyd[0] += time.perf_counter() - t
        setattr(h, name, timed)

    r = AmrRun(h, lmin, lmax, 1.4, cfl=AMR["cfl"], ed=0.1, ep=0.1, on_godunov=on_g)
    r.initialize(sedov_ic(3, lmin))
    r.coarse_step()  # warm-up step (first-call costs)
    hyd[0] = 0.0
    cu0 = r.cell_updates
    t0 = time.perf_counter()
    for _ in range(steps):
        r.coarse_step()
    wall = time.perf_counter() - t0
    a = h.arrays()
    out = {"variant": variant, "coarse_steps": steps, "wall_s": wall, "hydro_s": hyd[0],
           "cell_updates": r.cell_updates - cu0, "t": r.t,
           "octs_per_level": [h.count_grids(il) for il in range(lmin, lmax + 1)],
           "digest": hashlib.sha1(a["uold"].tobytes() + a["son"].tobytes()).hexdigest()}
    h.close()
    return out


def amr_exact_sample(guess, steps, lmin=7, lmax=10, ngridmax=400000):
    """Config 5's AMR part: the sub-cycled Sedov AMR run (tree maintenance by
    the reference's own TreeUpdater) with every godunov_fine on the GPU through
    rg_godunov_level_host, exact solver in converged mode (|dp|/p < 1e-14),
    plain or learned Newton start; runs in its own process (the reference
    prints a line per flagged cell)."""
    import hashlib

    import numpy as np
    sys.path.insert(0, str(ROOT / "tests"))
    import rgpu
    from refsupport import AmrRun, RefHarness, namelist, sedov_ic
    learned = guess == "learned"
    nml = namelist(slope_type=2, riemann="exact", levelmin=lmin, levelmax=lmax, err_grad_d=0.1, err_grad_p=0.1)
    h = RefHarness(3).create(nml, ngridmax=ngridmax, levelmin=lmin, nlevelmax=lmax, gamma=1.4)
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="exact", exact_niter=100, exact_tol=1e-14,
                                        exact_guess=1 if learned else 0), 0)
    ctx.set_autotune(False)  # same face kernel shape for both starts, no tuning inside the timed steps
    if learned:
        ctx.mlp_train()
    sent = {}
    hyd = [0.0]

    def on_g(run, il, dt, dx):
        t = time.perf_counter()
        a = run.h.arrays()
        if any(k not in sent or not np.array_equal(sent[k], a[k]) for k in ("son", "father", "nbor", "next", "headl")):
            ctx.sync_topology(run.h.grid())
            for k in ("son", "father", "nbor", "next", "headl"):
                sent[k] = a[k].copy()
        ctx.godunov_level_host(il, dt, dx, a["uold"], a["unew"])
        hyd[0] += time.perf_counter() - t

    r = AmrRun(h, lmin, lmax, 1.4, ed=0.1, ep=0.1, on_godunov=on_g)
    r.initialize(sedov_ic(3, lmin))
    r.coarse_step()  # warm-up step (plans, autotuner)
    ctx.exact_stats(reset=True)
    hyd[0] = 0.0
    cu0 = r.cell_updates
    t0 = time.perf_counter()
    for _ in range(steps):
        r.coarse_step()
    wall = time.perf_counter() - t0
    iters, calls = ctx.exact_stats()
    a = h.arrays()
    out = {"guess": guess, "coarse_steps": steps, "wall_s": wall, "hydro_s": hyd[0],
           "cell_updates": r.cell_updates - cu0, "hydro_cell_updates_per_s": (r.cell_updates - cu0) / hyd[0],
           "iters_per_interface": iters / max(calls, 1), "interfaces": calls,
           "digest": hashlib.sha1(a["uold"].tobytes()).hexdigest()}
    ctx.close()
    h.close()
    return out


def sod_sample(variant):
    """Config 1: 1D Sod, 1024 cells (reference levelmin=levelmax=11), MinMod +
    HLLC, reference CFL (courant 0.8; p <= 100 rho holds), to t = 0.245."""
    import hashlib

    import numpy as np
    import rg_tree
    L, gamma, tend = 11, 1.4, 0.245
    g = rg_tree.build_uniform(1, L)
    ids = g.cell_ids(L)
    dx = 1.0 / 2 ** L
    t, n = 0.0, 0
    if variant == "cpu":
        sys.path.insert(0, str(ROOT / "tests"))
        import refsupport as rs
        h = rs.RefHarness(1).create(rs.namelist(slope_type=1, riemann="hllc", levelmin=L, levelmax=L),
                                    ngridmax=g.ngridmax, levelmin=L, nlevelmax=L, gamma=gamma)
        h.refine_uniform(L)
        a = h.arrays()
        u = rg_tree.sod_state(g, L, gamma)
        a["uold"][:] = u
        a["unew"][:] = u
        t0 = time.perf_counter()
        while t < tend:
            dt = h.courant(L, dx, gamma, 0.8)
            h.set_unew(L)
            h.godunov_fine(L, dt, dx)
            h.set_uold(L)
            t += dt
            n += 1
        wall = time.perf_counter() - t0
        final = np.array(a["uold"]).reshape(3, -1)[:, ids - 1]
        h.close()
    else:
        import rgpu
        ctx = rgpu.Context(rgpu.make_params(1, slope_type=1, riemann="hllc", gamma=gamma, courant_factor=0.8), 0)
        ctx.sync_topology(g)
        u = rg_tree.sod_state(g, L, gamma)
        ctx.upload_state(u, u)
        t0 = time.perf_counter()
        t, n = ctx.level_run(L, dx, tend, pressure_cap=True)  # the whole run: one graph launch
        ctx.synchronize()
        wall = time.perf_counter() - t0
        out = np.empty_like(u)
        ctx.download_state(uold=out)
        ctx.close()
        final = out.reshape(3, -1)[:, ids - 1]
    return {"variant": variant, "steps": n, "t": t, "wall_s": wall, "cell_updates": n * len(ids),
            "digest": hashlib.sha1(np.ascontiguousarray(final).tobytes()).hexdigest()}


def profile_case_learned():
    """A small run of the learned part for ncu captures: training on 1e6 stress
    states for 2 epochs (launches: one k_exact_batch for the labels, then
    k_mlp_grad + k_adam per batch), then the exact solver on 4M stress pairs
    with the plain start (k_exact_batch #1) and the learned start (the
    tensor-core starts, k_mlp_guess_tc, then k_exact_batch #2 from them)."""
    import torch
    import rgpu
    ctx = rgpu.Context(rgpu.make_params(3, riemann="exact"), 0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.mlp_train(nsamples=1_000_000, epochs=2)
    n = 1 << 22
    ql = torch.empty(5 * n, dtype=torch.float64, device="cuda")
    qr = torch.empty_like(ql)
    gam = torch.empty(n, dtype=torch.float64, device="cuda")
    f = torch.empty_like(ql)
    ps = torch.empty(n, dtype=torch.float64, device="cuda")
    it = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.stress_states(n, 2026, ql.data_ptr(), qr.data_ptr(), gam.data_ptr())
    for learned in (False, True):
        ctx.exact_batch(n, ql.data_ptr(), qr.data_ptr(), gam.data_ptr(), f.data_ptr(), ps.data_ptr(), it.data_ptr(),
                        learned=learned, niter=100, tol=1e-14)
    ctx.synchronize()
    ctx.close()


def profile_case_amr():
    """A small run for ncu captures of the AMR step: the headline's run
    initialised on the device and 10 coarse steps, two coarse steps without a
    tree change (coarse steps 11 and 12, replayed graphs) inside the NVTX range
    "steps" (the launch list), then one level step each of level 7 (the 64^3
    base level) and level 10 (the finest) inside the NVTX range "capture"
    (ncu --nvtx --nvtx-include capture/)."""
    import torch
    import rgpu
    ctx = rgpu.Context(amr_params(rgpu), 0)
    run = amr_run(ctx)
    for _ in range(10):
        run.coarse_step()
    ctx.synchronize()
    torch.cuda.nvtx.range_push("steps")  # two whole coarse steps: the launch list
    for _ in range(2):
        run.coarse_step()
    ctx.synchronize()
    torch.cuda.nvtx.range_pop()
    torch.cuda.nvtx.range_push("capture")
    cells = {}
    for il in (7, 10):
        ctx.godunov_level(il, 1e-7, 1.0 / 2 ** il)
        cells[il] = ctx.cell_updates(il)
    ctx.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile_case": "amr", "cell_updates_per_launch": cells,
                      "face_variants": {il: ctx.face_config(il)[0] for il in (7, 10)}}))
    ctx.close()


def profile_case_uniform():
    """A small run for ncu captures of the brick face kernel: the uniform
    128^3 Sedov level, two warm-up substeps, then one eager substep inside the
    NVTX range "capture"."""
    import torch
    import rg_tree
    import rgpu
    L = 8
    g = rg_tree.build_uniform(3, L)
    u0 = rg_tree.sedov_state(g, L)
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", interpol_type=1, gamma=1.4,
                                        courant_factor=0.8), 0)
    ctx.sync_topology(g)
    ctx.upload_state(u0, u0)
    ctx.set_face_config(L, 10, 1)
    for _ in range(2):
        ctx.level_substep(L, 1.0 / 2 ** L, pressure_cap=False, use_graph=False)
    ctx.synchronize()
    torch.cuda.nvtx.range_push("capture")
    ctx.level_substep(L, 1.0 / 2 ** L, pressure_cap=False, use_graph=False)
    ctx.synchronize()
    torch.cuda.nvtx.range_pop()
    ctx.close()


def run_sample(flag, *args, timeout=900):
    cmd = [sys.executable, str(Path(__file__).resolve()), flag, *[str(a) for a in args]]
    # load every kernel when the context is created (in the sample's untimed
    # warm-up) instead of on its first launch inside the timed steps
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    for line in reversed(r.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError(f"{flag} failed: " + r.stderr[-2000:])


def amr_report(steps):
    """The AMR run through the reference's own AmrGrid / TreeUpdater /
    Simulation step, CPU hydro against the GPU drop-in (the reference-facing
    plugin: GpuHydroSolver through create_hydro_solver), coarse steps 2..1+steps."""
    ref = run_sample("--amr-sample", "cpu", steps)
    gpu = run_sample("--amr-sample", "gpu", steps)
    return {"workload": "the headline's Sedov AMR run through the reference's own AmrGrid/TreeUpdater/Simulation "
                        "step with the hydro solver swapped by create_hydro_solver",
            "coarse_steps": steps, "after": "initialisation and one warm-up coarse step",
            "reference_cpu": ref, "gpu_dropin": gpu, "bit_identical": ref["digest"] == gpu["digest"],
            "wall_speedup": ref["wall_s"] / gpu["wall_s"], "hydro_speedup": ref["hydro_s"] / gpu["hydro_s"],
            "gpu_hydro_cell_updates_per_s": gpu["cell_updates"] / gpu["hydro_s"],
            "note": "tree maintenance (flag/refine/restrict) on the host as in the reference; hydro time = "
                    "set_unew + godunov_fine + set_uold calls; the drop-in keeps the state on the device and moves "
                    "each level's cells in set_unew (up) and set_uold (down)"}


def amr_exact_report(steps):
    plain = run_sample("--amr-exact-sample", "plain", steps)
    learned = run_sample("--amr-exact-sample", "learned", steps)
    return {"workload": "3D Sedov AMR (levelmin 7, levelmax 10) with the exact solver in converged mode, tree "
                        "maintenance by the reference, every godunov_fine on the GPU (rg_godunov_level_host)",
            "plain": plain, "learned": learned,
            "iteration_ratio": plain["iters_per_interface"] / max(learned["iters_per_interface"], 1e-30),
            "same_state_bits": plain["digest"] == learned["digest"]}


def sod_report():
    ref = run_sample("--sod-sample", "cpu")
    gpu = run_sample("--sod-sample", "gpu")
    return {"workload": "1D Sod, 1024 cells (reference levelmin=levelmax=11), MinMod + HLLC, courant 0.8, "
                        "to t=0.245", "reference_cpu": ref, "gpu": gpu,
            "bit_identical": ref["digest"] == gpu["digest"] and ref["steps"] == gpu["steps"],
            "wall_speedup": ref["wall_s"] / gpu["wall_s"],
            "note": "GPU run: rg_level_run, all 1729 substeps in one CUDA graph launch whose WHILE node stops "
                    "at t >= 0.245 on the device (no dt read back between substeps); 1024 cells per substep, so "
                    "it is launch-latency bound"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--face-variant", type=int, default=None,
                    help="face-kernel shape of the uniform 128^3 report (0-10) instead of the autotuner's pick; "
                         "for profiler runs, whose serialised launches would skew the autotuner's timings")
    ap.add_argument("--no-newton", action="store_true", help="skip the exact-solver plain/learned report")
    ap.add_argument("--no-extra", action="store_true", help="skip the uniform, ensemble, drop-in and Sod reports")
    ap.add_argument("--amr-cpu-window", nargs=3, type=int, metavar=("WARMUP", "STEPS", "PARITY"),
                    help=argparse.SUPPRESS)
    ap.add_argument("--amr-sample", nargs=2, metavar=("VARIANT", "STEPS"), help=argparse.SUPPRESS)
    ap.add_argument("--sod-sample", metavar="VARIANT", help=argparse.SUPPRESS)
    ap.add_argument("--amr-exact-sample", nargs=2, metavar=("GUESS", "STEPS"), help=argparse.SUPPRESS)
    ap.add_argument("--stress-ref", metavar="NPZ", help=argparse.SUPPRESS)
    ap.add_argument("--profile-case", choices=["learned", "amr", "uniform"],
                    help="small run for ncu captures (no timing output)")
    args = ap.parse_args()
    if args.amr_cpu_window:
        w, k, par = args.amr_cpu_window
        print(json.dumps(amr_cpu_window(w, k, par or None)))
        return
    if args.amr_sample:
        print(json.dumps(amr_sample(args.amr_sample[0], int(args.amr_sample[1]))))
        return
    if args.sod_sample:
        print(json.dumps(sod_sample(args.sod_sample)))
        return
    if args.stress_ref:
        print(json.dumps(stress_ref(args.stress_ref)))
        return
    if args.amr_exact_sample:
        print(json.dumps(amr_exact_sample(args.amr_exact_sample[0], int(args.amr_exact_sample[1]))))
        return
    if args.profile_case:
        {"learned": profile_case_learned, "amr": profile_case_amr, "uniform": profile_case_uniform}[args.profile_case]()
        return
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if world > 1 and rank != 0:
            return
        out = reference_arm(args, rank, world)
        print(json.dumps(out))
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    cpu = cpu_run = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference on one core, before any CUDA work: its initialisation,
        # the W warm-up coarse steps and the first 2 coarse steps of the window
        cpu_run = run_cpu_window(args.warmup, 2, parity_after=args.warmup + 2)
        cpu = {"value": cpu_run["cells"] / cpu_run["seconds"], "unit": UNIT, "cores": 1, "kind": "reference",
               "sample": f"coarse steps {args.warmup + 1}..{args.warmup + 2} of the same AMR run (the first two of "
                         f"the window, {cpu_run['cells']} cell updates, {cpu_run['seconds']:.1f} s) after the "
                         f"reference's own initialisation and {args.warmup} coarse steps, single-threaded"}
    out = amr_headline(args, rank, world, local_rank)
    # the other configs' reports run on one GPU only: with N > 1 the other
    # ranks would wait for rank 0's single-GPU work at the final barrier; the
    # ensemble, whose boxes shard over the ranks, runs at every N
    single = world == 1
    if rank == 0:
        if cpu_run:
            out["parity_digest"]["reference_sha1_uold_son"] = cpu_run["digest"]
            out["parity_digest"]["bit_identical"] = cpu_run["digest"] == out["parity_digest"]["sha1_uold_son"]
        if single and not args.no_extra:
            out["sedov128"] = uniform_report(local_rank, 20, 3, args.face_variant)
    if rank == 0 and single and not args.no_newton:
        import torch
        out["newton"] = newton_report(local_rank, torch.cuda.Stream(), 10)
    if not args.no_extra:
        ens_out = ensemble_report(rank, world, local_rank, 100)
        if rank == 0:
            out["ensemble"] = ens_out
            if single:
                out["ensemble"]["parity"] = ensemble_parity(local_rank)
                out["amr_dropin"] = amr_report(3)
                if "newton" in out:
                    out["newton"]["amr_exact"] = amr_exact_report(3)
                out["sod1d"] = sod_report()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        out["cpu_baseline"] = cpu
        print(json.dumps(out))


if __name__ == "__main__":
    main()
