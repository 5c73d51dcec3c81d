#!/usr/bin/env python3
"""Throughput of the tracer advection step on B200.

Workload (the plain method at scale): doubly periodic analytic mesh
nx = ny = 1000 (998,001 nodes, 2,994,003 edges, 1,996,002 triangles), 64
levels, smooth seeded bathymetry with per-node bottom level uniform in
[3, 64] (seed 0), a seeded smooth layered flow that is discretely
divergence-free (|u| <= 1 m/s, w from continuity, dt at CFL 0.5 of the
faster of the horizontal and vertical crossings), two tracers
(temperature-like U[0,20] + Gaussian blobs, salinity-like 35 + N(0, 0.5)),
MUSCL + PPM + FCT in FP64, valuesAB := values each step
(fesom2_tracer_dwarf_b200.workloads.layered_flow_case).  One "step" advances
both tracers once.  Metric: tracer cell-updates/s = wet cells x tracers /
step time.

Arms:
  default            this library, through its C ABI (device-resident inputs
                     for "value"; host buffers copied in and out every step for
                     "e2e")
  --impl reference   the reference algorithm on the host cores: the CPU
                     oracle (a C restatement of the reference's Fortran, which
                     cannot be compiled here: no Fortran compiler), OpenMP over
                     all host threads, on the same full-size workload, with
                     inputs built by the oracle's own restatement of the
                     seeded generators (the product library is not loaded).

Multi-GPU (torchrun): every rank advects its own replica of the workload on
its own GPU with no data-path collective (weak scaling); a barrier brackets
the timed region and the device time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# 14 words per wet cell and tracer at storage precision: 3 tracer words
# (T read, T_AB read, T write) + 11 geometry / flow words
BYTES_PER_CELL = {"fp64": 112, "fp64fma": 112, "fp32": 56, "bf16": 3 * 2 + 11 * 4, "fp16": 3 * 2 + 11 * 4}
DTYPE = {"fp64": "f64", "fp64fma": "f64 (FMA-contracted kernels)", "fp32": "f32",
         "bf16": "bf16 storage / f32 compute", "fp16": "f16 storage / f32 compute"}
L2_BYTES = 126 * 2**20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nx", type=int, default=1000)
    p.add_argument("--nl", type=int, default=64)
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--precision", default="fp64", choices=["fp64", "fp64fma", "fp32", "bf16", "fp16"])
    p.add_argument("--step-path", default="five", choices=["fused", "five"],
                   help="the five-kernel path (default) or the fused patch kernel")
    p.add_argument("--cells-per-block", type=int, default=0,
                   help="most wet cells per block of the five-kernel schedules (0: the default, 512)")
    p.add_argument("--learned", action="store_true",
                   help="FP32 with the learned antidiffusive flux (shipped parameters) ahead of FCT")
    p.add_argument("--config", default="c2", choices=["c2", "c3", "c4", "dd"],
                   help="c2: the plain method at scale (default); c3: 48 tracers x 8 uneven members, one "
                        "persistent launch per step; c4: BF16/FP16/FP32 storage against FP64 at 2000x2000x48; "
                        "dd: the 1000x1000x64 step cut into strips on one GPU")
    p.add_argument("--parts", type=int, nargs="+", default=[2, 4, 8], help="dd: strip counts")
    a = p.parse_args()
    if a.learned:
        a.precision = "fp32"
    return a


def workload_name(nx, nl):
    return (f"periodic {nx}x{nx}x{nl} (left-oriented edges), smooth bathymetry U[3,{nl}] seed 0, "
            "divergence-free layered flow CFL 0.5, MUSCL+PPM+FCT, 2 tracers")


def workload_config(nx, nl, cells, dt, gpus):
    """The workload description both arms print (identical for the same
    workload): per-step algorithmic FP64 traffic against the L2 size."""
    step_gb = BYTES_PER_CELL["fp64"] * cells * 2 / 1e9
    return {"workload": workload_name(nx, nl), "wet_cells": cells, "tracers": 2, "dt_s": dt,
            "parallelism": f"replicas x{gpus}",
            "l2": f"inputs larger than L2 ({step_gb:.2f} GB of FP64 fields per step vs {L2_BYTES / 1e9:.2f} GB L2)",
            "bathymetry": "bottom levels from a smooth seeded random field with a uniform [3, nl] marginal "
                          "(independent per-node levels make the layered divergence-free flow grid-scale in the "
                          "vertical and blow up); neighbouring columns therefore have similar depths, which keeps "
                          "the wet-cell blocks of the schedule fuller than independent levels would"}


def make_inputs(api, nx, nl):
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, nx, nl, seed=0)
    return c.K, c.uv, c.w, c.T, c.S, c.dt, c.wet_cells


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-i", str(self.gpu),
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), float(f[3]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        loaded = [r for r in rows if r[2] > 200.0] or rows
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in loaded:
            for nm, v in zip(names, r[3:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(loaded)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(args):
    """DRAM bytes per step of the plain FP64 step at 1000x1000x64 from the
    committed ncu summary (profiles/step_c2_fp64.md, line
    'dram_bytes_per_step_scaled: X'); None for any other workload or
    precision, which that capture does not cover."""
    p = ROOT / "profiles" / "step_c2_fp64.md"
    if (args.precision != "fp64" or args.learned or args.nx != 1000 or args.nl != 64 or args.step_path != "five"
            or not p.exists()):
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_step_scaled:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# CPU arm: the oracle (a C restatement of the reference's Fortran) on the same
# workload.  Its inputs are built by the oracle's own restatement of the
# seeded generators (bit-identical to the library's, tests/test_synth_oracle.py),
# so this arm never loads the product library.
# ---------------------------------------------------------------------------
def cpu_run(nx, nl, steps, warmup=1, serial=False):
    """Runs the oracle (OpenMP on every host thread, or the serial build) on
    the periodic nx^2 x nl layered-flow workload, 2 tracers, MUSCL+PPM+FCT,
    valuesAB := values.  Returns (rate, threads, sample text, per-step
    seconds)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    o = pyoracle.Oracle(openmp=not serial)
    if not serial:
        o.set_threads(os.cpu_count() or 1)
    m, K, uv, w, T, S, dt, cells = pyoracle.layered_flow_case(o, nx, nl, seed=0)
    vals = np.ascontiguousarray(np.stack([T.T, S.T]))  # (2, nod2D, nl-1): each tracer a Fortran (nl-1, nod2D) block
    ab = vals.copy()
    if warmup:
        m.run(vals, ab, uv, w, dt, warmup, "MUSCL", "PPM", "FCT", refresh_ab=True)
    per = []
    for _ in range(steps):
        t0 = time.perf_counter()
        m.run(vals, ab, uv, w, dt, 1, "MUSCL", "PPM", "FCT", refresh_ab=True)
        per.append(time.perf_counter() - t0)
    sec = statistics.median(per)
    rate = 2 * cells / sec
    what = "the full workload" if nx == 1000 and nl == 64 else "a sample"
    sample = (f"{what}: periodic {nx}x{nx}x{nl} ({m.nod2D} nodes, {cells} wet cells), inputs from the oracle's "
              f"restatement of the seeded generators, 2 tracers, median of {steps} steps after {warmup} warm-up")
    return rate, (1 if serial else o.threads()), sample, per, cells, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    steps = max(1, args.steps)
    warmup = max(1, min(args.warmup, 2))
    rate, threads, sample, per, cells, dt = cpu_run(args.nx, args.nl, steps, warmup=warmup)
    sec = statistics.median(per)
    line = {
        "metric": "tracer cell-updates/s", "value": rate, "unit": "cell-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.nx, args.nl, cells, dt, args.gpus),
        "sample": sample,
        "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_ours(args):
    from fesom2_tracer_dwarf_b200.replicas import from_env, job_rate
    ranks = from_env("nccl")
    rank, world, local = ranks.rank, ranks.world, ranks.local

    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    api = FESOMTracerAdvection()
    api.cleanup()
    if api.lib.tracer_set_device(local) != 0:
        raise RuntimeError(api.lib.tracer_last_error().decode())
    K, uv, w, T, S, dt, cells = make_inputs(api, args.nx, args.nl)
    api.set_precision(args.precision)
    api.set_step_path(args.step_path)
    if args.cells_per_block:
        api.set_cells_per_block(args.cells_per_block)
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    for t in (1, 2):
        api.set_scheme(t, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    if args.learned:
        from fesom2_tracer_dwarf_b200.learned import trained_params
        params = trained_params()
        if api.lib.tracer_learn_set(params.ctypes.data_as(ctypes.c_void_p), 1) != 0:
            raise RuntimeError(api.lib.tracer_last_error().decode())
    api.advect_steps(args.warmup, dt)
    launches_per_step = api.lib.tracer_launches_per_step()
    dev_bytes = api.lib.tracer_device_bytes()

    barrier = ranks.barrier

    # device-resident throughput, CUDA events on the engine's stream
    clock = ClockSampler(local)
    clock.start()
    barrier()
    ms = api.time_steps(args.steps, dt)
    barrier()
    clocks = clock.stop()
    ms = ranks.max(ms)
    ms_per_step = ms / args.steps
    value = job_rate(2 * cells, world, ms_per_step / 1e3)

    # per-kernel breakdown (events around each launch), untimed otherwise
    nk = 8
    kms = np.zeros(nk)
    names = (ctypes.c_char_p * nk)()
    launches = np.zeros(1, dtype=np.int32)
    prof_steps = max(2, min(args.steps, 5))
    rc = api.lib.tracer_profile_steps(prof_steps, dt, kms.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.cast(names, ctypes.c_void_p), nk,
                                      launches.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise RuntimeError(api.lib.tracer_last_error().decode())
    kernel_ms = {names[i].decode(): kms[i] / prof_steps for i in range(nk) if names[i]}

    # end to end through the C ABI with host buffers: set both tracers from
    # host memory, one step, read both back, every step.  The headline uses
    # page-locked host arrays (tracer_host_register); the same loop on
    # pageable arrays goes through the library's pinned staging ring.
    L, N = args.nl - 1, T.shape[1]

    def e2e_loop(arrays):
        Th, Sh, outT, outS = arrays
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            api.set_values(1, Th)
            api.set_values(2, Sh)
            if api.advect_step(dt) != 0:
                raise RuntimeError(api.lib.tracer_last_error().decode())
            api.lib.tracer_get_values_id(1, outT.ctypes.data_as(ctypes.c_void_p), L, N)
            api.lib.tracer_get_values_id(2, outS.ctypes.data_as(ctypes.c_void_p), L, N)
        return ranks.max((time.perf_counter() - t0) / args.e2e_steps)

    def e2e_io_loop(arrays):
        """The same work through tracer_advect_step_io: both uploads, the
        per-tracer steps and both downloads pipelined on three streams."""
        Th, Sh, outT, outS = arrays
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            api.advect_step_io(dt, [Th, Sh], [outT, outS])
        return ranks.max((time.perf_counter() - t0) / args.e2e_steps)

    def ref_loop():
        """The reference harness's loop (src/fesom_analytic.F90:385-449):
        one step, then min / max / sum of tracer 1 read back, every step."""
        st = np.zeros(4)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            if api.advect_step(dt) != 0:
                raise RuntimeError(api.lib.tracer_last_error().decode())
            api.lib.tracer_get_stats_id(1, st.ctypes.data_as(ctypes.c_void_p))
        return ranks.max((time.perf_counter() - t0) / args.e2e_steps)

    ref_loop()
    ref_loop_sec = ref_loop()

    host = [np.asfortranarray(api.get_tracer_values(1)), np.asfortranarray(api.get_tracer_values(2)),
            np.zeros((L, N), order="F"), np.zeros((L, N), order="F")]
    e2e_pageable_sec = e2e_loop(host)
    for a in host:
        api.pin(a)
    e2e_loop(host)  # warm-up of the registered path
    e2e_serial_sec = e2e_loop(host)
    e2e_io_loop(host)  # warm-up (per-tracer buffers, streams)
    e2e_sec = e2e_io_loop(host)
    for a in host:
        api.unpin(a)
    h2d = 2 * L * N * 8  # the C ABI exchanges FP64 arrays whatever the device precision
    d2h = 2 * L * N * 8

    result = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        alg_bytes_step = BYTES_PER_CELL[args.precision] * cells * 2
        achieved = alg_bytes_step / (ms_per_step / 1e3) / 1e9
        traffic = committed_traffic(args)
        result = {
            "metric": "tracer cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[args.precision], "data": "synthetic",
            "config": dict(workload_config(args.nx, args.nl, cells, dt, world),
                           **({"cells_per_block": args.cells_per_block} if args.cells_per_block else {})),
            "device_bytes": dev_bytes,
            "precision": args.precision + (", learned antidiffusive flux (MLP on tcgen05) ahead of FCT"
                                           if args.learned else ""),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the five step "
                                            "kernels of one step on the 300x300x64 case of this workload, scaled by "
                                            "wet cells (x11.17) to this size; profiles/step_c2_fp64.md"
                                            if traffic else None),
                         "kernel": f"full step (all kernels of one step, {BYTES_PER_CELL[args.precision]} B/cell algorithmic)",
                         "peak_source": f"{peak_kind} hbm_gbs"},
            "kernel_ms_per_step": kernel_ms,
            "e2e": {"value": world * 2 * cells / e2e_sec, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "host_memory": "page-locked (tracer_host_register)",
                    "api": "tracer_advect_step_io (uploads, per-tracer steps, downloads pipelined)",
                    "ms_per_step": e2e_sec * 1e3},
            "e2e_serial": {"value": world * 2 * cells / e2e_serial_sec, "unit": "cell-updates/s",
                           "api": "tracer_set_values x2, tracer_advect_step, tracer_get_values_id x2",
                           "ms_per_step": e2e_serial_sec * 1e3},
            "e2e_pageable": {"value": world * 2 * cells / e2e_pageable_sec, "unit": "cell-updates/s",
                             "ms_per_step": e2e_pageable_sec * 1e3},
            "reference_loop": {"value": world * 2 * cells / ref_loop_sec, "unit": "cell-updates/s",
                               "what": "tracer_advect_step + tracer_get_stats every step (the reference "
                                       "harness's loop; state stays on the device)",
                               "ms_per_step": ref_loop_sec * 1e3},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
        }
    ranks.close()
    api.cleanup()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same workload at full size, a few steps (about 10-30 s of CPU work)
        rate, threads, sample, _, _, _ = cpu_run(args.nx, args.nl, 3)
        result["cpu_baseline"] = {"value": rate, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                                  "sample": sample}
        # the reference's own build is serial: the same oracle on one thread,
        # on a smaller mesh of the same recipe (a full-size serial step takes
        # about a minute)
        rate1, _, sample1, _, _, _ = cpu_run(min(args.nx, 150), args.nl, 3, serial=True)
        result["cpu_baseline_serial"] = {"value": rate1, "unit": "cell-updates/s", "cores": 1, "kind": "port",
                                         "sample": sample1}
    if rank == 0:
        print(json.dumps(result))
    return 0


# ---------------------------------------------------------------------------
# further configurations (one GPU; each prints one JSON line with the clocks
# sampled while it was timed)
# ---------------------------------------------------------------------------
def timed(gpu, fn):
    """Runs fn() with the clock sampler on; returns (fn's result, clocks)."""
    clock = ClockSampler(gpu)
    clock.start()
    try:
        out = fn()
    finally:
        clocks = clock.stop()
    return out, clocks


def run_c3(args):
    """48 tracers x 8 ensemble members on seeded analytic meshes of uneven
    size (nx = ny in [100, 800], nl in [20, 80], periodic and closed mixed),
    FP32 MUSCL+PPM+FCT: every batched path at the tile the autotuner picks
    (one persistent launch per phase and wave, one cooperative launch per
    step, the members' own per-batch launches), each replayed from a CUDA
    graph; the line's value is the fastest."""
    import re
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    from fesom2_tracer_dwarf_b200.batch import TracerBatch
    from fesom2_tracer_dwarf_b200.workloads import build_ensemble, ensemble_specs
    specs = ensemble_specs(8, 0, (100, 800), (20, 80))
    api = FESOMTracerAdvection()
    batch = TracerBatch()
    dts = build_ensemble(batch, api, specs, 48)
    batch.configure(dts, "MUSCL", "PPM", "FCT")
    info = batch.info()
    log = batch.autotune(2)
    tuned = {}
    for ln in log.splitlines():
        mt = re.match(r"path=(\w+) .*ms_per_step=([0-9.eE+-]+)", ln)
        if mt:
            tuned[mt.group(1)] = min(tuned.get(mt.group(1), 1e30), float(mt.group(2)))
    tile = batch.tile()
    chosen = batch.path()
    steps = max(args.steps, 1)
    paths, clocks_of = {}, {}
    for path in ("phases", "cooperative"):
        batch.set_path(path)
        batch.steps(max(args.warmup, 3), graph=True)
        ms_g, clocks_of[f"{path}_graph"] = timed(0, lambda: batch.time_steps(steps, graph=True) / steps)
        paths[f"{path}_graph"] = ms_g
        paths[f"{path}_no_graph"] = batch.time_steps(steps, graph=False) / steps
    batch.set_path(chosen)
    paths["separate_launches"] = batch.time_separate(steps) / steps
    paths["separate_launches_graph"], clocks_of["separate_launches_graph"] = timed(
        0, lambda: batch.time_separate(steps, graph=True) / steps)
    best = min(clocks_of, key=lambda k: paths[k])
    ms_graph, clocks = paths[best], clocks_of[best]
    cells = info["cell_tracers"]
    batch.close()
    api.cleanup()
    line = {"metric": "tracer cell-updates/s", "value": cells / (ms_graph / 1e3), "unit": "cell-updates/s",
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ms_graph, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "48 tracers x 8 members, nx=ny in [100,800], nl in [20,80], periodic/closed "
                                   f"mixed, seeds 0..7, MUSCL+PPM+FCT, the fastest batched path ({best})",
                       "members": specs, "cell_tracers": cells, "tile": tile, "autotuned_path": chosen,
                       "path": best},
            "paths_ms_per_step": paths, "autotune_best_ms_per_step": tuned,
            "clocks": clocks}
    print(json.dumps(line))
    return 0


def run_c4(args):
    """2000x2000x48 (or --nx/--nl), 200 steps by default: every storage mode
    against the bit-exact FP64 path on identical seeded inputs -- time per
    step (clocks sampled per mode), relative L2 and max-abs error over wet
    cells, content drift."""
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    from fesom2_tracer_dwarf_b200.precision import compare, run_mode
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    nx = args.nx if args.nx != 1000 else 2000
    nl = args.nl if args.nl != 64 else 48
    steps = args.steps if args.steps != 100 else 200
    api = FESOMTracerAdvection()
    api.cleanup()
    api.lib.tracer_set_device(0)
    c = layered_flow_case(api, nx, nl, seed=0)
    ref, clk = timed(0, lambda: run_mode(api, c, "fp64", steps))
    modes = {"fp64": {"ms_per_step": ref["ms_per_step"], "clocks": clk,
                      "cell_updates_per_s": 2 * c.wet_cells / (ref["ms_per_step"] / 1e3)}}
    for m in ("fp64fma", "fp32", "bf16", "bf16+sr", "fp16", "fp16+sr"):
        res, clk = timed(0, lambda: run_mode(api, c, m, steps))
        modes[m] = {"ms_per_step": res["ms_per_step"], "clocks": clk,
                    "cell_updates_per_s": 2 * c.wet_cells / (res["ms_per_step"] / 1e3),
                    "errors": compare(ref, res)}
    api.cleanup()
    best = modes["bf16+sr"]
    line = {"metric": "tracer cell-updates/s", "value": best["cell_updates_per_s"], "unit": "cell-updates/s",
            "n_gpus": 1, "steps": steps, "warmup": 0, "ms_per_step": best["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 storage / f32 compute (value); every mode listed",
            "data": "synthetic",
            "config": {"workload": f"periodic {nx}x{nx}x{nl}, smooth bathymetry, layered flow CFL 0.5, "
                                   "MUSCL+PPM+FCT, 2 tracers", "wet_cells": c.wet_cells, "steps": steps},
            "modes": modes, "clocks": best["clocks"]}
    print(json.dumps(line))
    return 0


def run_dd(args):
    """The 1000x1000x64 FP64 step cut into P index strips, every part on
    this GPU with the halo exchange after each step, against the whole mesh:
    redundant halo work, halo bytes per step, time per step of all parts."""
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    from fesom2_tracer_dwarf_b200.decomp import DomainDecomposition, partition_by_index
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    api = FESOMTracerAdvection()
    api.cleanup()
    c = layered_flow_case(api, args.nx, args.nl)
    N = api.mesh_dims()["nod2D"]
    api.allocate_tracers(2)
    api.set_values(1, c.T)
    api.set_values(2, c.S)
    for t in (1, 2):
        api.set_scheme(t, "MUSCL", "PPM", "FCT")
    api.set_velocity(c.uv, c.w)
    api.set_ab_refresh(True)
    api.advect_steps(max(args.warmup, 3), c.dt)
    steps = max(args.steps, 1)
    whole, clocks = timed(0, lambda: api.time_steps(steps, c.dt) / steps)
    parts = []
    for P in args.parts:
        dd = DomainDecomposition(api, partition_by_index(N, P), P)
        dd.allocate_tracers(2)
        for t in (1, 2):
            dd.set_scheme(t, "MUSCL", "PPM", "FCT")
        dd.set_velocity(c.uv, c.w)
        dd.set_values(1, c.T)
        dd.set_values(2, c.S)
        halo = sum(dd.transfer_nodes(i, p, False) for i in range(P) for p in range(P) if p != i)
        local = sum(dd.part_info(i)["nodes"] for i in range(P))
        dd.steps(3, c.dt)
        t0 = time.perf_counter()
        dd.steps(steps, c.dt, exchange=True)
        t1 = time.perf_counter()
        dd.steps(steps, c.dt, exchange=False)
        t2 = time.perf_counter()
        dd.destroy()
        parts.append({"parts": P, "local_over_owned_nodes": local / N,
                      "halo_bytes_per_step": halo * (args.nl - 1) * 2 * 8,
                      "ms_per_step_all_parts": (t1 - t0) * 1e3 / steps,
                      "ms_per_step_all_parts_no_exchange": (t2 - t1) * 1e3 / steps})
    api.cleanup()
    line = {"metric": "tracer cell-updates/s", "value": 2 * c.wet_cells / (whole / 1e3), "unit": "cell-updates/s",
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": whole, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args.nx, args.nl) + ", whole mesh (value) and P strips on one GPU "
                                                                     "(host-timed, exchange included)"},
            "parts": parts, "clocks": clocks}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "c3":
        return run_c3(args)
    if args.config == "c4":
        return run_c4(args)
    if args.config == "dd":
        return run_dd(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
