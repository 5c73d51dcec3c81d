"""Error of a reduced-precision mode against the FP64 path: FP32,
BF16-storage and FP16-storage runs of the tracer step (16-bit stores rounded
to nearest or stochastically) on identical seeded inputs.

The FP64 path is bit-identical to the CPU oracle (tests/test_gpu_parity.py
checks it at every size up to 1000x1000x64), so it serves as the FP64
reference at sizes where a CPU run would take hours.  Reported per mode and
tracer: relative L2 and max-abs error of the final field over wet cells, the
drift of the conserved content Sum(T*areasvol*hnode_new) (compensated FP64
sum on the device), and device time per step.  bench.py --config c4 runs the
2000x2000x48 configuration through these functions.
"""
from __future__ import annotations

import numpy as np


def run_mode(api, c, mode, steps, hor="MUSCL", ver="PPM", lim="FCT"):
    """Advance both tracers of case c (mesh already in api) steps steps in one
    mode: 'fp64', 'fp32', 'bf16', 'fp16', or a 16-bit mode with '+sr'
    (stochastic rounding of the stores)."""
    T, S, uv, w, dt, wet = c.T, c.S, c.uv, c.w, c.dt, c.wet
    prec, _, sr = mode.partition("+")
    api.set_precision(prec)
    api.set_rounding("stochastic" if sr == "sr" else "nearest")
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    for t in (1, 2):
        api.set_scheme(t, hor, ver, lim)
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    v0 = [api.volume_sum(t)[1] for t in (1, 2)]
    ms = api.time_steps(steps, dt)
    v1 = [api.volume_sum(t)[1] for t in (1, 2)]
    out = [api.get_tracer_values(t) for t in (1, 2)]
    offsets = [api.storage_offset(t) for t in (1, 2)]
    api.set_rounding("nearest")
    return {"fields": out, "wet": wet, "v0": v0, "v1": v1, "ms_per_step": ms / steps, "cells": c.wet_cells,
            "dt": dt, "offsets": offsets}


def compare(ref, res):
    wet = ref["wet"]
    rows = []
    for t in range(2):
        a, b = res["fields"][t][wet], ref["fields"][t][wet]
        rows.append({
            "tracer": t + 1,
            "l2_rel": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
            "linf_abs": float(np.max(np.abs(a - b))),
            "content_drift_rel": float((res["v1"][t] - res["v0"][t]) / res["v0"][t]),
            "content_drift_rel_fp64": float((ref["v1"][t] - ref["v0"][t]) / ref["v0"][t]),
        })
    return rows
