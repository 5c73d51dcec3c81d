"""Batched configuration: 48 tracers x 8 ensemble members on 8 analytic
meshes of uneven size (nx = ny in [100, 800], nl in [20, 80], closed-wall and
periodic mixed), seeded velocities per member, FP32, MUSCL+PPM+FCT.

Measured: the persistent one-launch step replayed from a CUDA graph (after
the autotuner has picked the tile), the same launch without the graph, and
the per-member separate launches of the plain engine.

    python -m fesom2_tracer_dwarf_b200.batch_study --members 8 --tracers 48
"""
from __future__ import annotations

import argparse
import json
import time

from .batch import TracerBatch
from .tracer import FESOMTracerAdvection
from .workloads import build_ensemble, ensemble_specs


def study(members=8, tracers=48, seed=0, steps=10, tune_steps=2, nx_range=(100, 800), nl_range=(20, 80)):
    specs = ensemble_specs(members, seed, nx_range, nl_range)
    api = FESOMTracerAdvection()
    batch = TracerBatch()
    t0 = time.perf_counter()
    dts = build_ensemble(batch, api, specs, tracers)
    build_s = time.perf_counter() - t0
    batch.configure(dts, "MUSCL", "PPM", "FCT")
    info = batch.info()
    log = batch.autotune(tune_steps)
    tile = batch.tile()
    batch.steps(2, graph=True)  # warm-up, graph capture
    ms_graph = batch.time_steps(steps, graph=True) / steps
    ms_plain = batch.time_steps(steps, graph=False) / steps
    ms_sep = batch.time_separate(steps) / steps
    ms_sep_graph = batch.time_separate(steps, graph=True) / steps
    cells = info["cell_tracers"]
    out = {
        "config": {"nx_range": list(nx_range), "nl_range": list(nl_range), "members": specs, "tracers_per_member": tracers, "scheme": "MUSCL+PPM+FCT", "precision": "fp32",
                   "cell_tracers": cells, "work_bytes": batch.info()["work_bytes"], "build_seconds": build_s},
        "tile": tile,
        "persistent_graph": {"ms_per_step": ms_graph, "cell_updates_per_s": cells / (ms_graph / 1e3)},
        "persistent_no_graph": {"ms_per_step": ms_plain, "cell_updates_per_s": cells / (ms_plain / 1e3)},
        "separate_launches": {"ms_per_step": ms_sep, "cell_updates_per_s": cells / (ms_sep / 1e3)},
        "separate_launches_graph": {"ms_per_step": ms_sep_graph, "cell_updates_per_s": cells / (ms_sep_graph / 1e3)},
        "speedup_vs_separate": ms_sep / ms_graph,
        "autotune_log": log.splitlines(),
    }
    batch.close()
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--members", type=int, default=8)
    p.add_argument("--tracers", type=int, default=48)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--nx-range", type=int, nargs=2, default=(100, 800))
    p.add_argument("--nl-range", type=int, nargs=2, default=(20, 80))
    a = p.parse_args()
    print(json.dumps(study(a.members, a.tracers, a.seed, a.steps, nx_range=tuple(a.nx_range),
                           nl_range=tuple(a.nl_range)), indent=1))


if __name__ == "__main__":
    main()
