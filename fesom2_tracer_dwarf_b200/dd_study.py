"""Cost of the domain-decomposed step on one GPU.

The 1000x1000x64 benchmark workload (``workloads.layered_flow_case``, FP64,
MUSCL+PPM+FCT, 2 tracers) cut into P index strips, every part on this GPU
with the halo exchange after each step, against the whole-mesh step:

* per part: owned / local nodes and wet cells (the redundant halo work),
  halo values sent per step;
* time per step of all parts (device-synchronised host time of ``steps``
  with the local exchange, and without it), and of the whole mesh.

On P GPUs each part would run alone; its share of the P-part time on one
GPU bounds its compute, and the halo bytes over NVLink bound its exchange.

    python -m fesom2_tracer_dwarf_b200.dd_study --parts 2 4 8 --steps 10
"""
from __future__ import annotations

import argparse
import json
import time

from . import FESOMTracerAdvection
from .decomp import DomainDecomposition, partition_by_index
from .workloads import layered_flow_case


def _whole(api, c, steps):
    api.allocate_tracers(2)
    api.set_values(1, c.T)
    api.set_values(2, c.S)
    for t in (1, 2):
        api.set_scheme(t, "MUSCL", "PPM", "FCT")
    api.set_velocity(c.uv, c.w)
    api.set_ab_refresh(True)
    api.advect_steps(2, c.dt)  # warm-up
    return api.time_steps(steps, c.dt) / steps


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=1000)
    ap.add_argument("--nl", type=int, default=64)
    ap.add_argument("--parts", type=int, nargs="+", default=[2, 4, 8])
    ap.add_argument("--steps", type=int, default=10)
    args = ap.parse_args(argv)
    api = FESOMTracerAdvection()
    c = layered_flow_case(api, args.nx, args.nl)
    N = api.mesh_dims()["nod2D"]
    out = {"workload": f"periodic {args.nx}x{args.nx}x{args.nl}, FP64, MUSCL+PPM+FCT, 2 tracers",
           "whole_ms_per_step": _whole(api, c, args.steps), "parts": []}
    for P in args.parts:
        part = partition_by_index(N, P)
        dd = DomainDecomposition(api, part, P)
        dd.allocate_tracers(2)
        for t in (1, 2):
            dd.set_scheme(t, "MUSCL", "PPM", "FCT")
        dd.set_velocity(c.uv, c.w)
        dd.set_values(1, c.T)
        dd.set_values(2, c.S)
        halo_nodes = sum(dd.transfer_nodes(i, p, False) for i in range(P) for p in range(P) if p != i)
        local_nodes = sum(dd.part_info(i)["nodes"] for i in range(P))
        dd.steps(2, c.dt)  # warm-up
        t0 = time.perf_counter()
        dd.steps(args.steps, c.dt, exchange=True)
        t1 = time.perf_counter()
        dd.steps(args.steps, c.dt, exchange=False)
        t2 = time.perf_counter()
        dd.destroy()
        out["parts"].append({
            "parts": P, "local_over_owned_nodes": local_nodes / N,
            "halo_values_per_step": halo_nodes * (args.nl - 1) * 2,
            "halo_bytes_per_step": halo_nodes * (args.nl - 1) * 2 * 8,
            "ms_per_step_all_parts": (t1 - t0) * 1e3 / args.steps,
            "ms_per_step_all_parts_no_exchange": (t2 - t1) * 1e3 / args.steps,
        })
        print(json.dumps(out["parts"][-1]), flush=True)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
