"""Domain-decomposed step on the GPU: every part runs the ordinary step on
its local mesh (owned nodes + 3 halo rings) and the halos are exchanged
after each step; the owned values must equal a step of the whole mesh bit
for bit -- analytic meshes cut into strips, the pi mesh cut by the
reference's METIS partitions (dist_2, dist_8), FP64 and FP32, and two
processes exchanging their halos through torch.distributed."""
import json
import math
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
FESOM2 = dict(angle_scale=math.pi / 180.0, cyclic_length=2.0 * math.pi)


def _global_run(api, T, S, uv, w, dt, nsteps, sch):
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    for t in (1, 2):
        api.set_scheme(t, *sch)
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    api.advect_steps(nsteps, dt)
    return api.get_tracer_values(1), api.get_tracer_values(2)


def _dd_run(api, part, nparts, T, S, uv, w, dt, nsteps, sch, exchange=True):
    from fesom2_tracer_dwarf_b200.decomp import DomainDecomposition
    dd = DomainDecomposition(api, part, nparts)
    dd.allocate_tracers(2)
    for t in (1, 2):
        dd.set_scheme(t, *sch)
    dd.set_velocity(uv, w)
    dd.set_values(1, T)
    dd.set_values(2, S)
    dd.steps(nsteps, dt, refresh_ab=True, exchange=exchange)
    out = dd.get_values(1), dd.get_values(2)
    dd.destroy()
    return out


def _analytic(api, nx=40, ny=34, nl=12):
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, nx, nl, ny=ny, seed=3)
    return c.T, c.S, c.uv, c.w, c.dt


@pytest.mark.parametrize("nparts", [2, 3, 5])
@pytest.mark.parametrize("mode", ["fp64", "fp32"])
def test_analytic_strips_bitwise(api, nparts, mode):
    from fesom2_tracer_dwarf_b200.decomp import partition_by_index
    api.set_precision(mode)
    T, S, uv, w, dt = _analytic(api)
    sch = ("MUSCL", "PPM", "FCT")
    g1, g2 = _global_run(api, T, S, uv, w, dt, 6, sch)
    part = partition_by_index(api.mesh_dims()["nod2D"], nparts)
    d1, d2 = _dd_run(api, part, nparts, T, S, uv, w, dt, 6, sch)
    assert_bitwise(d1, g1, f"{mode} {nparts} strips T")
    assert_bitwise(d2, g2, f"{mode} {nparts} strips S")


@pytest.mark.parametrize("n", [2, 8])
@pytest.mark.parametrize("sch", [("MUSCL", "PPM", "FCT"), ("MFCT", "QR4C", "FCT"), ("UPW1", "UPW1", "NONE")])
def test_pi_mesh_metis_partitions_bitwise(api, pi_mesh_dir, n, sch):
    from fesom2_tracer_dwarf_b200.decomp import read_dist
    api.load_mesh_from_files(pi_mesh_dir, **FESOM2)
    uv, w = api.synth_velocity(seed=9, umax=0.5, mode2=0.5)
    T = api.synth_tracer(seed=10, kind=0)
    S = api.synth_tracer(seed=11, kind=1)
    dt = 300.0
    g1, g2 = _global_run(api, T, S, uv, w, dt, 5, sch)
    part, nparts = read_dist(api, pi_mesh_dir / f"dist_{n}")
    d1, d2 = _dd_run(api, part, nparts, T, S, uv, w, dt, 5, sch)
    assert_bitwise(d1, g1, f"pi dist_{n} {sch} T")
    assert_bitwise(d2, g2, f"pi dist_{n} {sch} S")


def test_frozen_values_ab_bitwise(api):
    """valuesAB frozen at its initial value (the analytic driver's mode): the
    halo rows of valuesAB are set once and stay right."""
    from fesom2_tracer_dwarf_b200.decomp import DomainDecomposition, partition_by_index
    T, S, uv, w, dt = _analytic(api)
    sch = ("MUSCL", "PPM", "FCT")
    api.allocate_tracers(1)
    api.set_values(1, T)
    api.set_scheme(1, *sch)
    api.set_velocity(uv, w)
    api.set_ab_refresh(False)
    api.advect_steps(4, dt)
    g1 = api.get_tracer_values(1)
    part = partition_by_index(api.mesh_dims()["nod2D"], 3)
    dd = DomainDecomposition(api, part, 3)
    dd.allocate_tracers(1)
    dd.set_scheme(1, *sch)
    dd.set_velocity(uv, w)
    dd.set_values(1, T)
    dd.steps(4, dt, refresh_ab=False, exchange=True)
    d1 = dd.get_values(1)
    dd.destroy()
    assert_bitwise(d1, g1, "frozen valuesAB")


def test_without_exchange_the_halo_goes_stale(api):
    """Control: skipping the exchange changes owned values within a few steps."""
    from fesom2_tracer_dwarf_b200.decomp import partition_by_index
    T, S, uv, w, dt = _analytic(api)
    sch = ("MUSCL", "PPM", "FCT")
    g1, _ = _global_run(api, T, S, uv, w, dt, 6, sch)
    part = partition_by_index(api.mesh_dims()["nod2D"], 3)
    d1, _ = _dd_run(api, part, 3, T, S, uv, w, dt, 6, sch, exchange=False)
    assert not np.array_equal(d1, g1)


WORKER = r'''
import json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, torch
from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
from fesom2_tracer_dwarf_b200.decomp import DistributedTracer, partition_by_index
from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
from fesom2_tracer_dwarf_b200.replicas import from_env
r = from_env("gloo", timeout_s=120)
api = FESOMTracerAdvection()
c = layered_flow_case(api, 40, 12, ny=34, seed=3)
part = partition_by_index(api.mesh_dims()["nod2D"], r.world)
dt = DistributedTracer(api, part, r.rank, r.world, "cuda:0")
dt.allocate_tracers(2)
for t in (1, 2):
    dt.dd.set_scheme(t, "MUSCL", "PPM", "FCT")
dt.dd.set_velocity(c.uv, c.w)
dt.dd.set_values(1, c.T)
dt.dd.set_values(2, c.S)
dt.steps(6, c.dt)
np.savez(sys.argv[2] + f"/rank{r.rank}.npz", T=dt.dd.get_values(1), S=dt.dd.get_values(2), part=part)
r.barrier()
print(json.dumps({"rank": r.rank}))
dt.dd.destroy()
r.close()
'''


def test_two_processes_exchange_halos_bitwise(api, tmp_path):
    """Two ranks (gloo for the exchange, both on this GPU; their kernels
    never wait on each other) each own one strip; merged, their owned values
    equal the whole-mesh run."""
    from test_replicas import _launch
    _launch(["-c", WORKER, str(ROOT), str(tmp_path)])
    T, S, uv, w, dt = _analytic(api)
    g1, g2 = _global_run(api, T, S, uv, w, dt, 6, ("MUSCL", "PPM", "FCT"))
    m1, m2 = np.zeros_like(g1), np.zeros_like(g2)
    for rank in (0, 1):
        z = np.load(tmp_path / f"rank{rank}.npz")
        own = z["part"] == rank
        m1[:, own] = z["T"][:, own]
        m2[:, own] = z["S"][:, own]
    assert_bitwise(m1, g1, "2 ranks T")
    assert_bitwise(m2, g2, "2 ranks S")
