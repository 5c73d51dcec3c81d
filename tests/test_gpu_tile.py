"""The fused patch kernel (one thread block per mesh patch with three halo
rings on chip) against the CPU oracle and against the five-kernel path.

FP64: bit-identical fields after every step, for every horizontal scheme,
PPM and UPW1 vertical, with and without FCT, valuesAB frozen (separate
array) or refreshed (aliased to the values), on periodic meshes with random
bathymetry, the reference's incomplete periodic rings, closed walls, the
irregular pi mesh, patch sizes down to one owned node, and one step of the
1000x1000x64 workload.  FP32: both paths as close to FP64 as FP32 allows."""
import numpy as np
import pytest

import pyoracle
from test_gpu_parity import assert_bitwise, setup_pair, synth_case

pytestmark = pytest.mark.gpu

SCHEMES = [(h, v, l) for l in ("FCT", "NONE") for h in ("MUSCL", "MFCT", "UPW1") for v in ("PPM", "UPW1")]


@pytest.fixture(autouse=True)
def fused_path(api):
    """These tests run the fused kernel (the engine's default is the
    five-kernel path)."""
    api.set_step_path("fused")
    yield


def _info(api):
    return api.step_info()


@pytest.mark.parametrize("hor,ver,lim", SCHEMES)
@pytest.mark.parametrize("refresh", [True, False], ids=["ab_alias", "ab_frozen"])
def test_fused_matches_oracle_bitwise(api, oracle, hor, ver, lim, refresh):
    nx, ny, nl = 37, 29, 13
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, True, 21)
    sch = (hor, ver, lim, 1.0, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, True, True, K, [T, S], uv, w, [sch, sch], refresh)
    info = _info(api)
    assert info["path"] == 0 and info["fused"] and info["patches"] >= 4
    To, So = T.copy(order="F"), S.copy(order="F")
    TAB, SAB = T.copy(order="F"), S.copy(order="F")
    for step in range(4):
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F") if refresh else TAB, uv, w, dt, hor, ver, lim)
        m.step(So, So.copy(order="F") if refresh else SAB, uv, w, dt, hor, ver, lim)
        assert_bitwise(api.get_tracer_values(1), To, f"T {hor}/{ver}/{lim} step {step + 1}")
        assert_bitwise(api.get_tracer_values(2), So, f"S {hor}/{ver}/{lim} step {step + 1}")


def test_fused_reference_rings_and_ph(api, oracle):
    """The analytic dwarf with the reference's incomplete periodic rings
    (FCT bounds over ring elements on the wrap rows) and ph = 0.75."""
    api.init_analytic(20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = api.analytic_fields()
    sch = ("MUSCL", "PPM", "FCT", 0.75, 1.0)
    m = setup_pair(api, oracle, 20, 20, 10, True, False, None, [T], uv, w, [sch], False)
    assert _info(api)["fused"]
    To, TAB = T.copy(order="F"), T.copy(order="F")
    for step in range(6):
        api.advect_steps(1, 1000.0)
        m.step(To, TAB, uv, w, 1000.0, "MUSCL", "PPM", "FCT", ph=0.75)
        assert_bitwise(api.get_tracer_values(1), To, f"step {step + 1}")


@pytest.mark.parametrize("owned", [1, 5, 40, 225])
def test_fused_closed_walls_and_patch_sizes_bitwise(api, oracle, owned):
    """Closed walls (boundary edges, coastline nodes); patches from a single
    owned node (every region mostly halo) to the default size."""
    nx, ny, nl = 26, 22, 15
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, False, 8)
    api.set_patch_size(owned)
    sch = ("MUSCL", "PPM", "FCT", 1.0, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, False, True, K, [T], uv, w, [sch], True)
    assert _info(api)["fused"]
    To = T.copy(order="F")
    for step in range(4):
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F"), uv, w, dt, "MUSCL", "PPM", "FCT")
        assert_bitwise(api.get_tracer_values(1), To, f"step {step + 1}")


def test_paths_agree_bitwise_at_full_size(api):
    """One step of the 1000x1000x64 benchmark workload (2 tracers): the
    fused and the five-kernel paths give the same bits."""
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, 1000, 64, seed=0)
    res = {}
    for p in ("five", "fused"):
        api.set_step_path(p)
        api.allocate_tracers(2)
        api.set_values(1, c.T)
        api.set_values(2, c.S)
        for t in (1, 2):
            api.set_scheme(t, "MUSCL", "PPM", "FCT")
        api.set_velocity(c.uv, c.w)
        api.set_ab_refresh(True)
        api.advect_steps(1, c.dt)
        assert _info(api)["fused"] == (p == "fused")
        res[p] = (api.get_tracer_values(1), api.get_tracer_values(2))
    assert_bitwise(res["fused"][0], res["five"][0], "T")
    assert_bitwise(res["fused"][1], res["five"][1], "S")


def test_fp32_paths_match_fp64_alike(api):
    """FP32 (FMA contraction allowed, so the two paths need not agree bit for
    bit): on the smooth layered-flow workload both paths stay as close to
    the bit-exact FP64 result as FP32 arithmetic allows, and the fused one no
    further from it than the five-kernel one."""
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, 120, 24, seed=4)
    out = {}
    for prec, p in (("fp64", "fused"), ("fp32", "five"), ("fp32", "fused")):
        api.set_precision(prec)
        api.set_step_path(p)
        api.allocate_tracers(1)
        api.set_values(1, c.T)
        api.set_scheme(1, "MUSCL", "PPM", "FCT")
        api.set_velocity(c.uv, c.w)
        api.set_ab_refresh(True)
        api.advect_steps(10, c.dt)
        assert _info(api)["fused"] == (p == "fused")
        out[(prec, p)] = api.get_tracer_values(1)[c.wet]
    ref = out[("fp64", "fused")]
    err = {p: np.linalg.norm(out[("fp32", p)] - ref) / np.linalg.norm(ref) for p in ("five", "fused")}
    assert err["five"] < 1e-5 and err["fused"] < 1e-5, err
    assert err["fused"] <= 2.0 * err["five"] + 1e-7, err


def test_fused_pi_mesh_bitwise(api, oracle, pi_mesh_dir):
    """The irregular pi mesh (valence 2-8, coastlines, 4-45 wet layers)."""
    from test_gpu_pi_mesh import pi_case
    uv, w, T, S, dt = pi_case(api, pi_mesh_dir, "reference")
    m = pyoracle.OracleMesh.from_files(oracle, pi_mesh_dir)
    for hor in ("MUSCL", "UPW1"):
        api.allocate_tracers(1)
        api.set_values(1, T)
        api.set_scheme(1, hor, "PPM", "FCT")
        api.set_velocity(uv, w)
        api.set_ab_refresh(True)
        info = _info(api)
        assert info["fused"] and info["patches"] >= 8
        To = T.copy(order="F")
        for step in range(3):
            api.advect_steps(1, dt)
            m.step(To, To.copy(order="F"), uv, w, dt, hor, "PPM", "FCT")
            assert_bitwise(api.get_tracer_values(1), To, f"{hor} step {step + 1}")
