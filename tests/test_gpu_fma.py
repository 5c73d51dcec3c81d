"""Precision mode 4: the FP64 kernels compiled with FMA contraction.  Every
a*b+c the compiler fuses rounds once instead of twice, so results are no
longer bit-identical to the reference's arithmetic; they are held to the
FP64 tolerance of 1e-12 relative (to the field's largest magnitude) against
the CPU oracle on the analytic dwarf and the scheme matrix, and against the
bit-exact mode on the 1000x1000x64 workload, on both step paths; the
tracer content stays conserved to round-off."""
import numpy as np
import pytest

from test_gpu_parity import setup_pair, synth_case

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("path", ["fused", "five"])
def test_fma_analytic_dwarf_within_1e12(api, oracle, path):
    api.init_analytic(20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = api.analytic_fields()
    api.set_precision("fp64fma")
    api.set_step_path(path)
    sch = ("MUSCL", "PPM", "FCT", 1.0, 1.0)
    m = setup_pair(api, oracle, 20, 20, 10, True, False, None, [T], uv, w, [sch], False)
    To, TAB = T.copy(order="F"), T.copy(order="F")
    for step in range(10):
        api.advect_steps(1, 1000.0)
        m.step(To, TAB, uv, w, 1000.0, "MUSCL", "PPM", "FCT")
        g = api.get_tracer_values(1)
        assert rel(g, To) <= TOL, (step, rel(g, To))
    assert abs(api.get_statistics(1)["sum"] - 32490.0) < 1e-8


SCHEMES = [("MUSCL", "PPM", "FCT"), ("MFCT", "UPW1", "FCT"), ("UPW1", "PPM", "NONE"), ("MUSCL", "QR4C", "FCT"),
           ("MFCT", "CDIFF", "NONE")]


@pytest.mark.parametrize("hor,ver,lim", SCHEMES)
def test_fma_scheme_matrix_within_1e12(api, oracle, hor, ver, lim):
    nx, ny, nl = 23, 19, 11
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, True, 11)
    api.set_precision("fp64fma")
    sch = (hor, ver, lim, 1.0, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, True, True, K, [T], uv, w, [sch], True)
    To = T.copy(order="F")
    for step in range(3):
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F"), uv, w, dt, hor, ver, lim)
        assert rel(api.get_tracer_values(1), To) <= TOL


def test_fma_full_size_within_1e12_of_bit_exact(api):
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, 1000, 64, seed=0)
    out = {}
    for mode in ("fp64", "fp64fma"):
        api.set_precision(mode)
        api.allocate_tracers(2)
        api.set_values(1, c.T)
        api.set_values(2, c.S)
        for t in (1, 2):
            api.set_scheme(t, "MUSCL", "PPM", "FCT")
        api.set_velocity(c.uv, c.w)
        api.set_ab_refresh(True)
        v0 = api.volume_sum(1)[1]
        api.advect_steps(2, c.dt)
        out[mode] = (api.get_tracer_values(1), api.get_tracer_values(2), v0, api.volume_sum(1)[1])
    assert rel(out["fp64fma"][0], out["fp64"][0]) <= TOL
    assert rel(out["fp64fma"][1], out["fp64"][1]) <= TOL
    v0, v1 = out["fp64fma"][2], out["fp64fma"][3]
    assert abs(v1 - v0) <= 1e-12 * abs(v0)
    assert not np.array_equal(out["fp64fma"][0], out["fp64"][0])  # the FMA build really ran
