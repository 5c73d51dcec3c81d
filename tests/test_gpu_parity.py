"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64 kernels are built without FMA contraction and follow the reference's
operation order, so the bar is bit-identical fields after every step.
"""
import numpy as np
import pytest

import pyoracle

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def assert_bitwise(a, b, what=""):
    if not np.array_equal(bits(a), bits(b)):
        d = np.abs(a - b)
        i = np.unravel_index(np.argmax(d), d.shape)
        raise AssertionError(f"{what}: {np.count_nonzero(bits(a) != bits(b))} cells differ, max |diff| "
                             f"{d[i]:.3e} at {i}: gpu {a[i]!r} oracle {b[i]!r}")


def setup_pair(api, oracle, nx, ny, nl, periodic, full, K, tracers, uv, w, schemes, refresh, ab=None):
    api.init_analytic(nx, ny, nl, periodic=periodic, full_rings=full, node_K=K)
    api.allocate_tracers(len(tracers))
    for i, T in enumerate(tracers):
        api.set_values(i + 1, T, None if ab is None else ab[i])
        api.set_scheme(i + 1, *schemes[i])
    api.set_velocity(uv, w)
    api.set_ab_refresh(refresh)
    return pyoracle.OracleMesh(oracle, nx, ny, nl, periodic=periodic, full_rings=full, node_K=K)


def test_c1_analytic_muscl_ppm_fct_bitwise(api, oracle):
    """The analytic dwarf (20x20x10 periodic, reference rings, valuesAB frozen
    as in src/fesom_analytic.F90) with MUSCL/PPM/FCT: T and S bit-identical to
    the oracle after each of 10 steps; Sum T conserved."""
    api.init_analytic(20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = api.analytic_fields()
    sch = ("MUSCL", "PPM", "FCT", 1.0, 1.0)
    m = setup_pair(api, oracle, 20, 20, 10, True, False, None, [T, S], uv, w, [sch, sch], False)
    To, So = T.copy(order="F"), S.copy(order="F")
    TAB, SAB = T.copy(order="F"), S.copy(order="F")
    for step in range(10):
        api.advect_steps(1, 1000.0)
        m.step(To, TAB, uv, w, 1000.0, *sch[:3])
        m.step(So, SAB, uv, w, 1000.0, *sch[:3])
        assert_bitwise(api.get_tracer_values(1), To, f"T step {step + 1}")
        assert_bitwise(api.get_tracer_values(2), So, f"S step {step + 1}")
        st = api.get_statistics(1)
        assert st["nan"] == 0 and abs(st["sum"] - 32490.0) < 1e-9


def test_c1_upw1_golden(api, oracle):
    """UPW1/UPW1/NONE through the reference's own call sequence reproduces the
    README's printed numbers (README.md:51-52) on the GPU."""
    import json
    from pathlib import Path
    from test_oracle import fmt_e
    gold = json.loads((Path(__file__).parent / "golden" / "readme_upw1.json").read_text())
    api.init_analytic(20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = api.analytic_fields()
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    api.set_velocity(uv, w)
    for rec in gold["steps"]:
        assert api.advect_step(1000.0) == 0
        st = api.get_statistics(1)
        assert fmt_e(st["min"], 14, 6) == rec["min"].rjust(14)
        assert fmt_e(st["max"], 14, 6) == rec["max"].rjust(14)
        assert fmt_e(st["sum"], 18, 10) == rec["sum"].rjust(18)


def synth_case(api, nx, ny, nl, periodic, seed):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, int(periodic)), nl, seed)
    api.init_analytic(nx, ny, nl, periodic=periodic, full_rings=True, node_K=K)
    uv, w = api.synth_velocity(seed=seed + 1, umax=1.0, mode2=0.5)
    T = api.synth_tracer(seed=seed + 2, kind=0)
    S = api.synth_tracer(seed=seed + 3, kind=1)
    dx = 1.0e5 / (nx - 1)
    return K, uv, w, T, S, 0.5 * dx


SCHEMES = [(h, v, l) for l in ("FCT", "NONE") for h in ("MUSCL", "MFCT", "UPW1") for v in ("PPM", "QR4C", "CDIFF", "UPW1")]


@pytest.mark.parametrize("hor,ver,lim", SCHEMES)
def test_scheme_matrix_bitwise(api, oracle, hor, ver, lim):
    """Every horizontal x vertical x limiter combination on a periodic mesh
    with random bathymetry and a layered flow, valuesAB refreshed each step."""
    nx, ny, nl = 23, 19, 11
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, True, 11)
    sch = (hor, ver, lim, 1.0, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, True, True, K, [T], uv, w, [sch], True)
    To = T.copy(order="F")
    for step in range(3):
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F"), uv, w, dt, hor, ver, lim)
        assert_bitwise(api.get_tracer_values(1), To, f"{hor}/{ver}/{lim} step {step + 1}")


@pytest.mark.parametrize("lim", ["FCT", "NONE"])
def test_velocity_changes_between_steps_bitwise(api, oracle, lim):
    """The edge volume fluxes the engine keeps from step to step follow every
    new velocity: two steps with one flow, two with another, one with the
    first again, then one with zero velocity, each bit-identical to the
    oracle stepping with the velocity of that step."""
    nx, ny, nl = 21, 18, 9
    K, uv1, w1, T, S, dt = synth_case(api, nx, ny, nl, True, 31)
    uv2, w2 = api.synth_velocity(seed=77, umax=0.8, mode2=0.3)
    zuv, zw = np.zeros_like(uv1), np.zeros_like(w1)
    sch = ("MUSCL", "PPM", lim, 1.0, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, True, True, K, [T], uv1, w1, [sch], True)
    To = T.copy(order="F")
    plan = [(uv1, w1), (uv1, w1), (uv2, w2), (uv2, w2), (uv1, w1), (zuv, zw)]
    for step, (uv, w) in enumerate(plan):
        if step > 0 and uv is not plan[step - 1][0]:
            api.set_velocity(uv, w)
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F"), uv, w, dt, "MUSCL", "PPM", lim)
        assert_bitwise(api.get_tracer_values(1), To, f"{lim} step {step + 1}")


@pytest.mark.parametrize("ph", [1.0, 0.75, 0.0])
def test_closed_wall_bathymetry_bitwise(api, oracle, ph):
    """Closed-wall analytic mesh (boundary edges, nboundary_lay = 0 on the
    walls) with bathymetry; MUSCL with partial fourth-order weight ph."""
    nx, ny, nl = 17, 21, 9
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, False, 21)
    sch = ("MUSCL", "PPM", "FCT", ph, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, False, True, K, [T, S], uv, w, [sch, sch], True)
    To, So = T.copy(order="F"), S.copy(order="F")
    for step in range(4):
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F"), uv, w, dt, "MUSCL", "PPM", "FCT", ph)
        m.step(So, So.copy(order="F"), uv, w, dt, "MUSCL", "PPM", "FCT", ph)
        assert_bitwise(api.get_tracer_values(1), To, f"T step {step + 1}")
        assert_bitwise(api.get_tracer_values(2), So, f"S step {step + 1}")


def test_deep_columns_bitwise(api, oracle):
    """80 levels (the deepest batched configuration): columns and edges longer
    than a quarter of a block's cell capacity, closed walls and bathymetry."""
    nx, ny, nl = 15, 13, 80
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, False, 33)
    sch = ("MUSCL", "PPM", "FCT", 1.0, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, False, True, K, [T], uv, w, [sch], True)
    To = T.copy(order="F")
    for step in range(2):
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F"), uv, w, dt, "MUSCL", "PPM", "FCT")
        assert_bitwise(api.get_tracer_values(1), To, f"step {step + 1}")


def test_edge_cases_minimum_sizes(api, oracle):
    """Smallest meshes the generator allows (periodic 4x4, closed 2x2) with the
    thinnest columns (nl = 3: two layers, where PPM's end formulas overlap)."""
    for (nx, ny, periodic) in ((4, 4, True), (2, 2, False), (5, 3, False)):
        nl = 3
        api.init_analytic(nx, ny, nl, periodic=periodic, full_rings=True)
        uv, w = api.synth_velocity(seed=3, umax=0.5, mode2=0.5)
        T = api.synth_tracer(seed=4, kind=0)
        sch = ("MUSCL", "PPM", "FCT", 1.0, 1.0)
        m = setup_pair(api, oracle, nx, ny, nl, periodic, True, None, [T], uv, w, [sch], True)
        To = T.copy(order="F")
        for _ in range(3):
            api.advect_steps(1, 3000.0)
            m.step(To, To.copy(order="F"), uv, w, 3000.0, "MUSCL", "PPM", "FCT")
        assert_bitwise(api.get_tracer_values(1), To, f"{nx}x{ny}")


def test_ragged_columns_and_zero_velocity(api, oracle):
    """Ragged bathymetry with K at both ends of [3, nl] and zero velocity:
    bit-identical to the oracle, and the tracer moves by round-off only."""
    nx, ny, nl = 13, 11, 7
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, 1), nl, 31)
    idx = np.arange(K.size)
    K = np.where(idx % 5 == 0, 3, np.where(idx % 7 == 0, nl, K)).astype(np.int32)
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    T = api.synth_tracer(seed=9, kind=0)
    d = api.mesh_dims()
    uv = np.zeros((2, nl - 1, d["elem2D"]), order="F")
    w = np.zeros((nl, d["nod2D"]), order="F")
    sch = ("MUSCL", "PPM", "FCT", 1.0, 1.0)
    m = setup_pair(api, oracle, nx, ny, nl, True, True, K, [T], uv, w, [sch], True)
    To = T.copy(order="F")
    for _ in range(2):
        api.advect_steps(1, 100.0)
        m.step(To, To.copy(order="F"), uv, w, 100.0, "MUSCL", "PPM", "FCT")
    G = api.get_tracer_values(1)
    assert_bitwise(G, To, "zero velocity")
    assert np.max(np.abs(G - T)) <= 1e-13 * np.max(np.abs(T))


def test_determinism_repeat(api):
    """No float atomics: two runs from the same state agree bit for bit."""
    nx, ny, nl = 64, 48, 20
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, True, 41)
    outs = []
    for _ in range(2):
        api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)
        api.allocate_tracers(1)
        api.set_values(1, T)
        api.set_scheme(1, "MUSCL", "PPM", "FCT")
        api.set_velocity(uv, w)
        api.set_ab_refresh(True)
        api.advect_steps(5, dt)
        outs.append(api.get_tracer_values(1))
    assert_bitwise(outs[0], outs[1], "repeat")


def volume_sum(api, T):
    d = api.mesh_dims()
    nl = d["nl"]
    asv = api.mesh_array("areasvol").reshape(nl, -1, order="F")[: nl - 1]
    h = api.mesh_array("hnode_new").reshape(nl - 1, -1, order="F")
    nlev = api.mesh_array("nlevels_nod2D")
    wet = np.arange(nl - 1)[:, None] < (nlev[None, :] - 1)
    return float(np.sum(np.where(wet, T * asv * h, 0.0))), wet


def test_c2_size_one_step_bitwise_and_conservation(api):
    """The benchmark's 1000x1000x64 periodic case (smooth bathymetry,
    divergence-free layered flow, two tracers): one GPU step against the
    OpenMP oracle bit for bit, then 5 more steps conserving Sum(T*vol) to
    FP64 round-off."""
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    oracle = pyoracle.Oracle(openmp=True)
    nx = ny = 1000
    nl = 64
    c = layered_flow_case(api, nx, nl, seed=0)
    api.allocate_tracers(2)
    api.set_values(1, c.T)
    api.set_values(2, c.S)
    for t in (1, 2):
        api.set_scheme(t, "MUSCL", "PPM", "FCT")
    api.set_velocity(c.uv, c.w)
    api.set_ab_refresh(True)
    s0, wet = volume_sum(api, c.T)
    api.advect_steps(1, c.dt)
    m = pyoracle.OracleMesh(oracle, nx, ny, nl, periodic=True, full_rings=True, node_K=c.K, left_oriented=True)
    for tid, F in ((1, c.T), (2, c.S)):
        Fo = F.copy(order="F")
        m.step(Fo, Fo.copy(order="F"), c.uv, c.w, c.dt, "MUSCL", "PPM", "FCT")
        assert_bitwise(api.get_tracer_values(tid), Fo, f"C2 tracer {tid} step 1")
    del m
    api.advect_steps(5, c.dt)
    G = api.get_tracer_values(1)
    assert np.all(np.isfinite(G[wet]))
    s1, _ = volume_sum(api, G)
    assert abs(s1 - s0) <= 1e-12 * abs(s0)


def test_reciprocal_division_is_correctly_rounded(lib):
    """div_rcp (Markstein's correction from a once-per-cell reciprocal)
    returns the bits of the IEEE quotient on 2^28 random operand pairs
    spanning general, /6, area-like and thickness-like divisors."""
    import ctypes
    bad = ctypes.c_longlong(-1)
    ex = np.zeros(4)
    assert lib.tracer_selftest_division(1 << 28, 12345, ctypes.byref(bad), ex.ctypes.data_as(ctypes.c_void_p)) == 0
    assert bad.value == 0, f"a={ex[0]!r} b={ex[1]!r} got={ex[2]!r} expected={ex[3]!r}"
