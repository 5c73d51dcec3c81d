"""The CPU oracle against the reference's published numbers and the
invariants that pin the schemes no reference test covers."""
import json
from pathlib import Path

import numpy as np
import pytest

import pyoracle

GOLDEN = Path(__file__).resolve().parent / "golden"


def fmt_e(x, w, d):
    """Fortran Ew.d rendering, as the analytic driver prints (src/fesom_analytic.F90:446-447)."""
    s = f"{x:.{d - 1}E}"          # d significant digits
    mant, exp = s.split("E")
    digits = mant.replace("-", "").replace(".", "")
    e = int(exp) + 1
    sign = "-" if x < 0 else ""
    return f"{sign}0.{digits}E{e:+03d}".rjust(w)


def test_upw1_golden_readme(oracle):
    """UPW1/UPW1/NONE on the 20x20x10 periodic mesh reproduces README.md:51-52."""
    gold = json.loads((GOLDEN / "readme_upw1.json").read_text())
    m = pyoracle.OracleMesh(oracle, 20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = m.analytic_fields()
    TAB = T.copy(order="F")
    for rec in gold["steps"]:
        m.step(T, TAB, uv, w, 1000.0, "UPW1", "UPW1", "NONE")
        mn, mx, sm, nan = m.stats(T)
        assert fmt_e(mn, 14, 6) == rec["min"].rjust(14)
        assert fmt_e(mx, 14, 6) == rec["max"].rjust(14)
        assert fmt_e(sm, 18, 10) == rec["sum"].rjust(18)
        assert nan == 0


def test_upw1_golden_all_steps_sum_conserved(oracle):
    """Sum conserved at 0.3249000000E+05 with 0 NaN at every step (CLAUDE.md:13)."""
    m = pyoracle.OracleMesh(oracle, 20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = m.analytic_fields()
    TAB = T.copy(order="F")
    for _ in range(10):
        m.step(T, TAB, uv, w, 1000.0, "UPW1", "UPW1", "NONE")
        mn, mx, sm, nan = m.stats(T)
        assert fmt_e(sm, 18, 10).strip() == "0.3249000000E+05"
        assert nan == 0


def test_fixture_regression(oracle):
    """Committed MUSCL/PPM/FCT fixture of the 20x20x10 analytic run (made by
    tests/golden/make_fixtures.py) still reproduces bit for bit."""
    data = np.load(GOLDEN / "c1_muscl_ppm_fct.npz")
    m = pyoracle.OracleMesh(oracle, 20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = m.analytic_fields()
    TAB = T.copy(order="F")
    for step in range(int(data["nsteps"])):
        m.step(T, TAB, uv, w, 1000.0, "MUSCL", "PPM", "FCT")
    assert np.array_equal(T, data["T_final"])


def _volume_sum(m, T):
    asv = m.array("areasvol").reshape(m.nl, -1, order="F")[: m.nl - 1, :]
    h = m.array("hnode_new").reshape(m.nl - 1, -1, order="F")
    nlev = m.array("nlevels_nod2D")
    wet = np.arange(m.nl - 1)[:, None] < (nlev[None, :] - 1)
    return float(np.sum(np.where(wet, T * asv * h, 0.0)))


@pytest.mark.parametrize("hor,ver,periodic", [("MUSCL", "PPM", True), ("MFCT", "QR4C", True), ("UPW1", "CDIFF", True),
                                              ("MUSCL", "UPW1", True), ("MUSCL", "PPM", False), ("MFCT", "CDIFF", False)])
def test_fct_conserves_and_bounds(oracle, hor, ver, periodic):
    """Sum(T*vol) conserved to round-off and the FCT solution stays inside
    the local min/max of the old and low-order fields (lib/oce_adv_tra_fct.F90),
    on a periodic mesh and on one closed by walls, both with bathymetry."""
    import ctypes
    lib = pytest.importorskip("fesom2_tracer_dwarf_b200._lib").load()
    nx, ny, nl = 18, 14, 9
    N = lib.tracer_analytic_nodes(nx, ny, int(periodic))
    K = np.zeros(N, dtype=np.int32)
    lib.tracer_synth_bathymetry(N, nl, 3, K.ctypes.data_as(ctypes.c_void_p))
    m = pyoracle.OracleMesh(oracle, nx, ny, nl, periodic=periodic, full_rings=True, node_K=K)
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    api = FESOMTracerAdvection()
    api.cleanup()
    api.init_analytic(nx, ny, nl, periodic=periodic, full_rings=True, node_K=K)
    uv, w = api.synth_velocity(seed=1, umax=1.0, mode2=0.4)
    T = np.asfortranarray(api.synth_tracer(seed=2, kind=0))
    api.cleanup()
    dt = 0.5 * (1.0e5 / (nx - 1)) / 1.0
    s0 = _volume_sum(m, T)
    for _ in range(4):
        Told = T.copy(order="F")
        dh, dv, lo = m.step(T, Told.copy(order="F"), uv, w, dt, hor, ver, "FCT", want_terms=True)
        # every new value lies within the cluster bounds of (Told, LO) over the ring
        nlev = m.array("nlevels_nod2D")
        wet = np.arange(nl - 1)[:, None] < (nlev[None, :] - 1)
        big = np.where(wet, np.maximum(Told, lo), -np.inf)
        small = np.where(wet, np.minimum(Told, lo), np.inf)
        en = m.array("elem2D_nodes").reshape(3, -1, order="F") - 1
        lvl = m.array("nlevels")
        emax = np.full((nl - 1, m.elem2D), -np.inf)
        emin = np.full((nl - 1, m.elem2D), np.inf)
        for q in range(3):
            emax = np.maximum(emax, big[:, en[q]])
            emin = np.minimum(emin, small[:, en[q]])
        ewet = np.arange(nl - 1)[:, None] < (lvl[None, :] - 1)
        emax = np.where(ewet, emax, -np.inf)
        emin = np.where(ewet, emin, np.inf)
        nmax = np.full((nl - 1, m.nod2D), -np.inf)
        nmin = np.full((nl - 1, m.nod2D), np.inf)
        for q in range(3):
            np.maximum.at(nmax.T, en[q], emax.T)
            np.minimum.at(nmin.T, en[q], emin.T)
        up = np.vstack([nmax[:1], nmax[:-1]])
        dn = np.vstack([nmax[1:], nmax[-1:]])
        hi = np.maximum(np.maximum(up, nmax), dn)
        up = np.vstack([nmin[:1], nmin[:-1]])
        dn = np.vstack([nmin[1:], nmin[-1:]])
        lo_b = np.minimum(np.minimum(up, nmin), dn)
        tol = 1e-9 * np.max(np.abs(T[wet]))
        assert np.all(T[wet] <= hi[wet] + tol)
        assert np.all(T[wet] >= lo_b[wet] - tol)
    s1 = _volume_sum(m, T)
    assert abs(s1 - s0) <= 1e-12 * abs(s0)


def test_constant_field_stays_constant(oracle):
    """With a discretely non-divergent flow a constant tracer stays constant."""
    import ctypes
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    nx, ny, nl = 16, 16, 8
    api = FESOMTracerAdvection()
    api.cleanup()
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True)
    uv, w = api.synth_velocity(seed=5, umax=1.0, mode2=0.0)
    api.cleanup()
    m = pyoracle.OracleMesh(oracle, nx, ny, nl, periodic=True, full_rings=True)
    T = np.full((nl - 1, m.nod2D), 7.25, order="F")
    for _ in range(3):
        m.step(T, T.copy(order="F"), uv, w, 40.0, "MUSCL", "PPM", "FCT")
    assert np.max(np.abs(T - 7.25)) < 1e-12


def test_upw1_as_high_order_gives_zero_antidiffusion(oracle):
    """With UPW1 as the high-order scheme and T_AB = T, the antidiffusive flux
    is exactly 0, so FCT returns the low-order solution (to the round-off of
    T + (LO*h - T*h)/h)."""
    m = pyoracle.OracleMesh(oracle, 12, 12, 6, periodic=True, full_rings=True)
    T, S, uv, w = m.analytic_fields()
    T1 = T.copy(order="F")
    dh, dv, lo = m.step(T1, T.copy(order="F"), uv, w, 1000.0, "UPW1", "UPW1", "FCT", want_terms=True)
    assert np.max(np.abs(T1 - lo)) <= 1e-13 * np.max(np.abs(lo))


def test_left_oriented_mesh_transports_with_the_flow(oracle):
    """On the reference analytic mesh the horizontal and vertical edges carry
    edge_tri(1) on their right, so UPW1 moves a blob against the flow across
    them; with the left-oriented option a blob moves with a uniform flow."""
    nx, nl = 41, 4
    m = pyoracle.OracleMesh(oracle, nx, nx, nl, periodic=True, full_rings=True, left_oriented=True)
    T, S, uv, w = m.analytic_fields()
    x, y = m.array("coord").reshape(2, -1, order="F") * 6367500.0
    bump = np.exp(-((x - 3e4) ** 2 + (y - 5e4) ** 2) / 8e3 ** 2)
    dt = 0.5 * 1e5 / (nx - 1)
    for (u, v) in ((1.0, 0.0), (0.0, 1.0), (0.7, 0.7)):
        Tb = np.asfortranarray(np.tile(bump, (nl - 1, 1)))
        uvv = uv.copy(order="F")
        uvv[0], uvv[1] = u, v
        for _ in range(20):
            m.step(Tb, Tb.copy(order="F"), uvv, w, dt, "UPW1", "UPW1", "NONE")
        cx, cy = (Tb[0] * x).sum() / Tb[0].sum(), (Tb[0] * y).sum() / Tb[0].sum()
        assert abs(cx - (3e4 + 20 * dt * u)) < 300 and abs(cy - (5e4 + 20 * dt * v)) < 300
        assert Tb.min() >= 0.0


def test_layered_flow_case_preserves_constants_and_stays_bounded(oracle):
    """The benchmark's seeded case (smooth bathymetry, depth-independent
    curl(psi) plus zero-column-mean modes, w from the discrete continuity) on
    the left-oriented mesh: a constant tracer stays constant under
    MUSCL/PPM/FCT, and the blob tracer keeps its content exactly and stays
    within its initial range over a long run."""
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    nx, nl = 33, 12
    api = FESOMTracerAdvection()
    api.cleanup()
    c = layered_flow_case(api, nx, nl, seed=4)
    asv = api.mesh_array("areasvol").reshape(nl, -1, order="F")[: nl - 1]
    hn = api.mesh_array("hnode_new").reshape(nl - 1, -1, order="F")
    api.cleanup()
    assert np.abs(c.w).max() > 0.0 and np.abs(c.w[0]).max() == 0.0
    m = pyoracle.OracleMesh(oracle, nx, nx, nl, periodic=True, full_rings=True, node_K=c.K, left_oriented=True)
    C = np.full((nl - 1, m.nod2D), 3.5, order="F")
    for _ in range(5):
        m.step(C, C.copy(order="F"), c.uv, c.w, c.dt, "MUSCL", "PPM", "FCT")
    assert np.max(np.abs(C[c.wet] - 3.5)) < 1e-12
    T = c.T.copy(order="F")
    lo, hi = T[c.wet].min(), T[c.wet].max()
    c0 = (T * asv * hn)[c.wet].sum()
    for _ in range(60):
        m.step(T, T.copy(order="F"), c.uv, c.w, c.dt, "MUSCL", "PPM", "FCT")
    assert abs((T * asv * hn)[c.wet].sum() - c0) <= 1e-13 * abs(c0)
    assert T[c.wet].min() >= lo - 1e-10 and T[c.wet].max() <= hi + 1e-10


def test_smooth_bathymetry_marginal_is_uniform():
    """Per-node bottom levels of the smooth bathymetry cover [3, nl] evenly."""
    from fesom2_tracer_dwarf_b200 import synth_bathymetry_smooth
    K = synth_bathymetry_smooth(200, 200, 40, periodic=True, corr_cells=8.0, seed=0)
    assert K.min() == 3 and K.max() == 40
    counts = np.bincount(K)[3:]
    assert counts.min() > 0.5 * counts.mean() and counts.max() < 1.6 * counts.mean()
    # smooth: neighbours along x differ far less than independent draws
    # (mean |difference| (nl - 3) / 3 ~ 12 levels)
    G = K.reshape(199, 199)
    assert np.abs(np.diff(G, axis=1)).mean() < 5.0


def test_ensemble_specs_are_seeded_and_in_range():
    from fesom2_tracer_dwarf_b200.workloads import ensemble_specs
    a, b = ensemble_specs(8, seed=0), ensemble_specs(8, seed=0)
    assert a == b and len(a) == 8
    assert all(100 <= s["nx"] <= 800 and 20 <= s["nl"] <= 80 for s in a)
    assert {s["periodic"] for s in a} == {True, False}


def test_mlp_oracle_gradients_match_finite_differences():
    """Unquantised CPU MLP: analytic gradients of sum dy*y against central
    differences in FP64."""
    import mlp_oracle as mo
    rng = np.random.default_rng(3)
    X = rng.standard_normal((40, mo.F))
    dy = rng.standard_normal(40)
    p = mo.init_params(1).astype(np.float64)
    g = mo.grads(X, dy, p, quantize=False)
    idx = rng.choice(mo.NPARAMS, 60, replace=False).tolist() + [mo.OFF["b3"], mo.OFF["b1"], mo.OFF["w3"]]
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (dy @ mo.forward(X, p + e, False)[0] - dy @ mo.forward(X, p - e, False)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


@pytest.mark.parametrize("periodic", [True, False])
def test_openmp_oracle_equals_serial(oracle, periodic):
    """The OpenMP build of the oracle (the checker of the full-size GPU parity
    test and the CPU baseline) gives the serial build's bits: every node sums
    its edges in ascending edge id on both, whatever the thread count."""
    omp = pyoracle.Oracle(openmp=True)
    omp.set_threads(4)
    results = []
    for o in (oracle, omp):
        m, K, uv, w, T, S, dt, wet = pyoracle.layered_flow_case(o, 90, 24, seed=3, periodic=periodic)
        for hor, ver in (("MUSCL", "PPM"), ("MFCT", "QR4C")):
            X = np.asfortranarray(T.copy())
            for _ in range(3):
                m.step(X, X.copy(order="F"), uv, w, dt, hor, ver, "FCT")
            results.append(X)
    half = len(results) // 2
    for a, b in zip(results[:half], results[half:]):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert not np.array_equal(results[0], T)


@pytest.mark.parametrize("hor,ver", [("MUSCL", "PPM"), ("MFCT", "QR4C"), ("UPW1", "CDIFF"), ("MUSCL", "UPW1")])
def test_unlimited_schemes_conserve(oracle, hor, ver):
    """Without the limiter every scheme still conserves Sum(T*vol): the edge
    fluxes leave one node and enter the other, and the vertical fluxes vanish
    at the surface (w = 0 there) and the bottom."""
    m, K, uv, w, T, S, dt, wet = pyoracle.layered_flow_case(oracle, 40, 12, seed=5, periodic=True)
    X = np.asfortranarray(T.copy())
    s0 = _volume_sum(m, X)
    for _ in range(4):
        m.step(X, X.copy(order="F"), uv, w, dt, hor, ver, "NONE")
    assert np.all(np.isfinite(X))
    assert not np.array_equal(X, T)
    assert abs(_volume_sum(m, X) - s0) <= 1e-12 * abs(s0)
