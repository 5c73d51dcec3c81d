"""FP32 and 16-bit-storage modes against the bit-exact FP64 path (the
error budget of each mode is stated in the assertions)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_volume_sum_matches_host(api):
    from test_gpu_parity import synth_case, volume_sum
    K, uv, w, T, S, dt = synth_case(api, 40, 30, 14, True, 5)
    api.allocate_tracers(1)
    api.set_values(1, T)
    api.set_velocity(uv, w)
    st, content = api.volume_sum(1)
    host, wet = volume_sum(api, T)
    assert abs(content - host) <= 1e-13 * abs(host)
    assert abs(st - float(np.sum(T[wet]))) <= 1e-13 * abs(st)


@pytest.mark.parametrize("fmt", [0, 1], ids=["bf16", "fp16"])
def test_stochastic_rounding_is_unbiased_between_neighbours(lib, fmt):
    """2^20 inputs x 64 draws: every stochastically rounded store is one of
    the input's two storage neighbours, and the number rounded up matches
    sum(remainder / spacing) within 5 standard deviations."""
    import ctypes
    outside, z = ctypes.c_longlong(-1), ctypes.c_double(1e9)
    assert lib.tracer_selftest_sround(fmt, 1 << 20, 64, 1234, ctypes.byref(outside), ctypes.byref(z)) == 0
    assert outside.value == 0
    assert abs(z.value) < 5.0, z.value


@pytest.mark.parametrize("mode", ["bf16", "fp16"])
def test_16bit_storage_offset_roundtrip(api, mode):
    """16-bit storage keeps T - off on wet cells (off = FP32 wet-cell mean of
    the latest upload): a set/get round trip is within half a storage ulp of
    the anomaly, and dry cells come back exactly."""
    from test_gpu_parity import synth_case
    K, uv, w, T, S, dt = synth_case(api, 30, 26, 12, True, 9)
    api.set_precision(mode)
    api.allocate_tracers(1)
    S = np.asfortranarray(S)
    api.set_values(1, S)
    off = api.storage_offset(1)
    nlev = api.mesh_array("nlevels_nod2D")
    wet = np.arange(11)[:, None] < (nlev[None, :] - 1)
    assert abs(off - float(np.float32(S[wet].mean()))) <= 1e-6 * abs(off)
    G = api.get_tracer_values(1)
    a = np.abs(S[wet] - off)
    half_ulp = np.ldexp(1.0, np.frexp(np.maximum(a, 1e-30))[1] - (9 if mode == "bf16" else 12))
    # + FP32 rounding on the way, + FP16's subnormal spacing near zero
    assert np.all(np.abs(G[wet] - S[wet]) <= half_ulp + 1e-6 * (a + abs(off)) + 2.0 ** -24)
    assert np.array_equal(G[~wet], S[~wet])


@pytest.mark.parametrize("mode", ["bf16", "fp16"])
def test_stochastic_rounding_is_reproducible(api, mode):
    """The rounding stream is a function of (tracer, step, cell): two runs
    from the same inputs agree bit for bit, and differ from round-to-nearest
    by storage-level noise (relative L2 below 2e-2 after 5 steps)."""
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, 40, 16, seed=3)
    T, uv, w, dt = c.T, c.uv, c.w, c.dt
    api.set_precision(mode)
    runs = []
    for rounding in ("stochastic", "stochastic", "nearest"):
        api.set_rounding(rounding)
        api.allocate_tracers(1)
        api.set_values(1, T)
        api.set_scheme(1, "MUSCL", "PPM", "FCT")
        api.set_velocity(uv, w)
        api.set_ab_refresh(True)
        api.advect_steps(5, dt)
        runs.append(api.get_tracer_values(1))
    api.set_rounding("nearest")
    assert np.array_equal(runs[0], runs[1])
    assert not np.array_equal(runs[0], runs[2])
    d = np.linalg.norm(runs[0][c.wet] - runs[2][c.wet]) / np.linalg.norm(runs[2][c.wet])
    assert d < 2e-2, d


@pytest.fixture(scope="module")
def study():
    """Every mode against the FP64 path on the 160x160x24 case, 40 steps."""
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    from fesom2_tracer_dwarf_b200.precision import compare, run_mode
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    api = FESOMTracerAdvection()
    api.cleanup()
    c = layered_flow_case(api, 160, 24)
    ref = run_mode(api, c, "fp64", 40)
    out = {"modes": {}}
    for m in ("fp32", "bf16", "bf16+sr", "fp16", "fp16+sr"):
        out["modes"][m] = {"errors": compare(ref, run_mode(api, c, m, 40))}
    api.cleanup()
    return out


def test_fp32_error(study):
    for row in study["modes"]["fp32"]["errors"]:
        assert row["l2_rel"] < 1e-5, row
        assert abs(row["content_drift_rel"]) < 1e-5, row


# error budgets after 40 steps of the 160x160x24 case (relative L2 over wet
# cells against the bit-exact FP64 path; relative drift of the content).
# Measured on B200: bf16 1.0e-2 / 8e-6, bf16+sr 4.2e-3 / 7e-6,
# fp16 6.4e-4 / 4e-6, fp16+sr 5.3e-4 / 2e-6.
@pytest.mark.parametrize("mode,l2,drift", [("bf16", 2e-2, 5e-5), ("bf16+sr", 1e-2, 5e-5),
                                           ("fp16", 2e-3, 2e-5), ("fp16+sr", 2e-3, 2e-5)])
def test_16bit_storage_error(study, mode, l2, drift):
    for row in study["modes"][mode]["errors"]:
        assert row["l2_rel"] < l2, row
        assert abs(row["content_drift_rel"]) < drift, row


def test_stochastic_rounding_beats_nearest_for_bf16(study):
    """Stochastic rounding removes the stagnation of small increments that
    round-to-nearest BF16 stores suffer: lower error and drift."""
    for rn, sr in zip(study["modes"]["bf16"]["errors"], study["modes"]["bf16+sr"]["errors"]):
        assert sr["l2_rel"] < rn["l2_rel"]


def test_fp64_conserves(study):
    for row in study["modes"]["fp32"]["errors"]:
        assert abs(row["content_drift_rel_fp64"]) < 1e-13, row


def test_fp32_against_oracle_small(api, oracle):
    """FP32 mode against the CPU oracle directly on a small case."""
    import pyoracle
    from test_gpu_parity import synth_case
    nx, ny, nl = 23, 19, 11
    K, uv, w, T, S, dt = synth_case(api, nx, ny, nl, True, 11)
    api.set_precision("fp32")
    api.allocate_tracers(1)
    api.set_values(1, T)
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    api.advect_steps(3, dt)
    G = api.get_tracer_values(1)
    m = pyoracle.OracleMesh(oracle, nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    To = T.copy(order="F")
    for _ in range(3):
        m.step(To, To.copy(order="F"), uv, w, dt, "MUSCL", "PPM", "FCT")
    nlev = api.mesh_array("nlevels_nod2D")
    wet = np.arange(nl - 1)[:, None] < (nlev[None, :] - 1)
    assert np.linalg.norm(G[wet] - To[wet]) / np.linalg.norm(To[wet]) < 1e-5
