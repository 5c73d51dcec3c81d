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


@pytest.fixture(scope="module")
def study():
    from fesom2_tracer_dwarf_b200.precision_study import study as run
    return run(160, 24, 40)


def test_fp32_error(study):
    for row in study["modes"]["fp32"]["errors"]:
        assert row["l2_rel"] < 1e-5, row
        assert abs(row["content_drift_rel"]) < 1e-5, row


@pytest.mark.parametrize("mode,l2,drift", [("bf16", 2e-2, 5e-3), ("fp16", 3e-3, 1e-3)])
def test_16bit_storage_error(study, mode, l2, drift):
    for row in study["modes"][mode]["errors"]:
        assert row["l2_rel"] < l2, row
        assert abs(row["content_drift_rel"]) < drift, row


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
