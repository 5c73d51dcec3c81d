"""Binary restarts on the GPU path: a run written out with tracer_finalize
and read back with tracer_init continues bit-identically to the run that
never stopped (analytic dwarf with bathymetry, and the irregular pi mesh),
and the call sequence of the reference's python/demo_tracer.py main()
(tracer_init_mpi, tracer_init, ten tracer_advect_step + tracer_get_stats,
tracer_finalize, tracer_finalize_mpi) and tracer_run_workflow run from a
restart the library wrote."""
import ctypes

import numpy as np
import pytest

from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu


def _continue_bitwise(api, tmp_path, n1, n2, dt):
    ref = tmp_path / "restart"
    api.advect_steps(n1, dt)
    assert api.lib.tracer_finalize(str(ref).encode()) == 0, api.lib.tracer_last_error()
    api.cleanup()
    assert api.lib.tracer_init(str(ref).encode()) == 0, api.lib.tracer_last_error()
    api.advect_steps(n2, dt)
    return api.get_tracer_values(1), api.get_tracer_values(2)


def test_analytic_restart_continues_bitwise(api, tmp_path):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry

    def setup():
        K = synth_bathymetry(api.lib.tracer_analytic_nodes(30, 26, 1), 14, 2)
        api.init_analytic(30, 26, 14, periodic=True, full_rings=True, node_K=K)
        uv, w = api.synth_velocity(seed=3, umax=1.0, mode2=0.5)
        T, S = api.synth_tracer(seed=4, kind=0), api.synth_tracer(seed=5, kind=1)
        api.allocate_tracers(2)
        api.set_values(1, T)
        api.set_values(2, S)
        api.set_scheme(1, "MUSCL", "PPM", "FCT")
        api.set_scheme(2, "MFCT", "QR4C", "FCT")
        api.set_velocity(uv, w)

    dt = 0.5 * 1.0e5 / 29
    setup()
    api.advect_steps(5, dt)
    T5, S5 = api.get_tracer_values(1), api.get_tracer_values(2)
    api.cleanup()
    setup()
    T, S = _continue_bitwise(api, tmp_path, 2, 3, dt)
    assert_bitwise(T, T5, "T")
    assert_bitwise(S, S5, "S")


def test_pi_mesh_restart_continues_bitwise(api, tmp_path, pi_mesh_dir):
    from test_gpu_pi_mesh import pi_case

    def setup():
        uv, w, T, S, dt = pi_case(api, pi_mesh_dir, "reference")
        api.allocate_tracers(2)
        api.set_values(1, T)
        api.set_values(2, S)
        for t in (1, 2):
            api.set_scheme(t, "MUSCL", "PPM", "FCT")
        api.set_velocity(uv, w)
        return dt

    dt = setup()
    api.advect_steps(4, dt)
    T4, S4 = api.get_tracer_values(1), api.get_tracer_values(2)
    api.cleanup()
    setup()
    T, S = _continue_bitwise(api, tmp_path, 1, 3, dt)
    assert_bitwise(T, T4, "T")
    assert_bitwise(S, S4, "S")


def test_demo_main_sequence_and_workflow(api, tmp_path):
    """The analytic dwarf (reference fields) written as a restart, then the
    demo's main() sequence through the C ABI: the tracer content is
    conserved and nothing is NaN; tracer_run_workflow does the same."""
    api.init_analytic(20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = api.analytic_fields()
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    for t in (1, 2):
        api.set_scheme(t, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    restart = str(tmp_path / "fesom_bin_restart").encode()
    assert api.lib.tracer_finalize(restart) == 0
    api.cleanup()

    lib = api.lib
    assert lib.tracer_init_mpi(0) == 0
    assert lib.tracer_init(restart) == 0
    mn, mx, sm = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    sums = []
    for step in range(10):
        assert lib.tracer_advect_step(1000.0) == 0
        assert lib.tracer_get_stats(ctypes.byref(mn), ctypes.byref(mx), ctypes.byref(sm)) == 0
        sums.append(sm.value)
        assert np.isfinite(mn.value) and np.isfinite(mx.value)
    assert max(abs(s - sums[0]) for s in sums) <= 1e-9 * abs(sums[0])
    assert lib.tracer_finalize(restart) == 0
    assert lib.tracer_finalize_mpi() == 0
    api.cleanup()
    assert lib.tracer_run_workflow(restart, 3, 1000.0) == 0
    api.cleanup()
    assert lib.tracer_init(restart) == 0
    assert np.all(np.isfinite(api.get_tracer_values(1)))
