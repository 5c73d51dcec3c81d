"""tracer_get_stats / tracer_get_stats_id reduce on the device: min and max
bit-identical to the host's view of the field (nl-1 x nod2D, dry cells
included), the NaN count exact, the sum within 1e-13 relative of an exact
sum (compensated, in a fixed order: the same bits on every call)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(api, prec="fp64"):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(40, 33, 1), 17, 9)
    api.init_analytic(40, 33, 17, periodic=True, full_rings=True, node_K=K)
    api.set_precision(prec)
    T = api.synth_tracer(seed=2, kind=0)
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, api.synth_tracer(seed=3, kind=1))
    return T


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16"])
def test_device_stats_match_the_host_view(api, prec):
    _case(api, prec)
    for t in (1, 2):
        v = api.get_tracer_values(t)
        st = api.get_statistics(t)
        assert st["min"] == v.min() and st["max"] == v.max() and st["nan"] == 0
        exact = math.fsum(v.ravel())
        assert abs(st["sum"] - exact) <= 1e-13 * abs(exact)
        assert api.get_statistics(t) == st  # deterministic


def test_device_stats_count_nans(api):
    T = _case(api)
    T = T.copy(order="F")
    T[3, 7] = np.nan
    T[0, 100] = np.nan
    api.set_values(1, T)
    st = api.get_statistics(1)
    assert st["nan"] == 2
    ok = T[~np.isnan(T)]
    assert st["min"] == ok.min() and st["max"] == ok.max()
    T[0, 0] = np.nan  # the host loop seeds min and max with the first value
    api.set_values(1, T)
    st = api.get_statistics(1)
    assert st["nan"] == 3 and math.isnan(st["min"]) and math.isnan(st["max"])


@pytest.mark.parametrize("path", ["fused", "five"])
def test_nonfinite_new_values_are_flagged_on_the_device(api, path):
    """The update kernels count non-finite new values: none on a clean run;
    a NaN planted in one wet cell spreads to its neighbours within a step
    and is reported by tracer_step_status, and with the check on by
    tracer_advect_step itself (-1 and a message)."""
    import ctypes
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, 40, 12, seed=1)
    api.set_step_path(path)
    api.allocate_tracers(1)
    api.set_values(1, c.T)
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(c.uv, c.w)
    api.set_ab_refresh(True)
    n = ctypes.c_longlong(-1)
    api.advect_steps(2, c.dt)
    assert api.lib.tracer_step_status(ctypes.byref(n)) == 0 and n.value == 0
    T = c.T.copy(order="F")
    T[2, 300] = np.nan
    api.set_values(1, T)
    api.advect_steps(1, c.dt)
    assert api.lib.tracer_step_status(ctypes.byref(n)) == 0 and n.value >= 1
    assert api.lib.tracer_step_status(ctypes.byref(n)) == 0 and n.value == 0  # reset by the read
    assert api.lib.tracer_set_nan_check(1) == 0
    assert api.lib.tracer_advect_step(c.dt) == -1
    assert b"non-finite" in api.lib.tracer_last_error()
    api.lib.tracer_set_nan_check(0)
