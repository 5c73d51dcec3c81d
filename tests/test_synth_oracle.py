"""The oracle's restatement of the benchmark's seeded inputs (bathymetry,
layered flow, tracers, dt) equals the library's generators bit for bit, so
the CPU baseline, which builds its inputs with the oracle alone, runs the
same workload as the GPU arm."""
import numpy as np
import pytest


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64) if a.dtype == np.float64 else a,
                                                 b.view(np.uint64) if b.dtype == np.float64 else b)


@pytest.mark.parametrize("nx,nl,periodic,seed", [(30, 12, True, 0), (25, 9, False, 5), (41, 20, True, 3)])
def test_layered_flow_case_matches_the_library(api, oracle, nx, nl, periodic, seed):
    import pyoracle
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, nx, nl, periodic=periodic, seed=seed)
    m, K, uv, w, T, S, dt, wet = pyoracle.layered_flow_case(oracle, nx, nl, seed=seed, periodic=periodic)
    assert _same(K, c.K)
    assert _same(uv, c.uv)
    assert _same(w, c.w)
    assert _same(T, c.T)
    assert _same(S, c.S)
    assert dt == c.dt
    assert wet == c.wet_cells


def test_mt19937_64_matches_the_library_stream(api, oracle):
    """The bathymetry draws its modes from MT19937-64; a second seed and a
    large grid exercise many draws of the recurrence (more than one 312-word
    refill)."""
    import pyoracle
    from fesom2_tracer_dwarf_b200 import synth_bathymetry_smooth
    for seed in (1, 12345678901):
        a = synth_bathymetry_smooth(120, 90, 40, periodic=False, corr_cells=3.0, seed=seed)
        b = pyoracle.synth_bathymetry_smooth(oracle, 120, 90, 40, periodic=False, corr_cells=3.0, seed=seed)
        assert np.array_equal(a, b)
