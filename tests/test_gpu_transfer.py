"""Host <-> device transfers through the C ABI: page-locked host arrays
(tracer_host_register, one DMA each way) and pageable ones (the library's
pinned staging ring) must move the same bits, in every precision mode, for
values, valuesAB and reads."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(api, mode, T, TAB, uv, w, dt, pin):
    L, N = T.shape
    T = np.asfortranarray(T.copy())
    TAB = np.asfortranarray(TAB.copy())
    out = np.zeros((L, N), order="F")
    if pin:
        for a in (T, TAB, out):
            api.pin(a)
    try:
        api.set_precision(mode)
        api.allocate_tracers(1)
        api.set_values(1, T, TAB)
        api.set_scheme(1, "MUSCL", "PPM", "FCT")
        api.set_velocity(uv, w)
        api.set_ab_refresh(False)
        api.advect_steps(2, dt)
        rc = api.lib.tracer_get_values_id(1, out.ctypes.data, L, N)
        assert rc == 0
        return out.copy()
    finally:
        if pin:
            for a in (T, TAB, out):
                api.unpin(a)


@pytest.mark.parametrize("mode", ["fp64", "fp32", "bf16", "fp16"])
def test_registered_and_pageable_transfers_agree(api, mode):
    from test_gpu_parity import synth_case
    K, uv, w, T, S, dt = synth_case(api, 50, 41, 17, True, 21)
    TAB = T + 0.25 * np.sin(np.arange(T.size)).reshape(T.shape, order="F")
    a = _run(api, mode, T, TAB, uv, w, dt, pin=False)
    b = _run(api, mode, T, TAB, uv, w, dt, pin=True)
    assert np.array_equal(a, b)
    assert np.all(np.isfinite(a))


def test_transfer_larger_than_the_staging_ring(api):
    """A field of several ring slots (32 MiB each) round-trips exactly in FP64
    through the pageable path and the registered path."""
    nx, nl = 400, 40  # 159,201 nodes x 39 levels x 8 B = 50 MB per field
    api.init_analytic(nx, nx, nl, periodic=True, full_rings=True)
    api.allocate_tracers(1)
    L, N = nl - 1, api.mesh_dims()["nod2D"]
    V = np.asfortranarray(np.random.default_rng(5).standard_normal((L, N)))
    api.set_values(1, V)
    assert np.array_equal(api.get_tracer_values(1), V)
    out = np.zeros((L, N), order="F")
    api.pin(V)
    api.pin(out)
    try:
        api.set_values(1, V * 2.0 + 1.0)  # temporary: pageable path
        api.set_values(1, V)              # registered path
        assert api.lib.tracer_get_values_id(1, out.ctypes.data, L, N) == 0
    finally:
        api.unpin(V)
        api.unpin(out)
    assert np.array_equal(out, V)


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_step_io_matches_the_separate_calls(api, pinned, prec):
    """tracer_advect_step_io (pipelined when the host arrays are page-locked)
    gives the bits of set_values / advect_step / get_values, two steps in a
    row, with valuesAB refreshed and frozen."""
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    c = layered_flow_case(api, 60, 14, seed=2)
    L, N = c.T.shape
    for refresh in (True, False):
        api.set_precision(prec)
        api.allocate_tracers(2)
        for t, v in ((1, c.T), (2, c.S)):
            api.set_values(t, v)
            api.set_scheme(t, "MUSCL", "PPM", "FCT")
        api.set_velocity(c.uv, c.w)
        api.set_ab_refresh(refresh)
        ins = [np.asfortranarray(c.T + 0.5), np.asfortranarray(c.S - 0.25)]
        outs = [np.zeros((L, N), order="F"), np.zeros((L, N), order="F")]
        if pinned:
            for a in ins + outs:
                api.pin(a)
        try:
            for step in range(2):
                api.advect_step_io(c.dt, ins, outs)
                got = [o.copy() for o in outs]
                api.set_values(1, ins[0])
                api.set_values(2, ins[1])
                api.advect_steps(1, c.dt)
                ref = [api.get_tracer_values(1), api.get_tracer_values(2)]
                for g, r in zip(got, ref):
                    if prec == "fp64":
                        assert np.array_equal(g.view(np.uint64), r.view(np.uint64)), (step, refresh)
                    else:
                        # the pipelined call steps each tracer alone, advect_steps both
                        # in one batch: the FP32 kernels of different batch sizes may
                        # contract different multiply-adds into FMAs
                        assert np.allclose(g, r, rtol=2e-6, atol=0), (step, refresh, np.max(np.abs(g - r)))
                for a, g in zip(ins, got):
                    a[...] = g  # the next step starts from this one's result
        finally:
            if pinned:
                for a in ins + outs:
                    api.unpin(a)
