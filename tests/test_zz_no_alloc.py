"""tracer_advect_device_noalloc: the tracer step for callers that cannot
allocate device memory (their runtime owns the GPU's memory pool, or their
time loop must not allocate).  It runs the same kernels as tracer_advect_step
with its work space taken from a static device array, so its result must be
bit-identical to the existing entry point's -- the tolerance every FP64
parity test here uses -- on two calls in a row."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _setup(api, nx, ny, nl, seed):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, 1), nl, seed)
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    uv, w = api.synth_velocity(seed=seed + 1, umax=1.0, mode2=0.5)
    T = api.synth_tracer(seed=seed + 2, kind=0)
    api.allocate_tracers(1)
    api.set_values(1, T)
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    assert api.lib.tracer_init_for_advection() == 0
    return T, 0.5 * 1.0e5 / (nx - 1)


def test_noalloc_step_matches_tracer_advect_step(api):
    import torch
    T, dt = _setup(api, 24, 20, 11, 7)
    d = api.mesh_dims()
    N, L, S = d["nod2D"], d["nl"] - 1, d["level_stride"]
    pad = np.zeros((N, S))
    pad[:, :L] = T.T
    cur = torch.from_numpy(pad).cuda()
    outs = [torch.zeros_like(cur), torch.zeros_like(cur)]
    torch.cuda.synchronize()
    for call in range(2):
        out = outs[call]
        rc = api.lib.tracer_advect_device_noalloc(1, _p(cur), _p(cur), _p(out), dt)
        assert rc == 0, api.lib.tracer_last_error()
        api.advect_steps(1, dt)                      # the existing entry point, same step
        ref = api.get_tracer_values(1)
        got = np.asfortranarray(out.cpu().numpy()[:, :L].T)
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), f"call {call + 1}"
        cur = out


def test_noalloc_rejects_meshes_beyond_the_static_array(api):
    import torch
    assert api.lib.tracer_noalloc_scratch_bytes() == 64 << 20
    T, dt = _setup(api, 200, 200, 64, 3)
    d = api.mesh_dims()
    buf = torch.zeros((d["nod2D"], d["level_stride"]), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(buf)
    torch.cuda.synchronize()
    assert api.lib.tracer_advect_device_noalloc(1, _p(buf), _p(buf), _p(out), dt) == -1
    assert b"static" in api.lib.tracer_last_error()
