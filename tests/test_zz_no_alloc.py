"""tracer_advect_device_noalloc: the tracer step for callers that cannot
allocate device memory (their runtime owns the GPU's memory pool, or their
time loop must not allocate).  It runs the same kernels as tracer_advect_step
with its work space taken from a static device array, so its result must be
bit-identical to the existing entry point's -- the tolerance every FP64
parity test here uses -- on two calls in a row, for every limiter path (with
FCT the edge volume fluxes are stored and re-read; without it they are not).
It must also leave the device's free memory unchanged, run on the engine's
device from any host thread, and see inputs the caller wrote with
asynchronous copies on its own streams."""
import ctypes
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCHEMES = [("MUSCL", "PPM", "FCT"), ("MUSCL", "PPM", "NONE"), ("UPW1", "UPW1", "NONE"), ("UPW1", "UPW1", "FCT"),
           ("MFCT", "QR4C", "FCT")]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _setup(api, nx, ny, nl, seed, scheme=("MUSCL", "PPM", "FCT")):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, 1), nl, seed)
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    uv, w = api.synth_velocity(seed=seed + 1, umax=1.0, mode2=0.5)
    T = api.synth_tracer(seed=seed + 2, kind=0)
    api.allocate_tracers(1)
    api.set_values(1, T)
    api.set_scheme(1, *scheme)
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    assert api.lib.tracer_init_for_advection() == 0
    return T, 0.5 * 1.0e5 / (nx - 1)


def _padded(api, T):
    import torch
    d = api.mesh_dims()
    N, L, S = d["nod2D"], d["nl"] - 1, d["level_stride"]
    pad = np.zeros((N, S))
    pad[:, :L] = T.T
    return torch.from_numpy(pad).cuda(), L


@pytest.mark.parametrize("scheme", SCHEMES, ids=["/".join(s) for s in SCHEMES])
def test_noalloc_step_matches_tracer_advect_step(api, scheme):
    import torch
    T, dt = _setup(api, 24, 20, 11, 7, scheme)
    cur, L = _padded(api, T)
    outs = [torch.zeros_like(cur), torch.zeros_like(cur)]
    torch.cuda.synchronize()
    for call in range(2):
        out = outs[call]
        rc = api.lib.tracer_advect_device_noalloc(1, _p(cur), _p(cur), _p(out), dt)
        assert rc == 0, api.lib.tracer_last_error()
        assert api.lib.tracer_last_error() == b""
        api.advect_steps(1, dt)                      # the existing entry point, same step
        ref = api.get_tracer_values(1)
        got = np.asfortranarray(out.cpu().numpy()[:, :L].T)
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), f"call {call + 1}"
        cur = out


def test_noalloc_leaves_free_device_memory_unchanged(api):
    import torch
    T, dt = _setup(api, 24, 20, 11, 5)
    cur, _ = _padded(api, T)
    out = torch.zeros_like(cur)
    # the first call loads the step kernels' code (CUDA lazy module loading)
    assert api.lib.tracer_advect_device_noalloc(1, _p(cur), _p(cur), _p(out), dt) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert api.lib.tracer_advect_device_noalloc(1, _p(cur), _p(cur), _p(out), dt) == 0
        cur, out = out, cur
    free1, _ = torch.cuda.mem_get_info()
    assert free0 == free1


def test_noalloc_waits_for_the_callers_async_copies(api):
    """The host fills the input with an asynchronous copy on its own stream
    and calls without synchronising: the step must see the copied values."""
    import torch
    T, dt = _setup(api, 24, 20, 11, 9)
    src, L = _padded(api, T)
    ref_out = torch.zeros_like(src)
    torch.cuda.synchronize()
    assert api.lib.tracer_advect_device_noalloc(1, _p(src), _p(src), _p(ref_out), dt) == 0
    expect = ref_out.cpu().numpy().copy()

    host = src.cpu().pin_memory()
    dst = torch.zeros_like(src)
    out = torch.zeros_like(src)
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        for _ in range(4):      # queue enough work that the copy is still in flight
            dst.copy_(host, non_blocking=True)
    assert api.lib.tracer_advect_device_noalloc(1, _p(dst), _p(dst), _p(out), dt) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.array_equal(got[:, :L].view(np.uint64), expect[:, :L].view(np.uint64))


def test_noalloc_from_a_second_host_thread(api):
    """A host thread other than the one that created the engine (its own
    current-device state) runs the step on the engine's device."""
    import torch
    T, dt = _setup(api, 24, 20, 11, 11)
    cur, L = _padded(api, T)
    a, b = torch.zeros_like(cur), torch.zeros_like(cur)
    torch.cuda.synchronize()
    assert api.lib.tracer_advect_device_noalloc(1, _p(cur), _p(cur), _p(a), dt) == 0
    res = {}

    def worker():
        res["rc"] = api.lib.tracer_advect_device_noalloc(1, _p(cur), _p(cur), _p(b), dt)
        res["err"] = api.lib.tracer_last_error()

    th = threading.Thread(target=worker)
    th.start()
    th.join()
    assert res["rc"] == 0, res["err"]
    torch.cuda.synchronize()
    assert np.array_equal(a.cpu().numpy().view(np.uint64), b.cpu().numpy().view(np.uint64))


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
