"""The CUDA step on the reference's pi mesh (irregular spherical triangles,
elem_cos != 1, 2 to 8 elements per node, real bathymetry of 4 to 45 wet
layers, closed coastlines), read through tracer_load_mesh_from_files: bit-identical to the
oracle stepping on its own restatement of the same mesh files, in the
reference's conventions and in FESOM2's; conservation, constant preservation
and the FCT bounds over longer runs."""
import math

import numpy as np
import pytest

from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu

FESOM2 = dict(angle_scale=math.pi / 180.0, cyclic_length=2.0 * math.pi)
CONV = {"reference": {}, "fesom2": FESOM2}


def pi_case(api, mesh_dir, conv, seed=5):
    """Mesh, a seeded layered flow with w from the discrete continuity
    (|u| <= 0.5 m/s), two tracers and a dt at about CFL 0.3."""
    api.load_mesh_from_files(mesh_dir, **CONV[conv])
    uv, w = api.synth_velocity(seed=seed, umax=0.5, mode2=0.5)
    T = api.synth_tracer(seed=seed + 1, kind=0)
    S = api.synth_tracer(seed=seed + 2, kind=1)
    ea = api.mesh_array("elem_area")
    zbar = api.mesh_array("zbar")
    dz = float(np.min(zbar[:-1] - zbar[1:]))
    wmax = float(np.abs(w).max())
    dt = 0.3 * min(math.sqrt(ea.min()) / 0.5, dz / wmax if wmax > 0 else math.inf)
    return uv, w, T, S, dt


SCHEMES = [("MUSCL", "PPM", "FCT"), ("MFCT", "QR4C", "FCT"), ("UPW1", "UPW1", "NONE"), ("MUSCL", "CDIFF", "NONE")]


@pytest.mark.parametrize("conv", ["reference", "fesom2"])
@pytest.mark.parametrize("hor,ver,lim", SCHEMES)
def test_pi_mesh_bitwise(api, oracle, pi_mesh_dir, conv, hor, ver, lim):
    import pyoracle
    uv, w, T, S, dt = pi_case(api, pi_mesh_dir, conv)
    m = pyoracle.OracleMesh.from_files(oracle, pi_mesh_dir, **CONV[conv])
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    for t in (1, 2):
        api.set_scheme(t, hor, ver, lim)
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    To, So = T.copy(order="F"), S.copy(order="F")
    for step in range(4):
        api.advect_steps(1, dt)
        m.step(To, To.copy(order="F"), uv, w, dt, hor, ver, lim)
        m.step(So, So.copy(order="F"), uv, w, dt, hor, ver, lim)
        assert_bitwise(api.get_tracer_values(1), To, f"{conv} {hor}/{ver}/{lim} T step {step + 1}")
        assert_bitwise(api.get_tracer_values(2), So, f"{conv} {hor}/{ver}/{lim} S step {step + 1}")


@pytest.mark.parametrize("conv", ["reference", "fesom2"])
def test_pi_mesh_conservation_constancy_and_bounds(api, pi_mesh_dir, conv):
    """60 MUSCL/PPM/FCT steps: the volume integral of T drifts by round-off
    only, a constant field stays constant, and T stays inside its initial
    range (FCT)."""
    uv, w, T, S, dt = pi_case(api, pi_mesh_dir, conv)
    nlev = api.mesh_array("nlevels_nod2D")
    wet = np.arange(T.shape[0])[:, None] < (nlev[None, :] - 1)
    C = np.where(wet, 7.25, 0.0)
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, np.asfortranarray(C))
    for t in (1, 2):
        api.set_scheme(t, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    _, v0 = api.volume_sum(1)
    api.advect_steps(60, dt)
    _, v1 = api.volume_sum(1)
    assert abs(v1 - v0) <= 1e-12 * abs(v0)
    Tn, Cn = api.get_tracer_values(1), api.get_tracer_values(2)
    assert np.all(np.isfinite(Tn))
    assert np.max(np.abs(Cn[wet] - 7.25)) < 1e-11
    assert Tn[wet].min() >= T[wet].min() - 1e-12 and Tn[wet].max() <= T[wet].max() + 1e-12
    assert np.abs(Tn - T)[wet].max() > 1e-3  # the flow did move the field
