"""Learned antidiffusive flux inside the engine: a zero network reproduces the
plain scheme bit for bit; the learned flux still passes the unchanged FCT
limiter (content conserved, bounds kept); training on coarse-grained refined
runs lowers the one-step error of held-out data below the plain scheme's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plain_vs_zero(api):
    from fesom2_tracer_dwarf_b200.learned import coarse_setup, init_params
    from fesom2_tracer_dwarf_b200.workloads import cfl_dt
    nx, nl = 33, 10
    uv, w, amp, _ = coarse_setup(api, nx, nl, 4)
    dt = cfl_dt(api, nx, nx, nl, uv, w)
    T = api.synth_tracer(seed=3, kind=2)
    api.set_precision("fp32")
    api.allocate_tracers(1)
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    out = []
    for on in (False, True):
        p = init_params(5)  # zero output layer
        assert api.lib.tracer_learn_set(p.ctypes.data, int(on)) == 0
        api.set_values(1, T)
        api.advect_steps(3, dt)
        out.append(api.get_tracer_values(1))
    return out


def test_zero_network_reproduces_plain_scheme(api):
    plain, learned = _plain_vs_zero(api)
    assert np.array_equal(plain, learned)


@pytest.mark.parametrize("fct,tol", [(0, 0.05), (1, 0.15)])
def test_training_gradient_matches_finite_differences(api, fct, tol):
    """The gradient learn_step back-propagates (loss -> dL/dy through the
    unlimited step, or through the FCT step and its limiter ratios ->
    tensor-core backward) against central differences of the loss in the
    parameters the kernels keep in FP32 (b3, w3, b2).  The limited loss has
    kinks where a limiter factor switches argument, hence the wider tolerance."""
    import ctypes
    from fesom2_tracer_dwarf_b200.learned import coarse_setup, init_params
    from fesom2_tracer_dwarf_b200.workloads import cfl_dt
    nx, nl = 25, 6
    uv, w, amp, _ = coarse_setup(api, nx, nl, 8)
    dt = cfl_dt(api, nx, nx, nl, uv, w)
    T = np.asfortranarray(api.synth_tracer(seed=9, kind=2))
    target = np.asfortranarray(T + 0.05 * np.sin(np.arange(T.size)).reshape(T.shape, order="F"))
    api.set_precision("fp32")
    api.allocate_tracers(1)
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    rng = np.random.default_rng(2)
    p = init_params(3)
    p[5248:5312] = rng.standard_normal(64).astype(np.float32) * 0.3
    p[5312] = 0.05
    lib = api.lib

    def loss(q, update=False):
        assert lib.tracer_learn_set(np.ascontiguousarray(q, dtype=np.float32).ctypes.data, 0) == 0
        out = ctypes.c_double()
        assert lib.tracer_learn_step(T.ctypes.data, target.ctypes.data, dt, 0.0, int(update), fct,
                                     ctypes.byref(out)) == 0
        return out.value

    loss(p, update=True)
    g = np.zeros_like(p)
    assert lib.tracer_learn_grad(g.ctypes.data) == 0
    for i, eps in [(5312, 1e-2), (5248, 2e-2), (5270, 2e-2), (5290, 2e-2), (5184, 2e-2), (5200, 2e-2)]:
        e = np.zeros_like(p)
        e[i] = eps
        fd = (loss(p + e) - loss(p - e)) / (2 * eps)
        assert abs(fd - g[i]) <= tol * abs(fd) + 1e-9, (i, fd, g[i])


@pytest.fixture(scope="module")
def small_study():
    from fesom2_tracer_dwarf_b200.learned import study
    return study(nx=65, nl=12, refine=4, train_seeds=(1, 2, 3), val_seed=11, nsteps=12, iters=500, lr=3e-3,
                 fct=False)


def test_limiter_aware_training_lowers_the_limited_error():
    """Trained through the FCT step (gradient through the limiter ratios), the
    network lowers the one-step error of the limited scheme on an unseen
    trajectory."""
    from fesom2_tracer_dwarf_b200.learned import study
    out = study(nx=65, nl=12, refine=4, train_seeds=(1, 2, 3), val_seed=11, nsteps=12, iters=500, lr=3e-3,
                fct=True)
    f = out["one_step_loss"]["fct"]
    assert f["val_learned"] < 0.98 * f["val_plain"], f
    assert abs(out["rollout_val"]["learned"][1]) < 1e-6


def test_training_beats_plain_scheme_on_held_out_data(small_study):
    """Trained on three coarse-grained refined trajectories, the network lowers
    the one-step error of the (unlimited) MUSCL+PPM step on a fourth, unseen
    trajectory to well under the plain scheme's."""
    u = small_study["one_step_loss"]["unlimited"]
    assert u["val_learned"] < 0.5 * u["val_plain"], u
    assert u["train_learned"] < 0.5 * u["train_plain"], u


def test_learned_flux_through_fct_conserves_and_stays_bounded(small_study):
    """Through the unchanged FCT limiter the learned run conserves the content
    (FP32 round-off) and keeps the plain run's range; its error stays at or
    below the plain scheme's."""
    plain, learned = small_study["rollout_val"]["plain"], small_study["rollout_val"]["learned"]
    assert abs(learned[1]) < 1e-6
    assert learned[2] >= plain[2] - 1e-3 and learned[3] <= plain[3] + 1e-3
    assert learned[0] <= plain[0] * 1.01, (plain, learned)


def test_shipped_parameters_load(api):
    from fesom2_tracer_dwarf_b200.learned import trained_params
    p = trained_params()
    assert p.shape == (api.lib.tracer_mlp_num_params(),) and np.all(np.isfinite(p))
    assert np.abs(p[5248:5312]).max() > 0.0
