"""Learned antidiffusive flux: training data from coarse-grained runs of the
plain method on refined meshes, training on the GPU (tensor-core forward and
backward kernels), and evaluation against the refined solution.

Workload (learned configuration): doubly periodic analytic meshes with
left-oriented edges and a flat bottom; the coarse mesh has nx = ny nodes per
side, the fine one `refine` times as many cells per side and the same levels;
a seeded smooth depth-independent non-divergent flow (w = 0) of the same
amplitude on both; smooth seeded blob/front tracer fields.  The fine run (FP64, MUSCL+PPM+FCT, dt / refine)
is box-filtered onto the coarse nodes every `refine` fine steps.

    python -m fesom2_tracer_dwarf_b200.learned --nx 500 --nl 32 --refine 4
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import _lib
from .tracer import FESOMTracerAdvection
from .workloads import LX, MAX_DEPTH, cfl_dt

R_EARTH = 6367500.0


def grid_ij(api, nx):
    """(i, j) grid indices of the periodic analytic mesh's nodes."""
    xy = api.mesh_array("coord").reshape(2, -1, order="F") * R_EARTH
    d = LX / (nx - 1)
    return np.rint(xy[0] / d).astype(np.int64) % (nx - 1), np.rint(xy[1] / d).astype(np.int64) % (nx - 1)


def coarse_grain(Tf, fine_ij, coarse_ij, refine):
    """Trapezoid box filter (width `refine` fine cells) of a fine periodic field
    (L, Nf) onto the coarse nodes (L, Nc); separable, evaluated only at the
    coarse nodes."""
    L = Tf.shape[0]
    nf = int(fine_ij[0].max()) + 1
    nc = nf // refine
    G = np.zeros((L, nf, nf))
    G[:, fine_ij[1], fine_ij[0]] = Tf
    h = refine // 2
    w = np.ones(2 * h + 1)
    w[0] = w[-1] = 0.5
    w /= w.sum()
    Gp = np.concatenate([G[:, :, nf - h:], G, G[:, :, :h]], axis=2)         # wrap in x
    A = sum(w[b] * Gp[:, :, b:b + nf:refine][:, :, :nc] for b in range(2 * h + 1))
    Ap = np.concatenate([A[:, nf - h:, :], A, A[:, :h, :]], axis=1)        # wrap in y
    C = sum(w[a] * Ap[:, a:a + nf:refine, :][:, :nc, :] for a in range(2 * h + 1))
    return np.asfortranarray(C[:, coarse_ij[1], coarse_ij[0]])


def flow(api, seed, amp):
    """Depth-independent non-divergent flow curl(psi) of amplitude amp: w is
    zero on every resolution, so the fine and coarse runs see the same flow."""
    return api.synth_velocity(seed=seed, umax=-amp, mode1=0.0, mode2=0.0, baro=1.0)


def flow_amplitude(api, seed):
    """Amplitude that gives |u| <= 1 m/s on the current (coarse) mesh."""
    uv, _ = api.synth_velocity(seed=seed, umax=-1.0, mode1=0.0, mode2=0.0, baro=1.0)
    return 1.0 / float(np.sqrt(uv[0] ** 2 + uv[1] ** 2).max())


def trajectory(api, nx, nl, seed, nsteps, refine, dt_c, amp, coarse_ij):
    """Coarse-grained snapshots (nsteps + 1, L, Nc) of an FP64 run on the
    refined mesh, one per coarse step."""
    nxf = refine * (nx - 1) + 1
    api.cleanup()
    api.init_analytic(nxf, nxf, nl, periodic=True, full_rings=True, left_oriented=True)
    fine_ij = grid_ij(api, nxf)
    uv, w = flow(api, seed, amp)
    T = api.synth_tracer(seed=seed + 7, kind=2)
    api.set_precision("fp64")
    api.allocate_tracers(1)
    api.set_values(1, T)
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    snaps = [coarse_grain(T, fine_ij, coarse_ij, refine)]
    for _ in range(nsteps):
        api.advect_steps(refine, dt_c / refine)
        snaps.append(coarse_grain(api.get_tracer_values(1), fine_ij, coarse_ij, refine))
    api.cleanup()
    return np.stack(snaps)


def coarse_setup(api, nx, nl, seed, amp=None):
    api.cleanup()
    api.init_analytic(nx, nx, nl, periodic=True, full_rings=True, left_oriented=True)
    if amp is None:
        amp = flow_amplitude(api, seed)
    uv, w = flow(api, seed, amp)
    return uv, w, amp, grid_ij(api, nx)


def make_dataset(nx, nl, seeds, nsteps, refine=4):
    api = FESOMTracerAdvection()
    data = []
    for s in seeds:
        uv, w, amp, cij = coarse_setup(api, nx, nl, s)
        dt = cfl_dt(api, nx, nx, nl, uv, w)
        snaps = trajectory(api, nx, nl, s, nsteps, refine, dt, amp, cij)
        data.append({"seed": s, "amp": amp, "dt": dt, "uv": uv, "w": w, "snaps": snaps})
    return data


def init_params(seed=0):
    """He-initialised hidden layers, a zero output layer: the untrained network
    adds nothing to the plain scheme."""
    lib = _lib.load()
    n = lib.tracer_mlp_num_params()
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=np.float32)
    p[:1024] = rng.standard_normal(1024) * np.sqrt(2.0 / 16)
    p[1088:5184] = rng.standard_normal(4096) * np.sqrt(2.0 / 64)
    return p


class Trainer:
    """Coarse FP32 engine with the learned flux; one tracer."""

    def __init__(self, nx, nl, params=None):
        self.api = FESOMTracerAdvection()
        self.api.cleanup()
        self.api.init_analytic(nx, nx, nl, periodic=True, full_rings=True, left_oriented=True)
        self.api.set_precision("fp32")
        self.api.allocate_tracers(1)
        self.api.set_scheme(1, "MUSCL", "PPM", "FCT")
        self.api.set_ab_refresh(True)
        self.nx, self.nl = nx, nl
        self.params = init_params() if params is None else np.ascontiguousarray(params, dtype=np.float32)
        self.lib = self.api.lib
        self.current_seed = None

    def use(self, traj):
        if self.current_seed != traj["seed"]:
            self.api.set_velocity(traj["uv"], traj["w"])
            self.current_seed = traj["seed"]

    def load(self, p, on=True):
        """Put parameters p into the engine (the trainer's own copy is unchanged)."""
        q = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(self.lib, self.lib.tracer_learn_set(_lib.ptr(q), int(on)), "tracer_learn_set")

    def set_params(self, p, on=True):
        self.params = np.ascontiguousarray(p, dtype=np.float32)
        self.load(self.params, on)

    def get_params(self):
        p = np.zeros_like(self.params)
        _lib.check(self.lib, self.lib.tracer_learn_get(_lib.ptr(p)), "tracer_learn_get")
        return p

    def step_loss(self, traj, k, lr=0.0, update=False, fct=True):
        self.use(traj)
        loss = ctypes.c_double()
        a = np.asfortranarray(traj["snaps"][k])
        b = np.asfortranarray(traj["snaps"][k + 1])
        rc = self.lib.tracer_learn_step(_lib.ptr(a), _lib.ptr(b), traj["dt"], lr, int(update), int(fct),
                                        ctypes.byref(loss))
        _lib.check(self.lib, rc, "tracer_learn_step")
        return loss.value

    def train(self, data, iters, lr=1e-3, seed=0, lr_final=None, fct=False):
        self.set_params(self.params, on=False)
        rng = np.random.default_rng(seed)
        losses = []
        for it in range(iters):
            rate = lr if lr_final is None else lr * (lr_final / lr) ** (it / max(1, iters - 1))
            traj = data[rng.integers(len(data))]
            k = int(rng.integers(traj["snaps"].shape[0] - 1))
            losses.append(self.step_loss(traj, k, rate, True, fct))
        self.params = self.get_params()
        return losses

    def one_step_losses(self, traj, params=None, fct=True):
        """Mean one-step loss over a trajectory (MUSCL+PPM, FCT-limited when
        fct), for the given parameters (None: the plain scheme, a zero network)."""
        p = np.zeros_like(self.params) if params is None else params
        self.load(p, on=False)
        out = [self.step_loss(traj, k, fct=fct) for k in range(traj["snaps"].shape[0] - 1)]
        return float(np.mean(out))

    def rollout_error(self, traj, params=None, nsteps=None):
        """Relative L2 error against the coarse-grained refined run after
        nsteps coarse steps of MUSCL+PPM+FCT (learned when params is given),
        and the relative content drift."""
        api = self.api
        self.use(traj)
        if params is None:
            _lib.check(api.lib, api.lib.tracer_learn_set(None, 0), "tracer_learn_set")
        else:
            self.load(params, on=True)
        n = traj["snaps"].shape[0] - 1 if nsteps is None else nsteps
        api.set_values(1, traj["snaps"][0])
        v0 = api.volume_sum(1)[1]
        api.advect_steps(n, traj["dt"])
        T = api.get_tracer_values(1)
        v1 = api.volume_sum(1)[1]
        ref = traj["snaps"][n]
        if params is not None:
            _lib.check(api.lib, api.lib.tracer_learn_set(None, 0), "tracer_learn_set")
        return (float(np.linalg.norm(T - ref) / np.linalg.norm(ref)), float((v1 - v0) / v0),
                float(T.min()), float(T.max()))


def plain_error_at(nx_fine_factor, nx, nl, traj, refine):
    """Plain FP32 MUSCL+PPM+FCT at nx_fine_factor times the coarse resolution,
    coarse-grained: its relative L2 error against the refined reference."""
    api = FESOMTracerAdvection()
    api.cleanup()
    f = nx_fine_factor
    nxm = f * (nx - 1) + 1
    api.init_analytic(nxm, nxm, nl, periodic=True, full_rings=True, left_oriented=True)
    mij = grid_ij(api, nxm)
    uv, w = flow(api, traj["seed"], traj["amp"])
    T0 = api.synth_tracer(seed=traj["seed"] + 7, kind=2)
    api.set_precision("fp32")
    api.allocate_tracers(1)
    api.set_values(1, T0)
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(uv, w)
    api.set_ab_refresh(True)
    n = traj["snaps"].shape[0] - 1
    api.advect_steps(f * n, traj["dt"] / f)
    T = api.get_tracer_values(1)
    api.cleanup()
    api.init_analytic(nx, nx, nl, periodic=True, full_rings=True, left_oriented=True)
    cij = grid_ij(api, nx)
    api.cleanup()
    C = coarse_grain(T, mij, cij, f)
    ref = traj["snaps"][n]
    return float(np.linalg.norm(C - ref) / np.linalg.norm(ref))


TRAINED = __import__("pathlib").Path(__file__).resolve().parent / "data" / "learned_flux_500x32.npy"


def trained_params():
    """Parameters trained on the 500x500x32 configuration (4x refined,
    trained through the FCT step and its limiter ratios), shipped with the
    package."""
    return np.load(TRAINED).astype(np.float32)


def study(nx=500, nl=32, refine=4, train_seeds=(1, 2, 3), val_seed=11, nsteps=20, iters=600, lr=2e-3, fct=True):
    t0 = time.perf_counter()
    data = make_dataset(nx, nl, list(train_seeds) + [val_seed], nsteps, refine)
    t_data = time.perf_counter() - t0
    train, val = data[:-1], data[-1]
    tr = Trainer(nx, nl)
    base = {f: (float(np.mean([tr.one_step_losses(d, None, f) for d in train])), tr.one_step_losses(val, None, f))
            for f in (True, False)}
    t1 = time.perf_counter()
    losses = tr.train(train, iters, lr=lr, lr_final=lr / 20, fct=fct)
    t_train = time.perf_counter() - t1
    p = tr.params
    out = {
        "config": {"nx": nx, "nl": nl, "refine": refine, "train_seeds": list(train_seeds), "val_seed": val_seed,
                   "coarse_steps": nsteps, "iters": iters, "lr": lr, "trained_with_fct": fct,
                   "data_seconds": t_data, "train_seconds": t_train, "dt": val["dt"]},
        "one_step_loss": {
            ("fct" if f else "unlimited"): {
                "train_plain": base[f][0], "val_plain": base[f][1],
                "train_learned": float(np.mean([tr.one_step_losses(d, p, f) for d in train])),
                "val_learned": tr.one_step_losses(val, p, f)} for f in (True, False)},
        "training_curve": [float(x) for x in losses[:: max(1, iters // 50)]],
        "rollout_val": {"plain": tr.rollout_error(val, None), "learned": tr.rollout_error(val, p)},
    }
    out["rollout_val"]["plain_2x_resolution"] = plain_error_at(2, nx, nl, val, refine)
    out["params"] = p.tolist()
    return out


def main():
    a = argparse.ArgumentParser()
    a.add_argument("--nx", type=int, default=500)
    a.add_argument("--nl", type=int, default=32)
    a.add_argument("--refine", type=int, default=4)
    a.add_argument("--steps", type=int, default=20)
    a.add_argument("--iters", type=int, default=600)
    a.add_argument("--lr", type=float, default=2e-3)
    a.add_argument("--params-out", default=None)
    a.add_argument("--unlimited-training", action="store_true",
                   help="train on the unlimited step instead of through the FCT limiter")
    args = a.parse_args()
    out = study(args.nx, args.nl, args.refine, nsteps=args.steps, iters=args.iters, lr=args.lr,
                fct=not args.unlimited_training)
    if args.params_out:
        np.save(args.params_out, np.array(out["params"], dtype=np.float32))
    out.pop("params")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
