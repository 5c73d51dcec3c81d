"""Seeded synthetic workloads of the tracer step (shared by the benchmark, the
precision study and the tests).

``layered_flow_case`` builds the plain-method-at-scale case: a doubly periodic
(or closed) analytic mesh whose horizontal and vertical edges are reversed so
that edge_tri(1) lies left of every edge (the reference's analytic mesh,
lib/analytic_mesh.F90:386-441, has it on the right of those edges and on the
left of the diagonals, which makes a non-divergent field divergent on the
discrete operator); smooth bathymetry with per-node bottom level uniform in
[3, nl]; a smooth layered flow (a depth-independent non-divergent part plus two
zero-column-mean vertical modes, w from the discrete continuity, so that
constants stay constant), |u| <= 1 m/s; dt at CFL 0.5 of the faster of the
horizontal and vertical crossings; two tracers (temperature-like U[0,20] plus
Gaussian blobs; salinity-like 35 + N(0, 0.5)).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .tracer import FESOMTracerAdvection, synth_bathymetry_smooth

LX = LY = 1.0e5
MAX_DEPTH = 1000.0


@dataclass
class Case:
    nx: int
    ny: int
    nl: int
    periodic: bool
    K: np.ndarray        # per-node bottom level index (nlevels_nod2D)
    uv: np.ndarray       # (2, nl-1, elem2D) Fortran order
    w: np.ndarray        # (nl, nod2D) Fortran order
    T: np.ndarray        # (nl-1, nod2D) temperature-like
    S: np.ndarray        # (nl-1, nod2D) salinity-like
    dt: float
    wet_cells: int       # wet (level, node) cells of one tracer
    wet: np.ndarray      # (nl-1, nod2D) bool mask of wet cells


def cfl_dt(api: FESOMTracerAdvection, nx: int, ny: int, nl: int, uv, w, cfl=0.5) -> float:
    """dt at the given CFL number of the faster of the horizontal (|u| dt / dx)
    and vertical (|w| dt / dz) crossings on the uniform analytic grid."""
    dx = min(LX / (nx - 1), LY / (ny - 1))
    dz = MAX_DEPTH / (nl - 1)
    umax = float(np.sqrt(uv[0] ** 2 + uv[1] ** 2).max())
    wmax = float(np.abs(w).max())
    rate = max(umax / dx, wmax / dz)
    return cfl / rate if rate > 0.0 else 1.0


def layered_flow_case(api: FESOMTracerAdvection, nx: int, nl: int, ny: int | None = None, periodic=True, seed=0,
                      corr_cells: float | None = None) -> Case:
    """Build the mesh in ``api`` (init_analytic) and return the seeded inputs."""
    ny = nx if ny is None else ny
    corr = corr_cells if corr_cells is not None else max(4.0, max(nx, ny) / 25.0)
    K = synth_bathymetry_smooth(nx, ny, nl, periodic=periodic, corr_cells=corr, seed=seed)
    api.init_analytic(nx, ny, nl, Lx=LX, Ly=LY, max_depth=MAX_DEPTH, periodic=periodic, full_rings=True,
                      node_K=K, left_oriented=True)
    uv, w = api.synth_velocity(seed=seed + 1, umax=1.0, mode2=0.5, baro=1.0)
    T = api.synth_tracer(seed=seed + 2, kind=0)
    S = api.synth_tracer(seed=seed + 3, kind=1)
    nlev = api.mesh_array("nlevels_nod2D")
    wet = np.arange(nl - 1)[:, None] < (nlev[None, :] - 1)
    return Case(nx, ny, nl, periodic, K, uv, w, T, S, cfl_dt(api, nx, ny, nl, uv, w), int(wet.sum()), wet)


def ensemble_specs(members=8, seed=0, nx_range=(100, 800), nl_range=(20, 80)):
    """Seeded member meshes of the batched configuration: nx = ny drawn from
    nx_range, nl from nl_range, closed-wall and periodic alternating from a
    seeded coin."""
    rng = np.random.default_rng(seed)
    specs = []
    for m in range(members):
        specs.append({"nx": int(rng.integers(nx_range[0], nx_range[1] + 1)),
                      "nl": int(rng.integers(nl_range[0], nl_range[1] + 1)),
                      "periodic": bool(rng.integers(0, 2)), "seed": int(seed * 1000 + 17 * m + 1)})
    return specs


def build_ensemble(batch, api: FESOMTracerAdvection, specs, ntracers=48):
    """Adds one batch member per spec (mesh, velocity and ntracers seeded
    tracer fields, alternately temperature- and salinity-like); the single-mesh
    api builds each member's inputs.  Returns the per-member dt."""
    dts = []
    for s in specs:
        api.cleanup()
        c = layered_flow_case(api, s["nx"], s["nl"], periodic=s["periodic"], seed=s["seed"])
        m = batch.add_member(s["nx"], s["nx"], s["nl"], ntracers, periodic=s["periodic"], node_K=c.K)
        batch.set_velocity(m, c.uv, c.w)
        for t in range(1, ntracers + 1):
            batch.set_values(m, t, api.synth_tracer(seed=s["seed"] * 101 + t, kind=t % 2))
        dts.append(c.dt)
    api.cleanup()
    return dts
