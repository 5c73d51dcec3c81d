"""The domain decomposition's halo argument, checked on the CPU with the
oracle: every part's local mesh (owned nodes + 3 halo rings, built by the
library) is stepped by the oracle, the halo values are exchanged in numpy
after each step, and the owned values must equal the oracle's step of the
whole mesh bit for bit -- for irregular, seeded random partitions of an
analytic mesh with bathymetry and of the pi mesh."""
import math

import numpy as np
import pytest

import pyoracle
from fesom2_tracer_dwarf_b200 import _lib

FESOM2 = dict(angle_scale=math.pi / 180.0, cyclic_length=2.0 * math.pi)


def _arrays(api):
    d = api.mesh_dims()
    return d, {name: api.mesh_array(name) for name in pyoracle.OracleMesh.FROM_ARRAYS}


def _oracle_mesh(oracle, api, periodic, Lx, Ly):
    d, arr = _arrays(api)
    return pyoracle.OracleMesh.from_arrays(oracle, d["nl"], d["nod2D"], d["elem2D"], d["edge2D"], arr,
                                           periodic=periodic, Lx=Lx, Ly=Ly)


def _random_partition(edges, nod2D, nparts, seed):
    """Parts grown breadth-first from seeded random nodes over the edges."""
    rng = np.random.default_rng(seed)
    nb = [[] for _ in range(nod2D)]
    for a, b in edges:
        nb[a].append(b)
        nb[b].append(a)
    part = np.full(nod2D, -1, dtype=np.int32)
    fronts = []
    for q, s in enumerate(rng.choice(nod2D, nparts, replace=False)):
        part[s] = q
        fronts.append([int(s)])
    while any(fronts):
        for q in range(nparts):
            nxt = []
            for n in fronts[q]:
                for m in nb[n]:
                    if part[m] < 0:
                        part[m] = q
                        nxt.append(m)
            fronts[q] = nxt
    assert (part >= 0).all()
    return part


def _decomposed_run(api, oracle, rebuild, part, nparts, T, uv, w, dt, nsteps, sch, periodic, Lx, Ly, rings=3):
    parts = []
    for q in range(nparts):
        rebuild()
        dims = np.zeros(4, dtype=np.int32)
        _lib.check(api.lib, api.lib.tracer_partition_install_part(_lib.ptr(part), nparts, q, rings, _lib.ptr(dims)),
                   "tracer_partition_install_part")
        nodes = np.zeros(dims[1], dtype=np.int32)
        elems = np.zeros(dims[2], dtype=np.int32)
        _lib.check(api.lib, api.lib.tracer_partition_part_ids(_lib.ptr(nodes), _lib.ptr(elems)),
                   "tracer_partition_part_ids")
        nodes, elems = nodes - 1, elems - 1
        m = _oracle_mesh(oracle, api, periodic, Lx, Ly)
        parts.append({"m": m, "nodes": nodes, "owned": int(dims[0]), "T": np.asfortranarray(T[:, nodes]),
                      "uv": np.asfortranarray(uv[:, :, elems]), "w": np.asfortranarray(w[:, nodes])})
    G = np.array(T, order="F")
    for _ in range(nsteps):
        for p in parts:
            p["m"].step(p["T"], p["T"].copy(order="F"), p["uv"], p["w"], dt, *sch)
        for p in parts:  # owners publish
            G[:, p["nodes"][:p["owned"]]] = p["T"][:, :p["owned"]]
        for p in parts:  # halos refreshed
            p["T"][:, p["owned"]:] = G[:, p["nodes"][p["owned"]:]]
    return G


def test_oracle_from_library_arrays_steps_like_the_analytic_oracle(api, oracle):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    nx, ny, nl = 19, 15, 7
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, 1), nl, 4)
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    uv, w = api.synth_velocity(seed=5, umax=1.0, mode2=0.5)
    T = api.synth_tracer(seed=6, kind=0)
    a = pyoracle.OracleMesh(oracle, nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    b = _oracle_mesh(oracle, api, True, 1.0e5, 1.0e5)
    Ta, Tb = T.copy(order="F"), T.copy(order="F")
    for _ in range(3):
        a.step(Ta, Ta.copy(order="F"), uv, w, 0.5 * 1.0e5 / (nx - 1), "MUSCL", "PPM", "FCT")
        b.step(Tb, Tb.copy(order="F"), uv, w, 0.5 * 1.0e5 / (nx - 1), "MUSCL", "PPM", "FCT")
    assert np.array_equal(Ta.view(np.int64), Tb.view(np.int64))


@pytest.mark.parametrize("nparts,seed", [(3, 1), (5, 2)])
def test_random_partitions_of_an_analytic_mesh(api, oracle, nparts, seed):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    nx, ny, nl = 26, 22, 8
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, 1), nl, 7)

    def rebuild():
        api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)

    rebuild()
    uv, w = api.synth_velocity(seed=8, umax=1.0, mode2=0.5)
    T = api.synth_tracer(seed=9, kind=0)
    dt = 0.5 * 1.0e5 / (nx - 1)
    sch = ("MUSCL", "PPM", "FCT")
    d, garr = _arrays(api)
    whole = _oracle_mesh(oracle, api, True, 1.0e5, 1.0e5)
    Tg = T.copy(order="F")
    for _ in range(4):
        whole.step(Tg, Tg.copy(order="F"), uv, w, dt, *sch)
    edges = garr["edges"].reshape(-1, 2) - 1
    part = _random_partition(edges, d["nod2D"], nparts, seed)
    G = _decomposed_run(api, oracle, rebuild, part, nparts, T, uv, w, dt, 4, sch, True, 1.0e5, 1.0e5)
    assert np.array_equal(G.view(np.int64), Tg.view(np.int64))


@pytest.mark.parametrize("sch", [("MUSCL", "PPM", "FCT"), ("MFCT", "QR4C", "FCT")])
def test_random_partition_of_the_pi_mesh(api, oracle, pi_mesh_dir, sch):
    def rebuild():
        api.load_mesh_from_files(pi_mesh_dir, **FESOM2)

    rebuild()
    uv, w = api.synth_velocity(seed=3, umax=0.5, mode2=0.5)
    T = api.synth_tracer(seed=4, kind=0)
    dt = 300.0
    d, garr = _arrays(api)
    whole = _oracle_mesh(oracle, api, False, 0.0, 0.0)
    Tg = T.copy(order="F")
    for _ in range(3):
        whole.step(Tg, Tg.copy(order="F"), uv, w, dt, *sch)
    edges = garr["edges"].reshape(-1, 2) - 1
    part = _random_partition(edges, d["nod2D"], 6, 11)
    G = _decomposed_run(api, oracle, rebuild, part, 6, T, uv, w, dt, 3, sch, False, 0.0, 0.0)
    assert np.array_equal(G.view(np.int64), Tg.view(np.int64))


def test_two_halo_rings_are_not_enough(api, oracle):
    """Control: with two rings the FCT ratios of the owned nodes' neighbours
    read bounds the part cannot compute, and the owned values differ."""
    nx, ny, nl = 22, 18, 7

    def rebuild():
        api.init_analytic(nx, ny, nl, periodic=True, full_rings=True)

    rebuild()
    uv, w = api.synth_velocity(seed=8, umax=1.0, mode2=0.5)
    T = api.synth_tracer(seed=9, kind=0)
    dt = 0.5 * 1.0e5 / (nx - 1)
    sch = ("MUSCL", "PPM", "FCT")
    d, garr = _arrays(api)
    whole = _oracle_mesh(oracle, api, True, 1.0e5, 1.0e5)
    Tg = T.copy(order="F")
    for _ in range(3):
        whole.step(Tg, Tg.copy(order="F"), uv, w, dt, *sch)
    part = _random_partition(garr["edges"].reshape(-1, 2) - 1, d["nod2D"], 3, 1)
    G3 = _decomposed_run(api, oracle, rebuild, part, 3, T, uv, w, dt, 3, sch, True, 1.0e5, 1.0e5, rings=3)
    G2 = _decomposed_run(api, oracle, rebuild, part, 3, T, uv, w, dt, 3, sch, True, 1.0e5, 1.0e5, rings=2)
    assert np.array_equal(G3.view(np.int64), Tg.view(np.int64))
    assert not np.array_equal(G2.view(np.int64), Tg.view(np.int64))
