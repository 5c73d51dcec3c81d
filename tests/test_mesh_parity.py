"""The product's host mesh builder (csrc/mesh.cpp) against the oracle's
restatement of lib/analytic_mesh.F90 + lib/oce_mesh.F90: every array the
advection step reads must be bit-identical."""
import numpy as np
import pytest

import pyoracle

CASES = [
    # nx, ny, nl, periodic, full_rings, bathymetry seed (None = flat), left-oriented
    (15, 12, 7, True, True, 8, True),
    (9, 11, 5, False, True, 9, True),
    (20, 20, 10, True, False, None, False),
    (20, 20, 10, True, True, None, False),
    (9, 7, 6, False, True, None, False),
    (17, 13, 9, True, True, 4, False),
    (11, 15, 8, False, True, 6, False),
    (6, 5, 4, True, False, None, False),
]

FIELDS_D = ["coord", "elem_area", "area", "areasvol", "edge_dxdy", "edge_cross_dxdy", "gradient_sca", "hnode",
            "hnode_new", "helem", "zbar"]
FIELDS_I = ["elem2D_nodes", "edges", "edge_tri", "nlevels", "nlevels_nod2D", "nlevels_nod2D_min",
            "edge_up_dn_tri", "nboundary_lay"]


@pytest.mark.parametrize("nx,ny,nl,periodic,full,seed,left", CASES)
def test_mesh_bitwise(oracle, api, nx, ny, nl, periodic, full, seed, left):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    K = None
    if seed is not None:
        K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, int(periodic)), nl, seed)
    api.init_analytic(nx, ny, nl, periodic=periodic, full_rings=full, node_K=K, left_oriented=left)
    m = pyoracle.OracleMesh(oracle, nx, ny, nl, periodic=periodic, full_rings=full, node_K=K, left_oriented=left)
    d = api.mesh_dims()
    assert (d["nl"], d["nod2D"], d["elem2D"], d["edge2D"]) == (m.nl, m.nod2D, m.elem2D, m.edge2D)
    for name in FIELDS_I + FIELDS_D:
        a = api.mesh_array(name)
        b = m.array(name)
        if name in ("area", "areasvol"):
            b = b[: m.nl * m.nod2D]
        assert a.shape == b.shape, name
        if a.dtype.kind == "f":
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name
        else:
            assert np.array_equal(a, b), name
    # element rings (nod_in_elem2D), same members in the same order
    num = api.mesh_array("ring_num")
    onum = m.array("nod_in_elem2D_num")[: m.nod2D]
    assert np.array_equal(num, onum)


def test_up_down_triangles_found_on_periodic_mesh(api):
    """With the minimum-image wrap nearly every edge of the periodic mesh finds
    both its upwind and downwind triangles (the reference's cyclic_length trim
    never fires on a Cartesian mesh, lib/oce_muscl_adv.F90:248-249)."""
    api.init_analytic(40, 40, 5, periodic=True, full_rings=True)
    ud = api.mesh_array("edge_up_dn_tri")
    assert (ud == 0).mean() < 0.01


def test_bathymetry_levels(api):
    """Element levels are the minimum of their nodes' K, node levels the
    maximum over the ring; every wet node layer has positive area."""
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    nx = ny = 21
    nl = 12
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, 1), nl, 0)
    assert K.min() >= 3 and K.max() <= nl
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    en = api.mesh_array("elem2D_nodes").reshape(3, -1, order="F") - 1
    lv = api.mesh_array("nlevels")
    assert np.array_equal(lv, K[en].min(axis=0))
    nlev = api.mesh_array("nlevels_nod2D")
    area = api.mesh_array("area").reshape(nl, -1, order="F")
    for n in range(0, nlev.size, 7):
        assert np.all(area[: nlev[n] - 1, n] > 0)
        assert np.all(area[nlev[n] - 1:, n] == 0)
