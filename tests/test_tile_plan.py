"""The fused kernel's patch plan, built and checked on the host (no GPU):
every node owned by exactly one patch, three halo rings around each patch,
incidence lists in ascending edge id with the right far node, flags and
levels, every edge of an N1 node in E1, up/down triangles and element rings
inside the patch, and every region small enough for one thread block."""
import numpy as np
import pytest


def plan(api, max_owned):
    out = np.zeros(8)
    rc = api.lib.tracer_tile_plan_check(max_owned, out.ctypes.data)
    assert rc == 0, api.lib.tracer_last_error()
    return dict(zip(["patches", "min_owned", "max_n2", "max_n3", "max_e2", "max_el", "node_ratio", "edge_ratio"],
                    out.tolist()))


@pytest.mark.parametrize("nx,ny,periodic,full", [(20, 20, True, False), (33, 27, True, True), (19, 24, False, True)])
def test_analytic_plans(api, nx, ny, periodic, full):
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, int(periodic)), 12, 5)
    api.init_analytic(nx, ny, 12, periodic=periodic, full_rings=full, node_K=K)
    for owned in (1, 7, 60, 225, 10000):
        p = plan(api, owned)
        assert p["max_n2"] <= 384 and p["max_n3"] - 0 <= 768
        assert p["patches"] >= 1


def test_large_analytic_plan_redundancy(api):
    """At 300x300 the patches are about 15x15 owned nodes: the regions fit
    the block and the halo work stays near (17^2)/15^2 edges and (19^2)/15^2
    LO nodes per owned node."""
    api.init_analytic(300, 300, 5, periodic=True, full_rings=True)
    p = plan(api, 225)
    assert 380 < p["patches"] < 420
    assert p["max_n2"] <= 384
    assert p["node_ratio"] < 1.75 and p["edge_ratio"] < 1.45


def test_pi_mesh_plan(api, pi_mesh_dir):
    """The irregular pi mesh (valence 2-8, coastlines): regions that would
    not fit are split until they do."""
    assert api.lib.tracer_load_mesh_from_files(str(pi_mesh_dir).encode()) == 0
    for owned in (50, 225, 1000):
        p = plan(api, owned)
        assert p["max_n2"] <= 384
