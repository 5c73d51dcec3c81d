"""The ASCII mesh reader (tracer_load_mesh_from_files) on the reference's pi
mesh: the library's host mesh against the oracle's independent restatement of
mesh_setup (lib/oce_mesh.F90:49-94), bit for bit, in the reference's
conventions and in FESOM2's; geometric sanity; error handling.  CPU only."""
import math
import shutil

import numpy as np
import pytest

R_EARTH = 6367500.0
FESOM2 = dict(angle_scale=math.pi / 180.0, cyclic_length=2.0 * math.pi)

ARRAYS = ["coord", "elem2D_nodes", "edges", "edge_tri", "nlevels", "nlevels_nod2D", "elem_area", "area", "areasvol",
          "edge_dxdy", "edge_cross_dxdy", "gradient_sca", "elem_cos", "edge_up_dn_tri", "nboundary_lay", "hnode",
          "helem", "zbar"]


def _bits(a):
    a = np.asarray(a)
    return a.view(np.int64) if a.dtype == np.float64 else a


@pytest.mark.parametrize("conv", ["reference", "fesom2"])
def test_reader_matches_oracle_bitwise(api, oracle, pi_mesh_dir, conv):
    import pyoracle
    kw = {} if conv == "reference" else FESOM2
    api.load_mesh_from_files(pi_mesh_dir, **kw)
    m = pyoracle.OracleMesh.from_files(oracle, pi_mesh_dir, **kw)
    d = api.mesh_dims()
    assert (d["nl"], d["nod2D"], d["elem2D"], d["edge2D"]) == (48, 3140, 5839, 8986)
    assert (m.nl, m.nod2D, m.elem2D, m.edge2D) == (48, 3140, 5839, 8986)
    for name in ARRAYS:
        a, b = api.mesh_array(name), m.array(name)
        assert a.size == b.size, name
        assert np.array_equal(_bits(a), _bits(b)), name


def test_fesom2_conventions_give_the_ocean_area(api, pi_mesh_dir):
    """With angles in degrees and the longitude wrapped at the seam, every
    element is a small positive spherical triangle and the surface areas add
    up to the pi mesh's ocean (two thirds of the sphere); the edge cross
    vectors are shorter than the largest element."""
    api.load_mesh_from_files(pi_mesh_dir, **FESOM2)
    ea = api.mesh_array("elem_area")
    sphere = 4.0 * math.pi * R_EARTH ** 2
    assert ea.min() > 0.0 and ea.max() < 2e-3 * sphere
    assert 0.6 < ea.sum() / sphere < 0.72
    area = api.mesh_array("area").reshape(-1, 48)  # (nod2D, nl) in Fortran order
    assert abs(area[:, 0].sum() - ea.sum()) < 1e-9 * ea.sum()
    cos = api.mesh_array("elem_cos")
    assert cos.min() > 0.0 and cos.max() <= 1.0 and cos.min() < 0.5  # elem_cos != 1 on a sphere
    cross = np.abs(api.mesh_array("edge_cross_dxdy"))
    assert cross.max() < math.sqrt(ea.max()) * 2.0
    # element rings have irregular valence
    ring = api.mesh_array("ring_num")
    assert ring.min() < 6 < ring.max()


def test_reference_conventions_reproduce_the_seam_elements(api, pi_mesh_dir):
    """The reference's cyclic_length (360) never trims differences of
    coordinates in radians, so elements straddling the longitude seam keep
    their unwrapped width, as its mesh_areas computes them; elsewhere the two
    conventions differ only through the rotation."""
    api.load_mesh_from_files(pi_mesh_dir)
    ea = api.mesh_array("elem_area")
    assert ea.min() > 0.0
    assert ea.max() > 100.0 * np.median(ea)
    coord = api.mesh_array("coord").reshape(-1, 2)
    en = api.mesh_array("elem2D_nodes").reshape(-1, 3) - 1
    span = np.ptp(coord[en, 0], axis=1)
    seam = span > math.pi
    assert seam.any()
    assert np.median(ea[seam]) > 50.0 * np.median(ea[~seam])


def test_unrotated_request_is_refused_like_the_reference(api, pi_mesh_dir):
    """rotate = 0 on a mesh with no ocean next to the rotated pole is the
    reference's 'mesh seems to be unrotated' error (lib/oce_mesh.F90:312-330)."""
    with pytest.raises(RuntimeError, match="unrotated"):
        api.load_mesh_from_files(pi_mesh_dir, rotate=False)


@pytest.mark.parametrize("damage", ["missing", "truncated", "bad_index"])
def test_malformed_mesh_directory_fails_cleanly(api, pi_mesh_dir, tmp_path, damage):
    d = tmp_path / "mesh"
    shutil.copytree(pi_mesh_dir, d)
    if damage == "missing":
        (d / "edge_tri.out").unlink()
        what = "edge_tri.out"
    elif damage == "truncated":
        text = (d / "elem2d.out").read_text().splitlines()
        (d / "elem2d.out").write_text("\n".join(text[: len(text) // 2]) + "\n")
        what = "elem2d.out"
    else:
        text = (d / "edges.out").read_text().splitlines()
        text[5] = "  1  999999"
        (d / "edges.out").write_text("\n".join(text) + "\n")
        what = "edges.out"
    with pytest.raises(RuntimeError, match=what):
        api.load_mesh_from_files(d)
    # the library stays usable
    api.load_mesh_from_files(pi_mesh_dir)
    assert api.mesh_dims()["nod2D"] == 3140


def test_synthetic_flow_keeps_constants_on_stretched_layers(api, oracle, pi_mesh_dir):
    """The seeded layered flow's vertical modes have zero thickness-weighted
    column mean, so w from the discrete continuity closes at the surface even
    on the pi mesh's 5 m to 250 m layers: a constant stays constant under the
    oracle's MUSCL/PPM/FCT step (and the content is conserved)."""
    import pyoracle
    api.load_mesh_from_files(pi_mesh_dir, **FESOM2)
    uv, w = api.synth_velocity(seed=5, umax=0.5, mode2=0.5)
    m = pyoracle.OracleMesh.from_files(oracle, pi_mesh_dir, **FESOM2)
    nlev = api.mesh_array("nlevels_nod2D")
    wet = np.arange(47)[:, None] < (nlev[None, :] - 1)
    C = np.asfortranarray(np.where(wet, 7.25, 0.0))
    for _ in range(5):
        m.step(C, C.copy(order="F"), uv, w, 600.0, "MUSCL", "PPM", "FCT")
    assert np.max(np.abs(C[wet] - 7.25)) < 1e-12
