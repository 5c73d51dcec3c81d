"""Raw binary output for the reference's plotting scripts
(lib/mesh_output.F90:19-161, read by visualization/plot_mesh.py and
plot_scalars.py): files, shapes and values as those readers take them."""
import numpy as np


def _info(path):
    out = {}
    for line in open(path):
        k, v = line.strip().split("=", 1)
        out[k] = v
    return out


def test_mesh_and_scalar_files(api, tmp_path):
    nx, ny, nl = 9, 7, 6
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, max_depth=800.0)
    T, S, uv, w = api.analytic_fields()
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    api.write_mesh(tmp_path)
    d = api.mesh_dims()
    info = _info(tmp_path / "mesh_info.txt")
    assert (int(info["nod2D"]), int(info["elem2D"]), int(info["nl"])) == (d["nod2D"], d["elem2D"], nl)
    xy = np.fromfile(tmp_path / "coord_nod2D.bin", dtype=np.float64).reshape((2, d["nod2D"]), order="F")
    assert np.allclose(xy, api.mesh_array("coord").reshape(2, -1, order="F") * 6367500.0)
    tri = np.fromfile(tmp_path / "elem2D_nodes.bin", dtype=np.int32).reshape((3, d["elem2D"]), order="F").T
    assert np.array_equal(tri.T.ravel(order="F"), api.mesh_array("elem2D_nodes") - 1)
    assert np.allclose(np.fromfile(tmp_path / "zbar.bin", dtype=np.float64), -np.arange(nl) * 800.0 / (nl - 1))
    assert np.allclose(np.fromfile(tmp_path / "depth.bin", dtype=np.float64), -800.0)  # flat analytic bottom

    api.open_scalar_output(tmp_path, 2)
    api.write_scalar_step()
    api.set_values(1, T + 1.0)
    api.write_scalar_step()
    api.write_scalar_step()
    api.close_scalar_output()
    sinfo = _info(tmp_path / "scalar_info.txt")
    assert sinfo["tracer_1"] == "temperature" and sinfo["tracer_2"] == "salinity" and sinfo["wp"] == "8"
    nz, nn = int(sinfo["nz"]), int(sinfo["nod2D"])
    frames = np.fromfile(tmp_path / "temperature.bin", dtype=np.float64).reshape((3, nn, nz))
    assert np.array_equal(frames[0].T, T) and np.array_equal(frames[1].T, T + 1.0)
    sal = np.fromfile(tmp_path / "salinity.bin", dtype=np.float64).reshape((3, nn, nz))
    assert np.array_equal(sal[2].T, S)
