"""The reference's own Python scripts run against this library, on the CPU.

Each test loads the reference's script from its source tree (present where
the reference is checked out beside the repository; skipped elsewhere),
repoints its library path at libfesom_tracer.so and runs the script's own
functions unchanged:
  * python/verify_c_interface.py: verify_library, verify_functions (its list
    of the C symbols) and demonstrate_usage (its call sequence: MPI init,
    mesh dims, partition, allocate tracers, set values, zero velocity);
  * python/demo_tracer.py: the FESOMTracerAdvection class reads a restart
    the library wrote (initialize, get_tracer_values, get_statistics,
    finalize) -- the steps of its main() need the GPU;
  * visualization/plot_scalars.py: load_mesh and load_scalars read the
    library's mesh and scalar output files.
"""
import os
import sys
import types
from pathlib import Path

import numpy as np
import pytest

REF = Path(os.environ.get("FESOM_REFERENCE_TREE", "/root/reference"))
pytestmark = pytest.mark.skipif(not (REF / "python" / "demo_tracer.py").exists(),
                                reason="the reference source tree is not present")


def load_script(path: Path, module_file: Path, name: str):
    """Executes a reference script's source as a module whose __file__ is
    module_file (so its relative library path resolves beside it)."""
    mod = types.ModuleType(name)
    mod.__file__ = str(module_file)
    code = compile(path.read_text(), str(path), "exec")
    exec(code, mod.__dict__)
    return mod


def test_verify_c_interface_script(lib, tmp_path, capsys):
    from fesom2_tracer_dwarf_b200 import _lib
    mod = load_script(REF / "python" / "verify_c_interface.py", tmp_path / "verify_c_interface.py", "ref_verify")
    mod.LIB_PATH = Path(_lib.LIB_PATH)
    rlib = mod.verify_library()
    assert rlib is not None
    assert mod.verify_functions(rlib)
    assert lib.tracer_cleanup() == 0
    assert mod.demonstrate_usage(rlib)
    assert lib.tracer_cleanup() == 0


def _write_state(api, tmp_path):
    """A 12x10x7 periodic analytic mesh with bathymetry, two tracers with
    different schemes and separate valuesAB, a flow; written as a restart."""
    from fesom2_tracer_dwarf_b200 import synth_bathymetry
    nx, ny, nl = 12, 10, 7
    K = synth_bathymetry(api.lib.tracer_analytic_nodes(nx, ny, 1), nl, 3)
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, node_K=K)
    uv, w = api.synth_velocity(seed=4, umax=0.5, mode2=0.5)
    T = api.synth_tracer(seed=5, kind=0)
    S = api.synth_tracer(seed=6, kind=1)
    api.allocate_tracers(2)
    api.set_values(1, T, T + 0.25)
    api.set_values(2, S)
    api.set_scheme(1, "MUSCL", "PPM", "FCT", 0.75, 1.0)
    api.set_scheme(2, "MFCT", "QR4C", "NONE", 1.0, 0.5)
    api.set_velocity(uv, w)
    mesh = {k: api.mesh_array(k) for k in ("elem2D_nodes", "edges", "edge_tri", "nlevels", "nlevels_nod2D",
                                           "area", "areasvol", "hnode", "hnode_new", "helem", "gradient_sca",
                                           "edge_cross_dxdy", "edge_dxdy", "elem_area", "zbar",
                                           "edge_up_dn_tri", "nboundary_lay")}
    out = tmp_path / "fesom_bin_restart"
    assert api.lib.tracer_finalize(str(out).encode()) == 0, api.lib.tracer_last_error()
    return out, mesh, T, S, uv, w


def read_record(path):
    """gfortran sequential record framing: the concatenated payload of one
    logical record (leading marker negative while more subrecords follow)."""
    raw = path.read_bytes()
    pos, out = 0, b""
    while True:
        lead = int.from_bytes(raw[pos:pos + 4], "little", signed=True)
        n = abs(lead)
        out += raw[pos + 4:pos + 4 + n]
        tail = int.from_bytes(raw[pos + 4 + n:pos + 8 + n], "little", signed=True)
        assert abs(tail) == n
        pos += 8 + n
        if lead >= 0:
            break
    assert pos == len(raw)
    return out


def test_restart_files_and_round_trip(api, tmp_path):
    out, mesh, T, S, uv, w = _write_state(api, tmp_path)
    np1 = out / "np1"
    assert sorted(p.name for p in np1.iterdir()) == ["t_dynamics.0", "t_mesh.0", "t_partit.0", "t_tracer.0"]
    assert (out / "meta.time").read_text().splitlines()[:3] == ["0", "0", "! year: 0"]
    # the tracer record read field by field (lib/MOD_TRACER.F90:104-206)
    rec = read_record(np1 / "t_tracer.0")
    L, N = T.shape
    i4 = lambda o: int.from_bytes(rec[o:o + 4], "little", signed=True)
    assert i4(0) == 2
    assert (i4(4), i4(8)) == (L, N)
    vals = np.frombuffer(rec[12:12 + 8 * L * N], dtype=np.float64).reshape((L, N), order="F")
    assert np.array_equal(vals, T)
    o = 12 + 8 * L * N
    assert (i4(o), i4(o + 4), i4(o + 8)) == (0, 0, 0)  # valuesold unallocated
    o += 12
    assert (i4(o), i4(o + 4)) == (L, N)
    ab = np.frombuffer(rec[o + 8:o + 8 + 8 * L * N], dtype=np.float64).reshape((L, N), order="F")
    assert np.array_equal(ab, T + 0.25)
    o += 8 + 8 * L * N + 4 + 24 + 4  # smooth_bh_tra, gamma0..2, i_vert_diff
    assert rec[o:o + 60].decode() == "MUSCL".ljust(20) + "PPM".ljust(20) + "FCT".ljust(20)
    assert np.frombuffer(rec[o + 60:o + 76], dtype=np.float64).tolist() == [0.75, 1.0]
    assert i4(o + 76) == 1

    api.cleanup()
    assert api.lib.tracer_init(str(out).encode()) == 0, api.lib.tracer_last_error()
    for k, v in mesh.items():
        assert np.array_equal(api.mesh_array(k), v), k
    assert np.array_equal(api.get_tracer_values(1), T)
    assert np.array_equal(api.get_tracer_values(2), S)
    # a second write of the state read back gives the same files
    out2 = tmp_path / "again"
    assert api.lib.tracer_finalize(str(out2).encode()) == 0
    for f in ("t_mesh.0", "t_partit.0", "t_tracer.0", "t_dynamics.0"):
        assert (out / "np1" / f).read_bytes() == (out2 / "np1" / f).read_bytes(), f


def test_restart_errors(api, tmp_path):
    assert api.lib.tracer_init(str(tmp_path / "missing").encode()) == -1
    assert b"could not find restart directory" in api.lib.tracer_last_error()
    out, *_ = _write_state(api, tmp_path)
    api.cleanup()
    bad = out / "np1" / "t_tracer.0"
    bad.write_bytes(bad.read_bytes()[:100])
    assert api.lib.tracer_init(str(out).encode()) == -1
    assert b"t_tracer.0" in api.lib.tracer_last_error()
    assert api.lib.tracer_finalize(str(tmp_path / "x").encode()) == -1  # not initialised


def test_load_mesh_partition(api, tmp_path):
    out, mesh, *_ = _write_state(api, tmp_path)
    api.cleanup()
    assert api.lib.tracer_load_mesh_partition(str(out).encode()) == 0, api.lib.tracer_last_error()
    for k in ("elem2D_nodes", "edges", "nlevels_nod2D", "edge_up_dn_tri", "nboundary_lay", "hnode"):
        assert np.array_equal(api.mesh_array(k), mesh[k]), k


def test_demo_tracer_class_reads_the_librarys_restart(api, tmp_path, capsys):
    out, mesh, T, S, uv, w = _write_state(api, tmp_path)
    api.cleanup()
    from fesom2_tracer_dwarf_b200 import _lib
    libdir = tmp_path / "demo" / "lib"
    libdir.mkdir(parents=True)
    (libdir / "libfesom_tracer_Fortran.so").symlink_to(Path(_lib.LIB_PATH).resolve())
    mod = load_script(REF / "python" / "demo_tracer.py", tmp_path / "demo" / "demo_tracer.py", "ref_demo")
    tr = mod.FESOMTracerAdvection()
    assert tr.initialize_mpi(0) == 0
    assert tr.initialize(str(out)) == 0
    v = tr.get_tracer_values()
    assert np.array_equal(v, T)
    st = tr.get_statistics()
    assert st["min"] == T.min() and st["max"] == T.max() and abs(st["sum"] - T.sum()) <= 1e-12 * abs(T.sum())
    out2 = tmp_path / "written_by_demo"
    assert tr.finalize(str(out2)) == 0
    assert tr.finalize_mpi() == 0
    assert (out2 / "np1" / "t_tracer.0").read_bytes() == (out / "np1" / "t_tracer.0").read_bytes()


def test_reference_shaped_set_velocity_with_edge_count_is_rejected(api):
    """tracer_set_velocity(uv, w, nl, nod2D, edge2D) as the reference's
    array path calls it: uv sized by EDGES is refused with a message, not
    misread."""
    api.init_analytic(8, 7, 5, periodic=True)
    d = api.mesh_dims()
    nl, N, E = d["nl"], d["nod2D"], d["edge2D"]
    uv = np.zeros((nl - 1, E, 2), order="F")
    w = np.zeros((nl, N), order="F")
    assert api.lib.tracer_set_velocity(uv.ctypes.data, w.ctypes.data, nl, N, E) == -1
    assert b"elem2D" in api.lib.tracer_last_error()


def test_plot_scalars_readers(api, tmp_path):
    """visualization/plot_scalars.py's load_mesh / load_scalars read the
    library's output files (lib/mesh_output.F90:19-161 layouts)."""
    mod = load_script(REF / "visualization" / "plot_scalars.py", tmp_path / "plot_scalars.py", "ref_plot")
    nx, ny, nl = 9, 7, 6
    api.init_analytic(nx, ny, nl, periodic=True, full_rings=True, max_depth=800.0)
    T, S, uv, w = api.analytic_fields()
    api.allocate_tracers(2)
    api.set_values(1, T)
    api.set_values(2, S)
    api.write_mesh(tmp_path)
    api.open_scalar_output(tmp_path, 1)
    api.write_scalar_step()
    api.set_values(1, T + 2.0)
    api.write_scalar_step()
    api.close_scalar_output()
    x, y, tri, zbar, depth = mod.load_mesh(str(tmp_path))
    d = api.mesh_dims()
    assert x.shape == (d["nod2D"],) and tri.shape == (d["elem2D"], 3)
    assert np.array_equal(tri.ravel(), api.mesh_array("elem2D_nodes") - 1)
    assert np.allclose(zbar, -np.arange(nl) * 800.0 / (nl - 1))
    info, data = mod.load_scalars(str(tmp_path))
    assert info["nod2D"] == d["nod2D"] and info["nsteps"] == 1 and info["num_tracers"] == 2
    temp = data[info["tracer_names"][0]]
    assert np.array_equal(temp[0], T.T) and np.array_equal(temp[1], (T + 2.0).T)
