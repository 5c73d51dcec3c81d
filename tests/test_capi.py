"""The C ABI: exports, the reference's symbol list, and its error handling.
Nothing here launches a kernel."""
import ctypes
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "fesom_tracer.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9 ]+?\s*\*?\s*(tracer_[a-z_0-9]+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n


def test_reference_symbol_list(lib):
    """The 20 names python/verify_c_interface.py:68-95 checks, plus the three
    mesh-loading calls of lib/tracer_c_interface.F90."""
    from fesom2_tracer_dwarf_b200 import REFERENCE_SYMBOLS
    assert len(REFERENCE_SYMBOLS) == 23
    for n in REFERENCE_SYMBOLS:
        assert hasattr(lib, n), n


def test_bindings_cover_header(lib):
    from fesom2_tracer_dwarf_b200._lib import SIGNATURES
    assert set(header_functions()) == set(SIGNATURES)


def test_uninitialised_calls_fail(api):
    lib = api.lib
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    assert lib.tracer_get_stats(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)) == -1
    nz, nn = ctypes.c_int(), ctypes.c_int()
    assert lib.tracer_get_size(ctypes.byref(nz), ctypes.byref(nn)) == -1
    assert lib.tracer_advect_step(1.0) == -1
    assert lib.tracer_init_ale_arrays() == -1
    assert lib.tracer_init_for_advection() == -1


def test_unsupported_inputs_fail(api):
    lib = api.lib
    assert lib.tracer_init_mpi(0) == 0
    assert lib.tracer_finalize_mpi() == 0
    assert lib.tracer_init(b"/nonexistent") == -1
    assert lib.tracer_finalize(b"/nonexistent") == -1
    assert lib.tracer_run_workflow(b"/nonexistent", 3, 1.0) == -1
    assert lib.tracer_load_mesh_partition(b"/nonexistent") == -1
    assert lib.tracer_load_mesh_from_files(b"/nonexistent") == -1
    assert lib.tracer_last_error()


def test_array_path_validation(api):
    """Call order of docs/INTERFACES.md:83-95 with bad inputs."""
    lib = api.lib
    assert lib.tracer_set_mesh_dims(10, 5, 8, 4) == 0
    nlev = np.full(5, 9, dtype=np.int32)
    ulev = np.ones(5, dtype=np.int32)
    P = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    assert lib.tracer_set_levels(P(nlev), P(ulev), 5) == 0
    ulev[2] = 2
    assert lib.tracer_set_levels(P(nlev), P(ulev), 5) == -1  # cavities
    assert lib.tracer_set_partition(5, 3) == -1              # halo nodes
    assert lib.tracer_set_partition(5, 0) == 0
    assert lib.tracer_allocate_tracers(2, 10, 5, 2) == 0
    v = np.ones((9, 5), order="F")
    assert lib.tracer_set_values(3, P(v), 10, 5) == -1       # bad tracer id
    assert lib.tracer_set_values(1, P(v), 10, 6) == -1       # bad dims
    assert lib.tracer_set_values(1, P(v), 10, 5) == 0
    assert lib.tracer_init_complete() == 0
    s = np.zeros(4)
    assert lib.tracer_get_stats_id(1, P(s)) == 0 and s[0] == 1.0 and s[2] == 45.0
    # advection needs connectivity (docs/INTERFACES.md:197)
    assert lib.tracer_advect_step(1.0) == -1
    assert lib.tracer_set_scheme(1, b"MUSCL", b"PPM", b"FCT", 1.0, 1.0) == 0
    assert lib.tracer_set_scheme(1, b"QUICK", b"PPM", b"FCT", 1.0, 1.0) == -1


def test_analytic_init_without_gpu_work(api):
    api.init_analytic(20, 20, 10, periodic=True, full_rings=False)
    d = api.mesh_dims()
    assert (d["nl"], d["nod2D"], d["elem2D"], d["edge2D"]) == (10, 361, 722, 1083)
    assert d["level_stride"] == 12
    T, S, uv, w = api.analytic_fields()
    assert T.shape == (9, 361) and uv.shape == (2, 9, 722)
    assert abs(T.sum() - 32490.0) < 1e-9
    nz, nn = ctypes.c_int(), ctypes.c_int()
    assert api.lib.tracer_get_size(ctypes.byref(nz), ctypes.byref(nn)) == 0
    assert (nz.value, nn.value) == (9, 361)
