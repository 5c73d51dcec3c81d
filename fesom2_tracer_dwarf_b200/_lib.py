"""ctypes bindings of lib/libfesom_tracer.so (declared in include/fesom_tracer.h).

The library is built in-tree (``make -C fesom2_tracer_dwarf_b200``); loading
fails loudly when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("FESOM_TRACER_LIB", PKG_DIR / "lib" / "libfesom_tracer.so"))

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_double_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); pointers are passed as void* so numpy buffers
# (any layout already validated by the caller) go straight through.
SIGNATURES = {
    # reference interface, lib/tracer_c_interface.F90
    "tracer_init_mpi": (ctypes.c_int, [ctypes.c_int]),
    "tracer_finalize_mpi": (ctypes.c_int, []),
    "tracer_init": (ctypes.c_int, [ctypes.c_char_p]),
    "tracer_advect_step": (ctypes.c_int, [ctypes.c_double]),
    "tracer_get_stats": (ctypes.c_int, [_c_double_p, _c_double_p, _c_double_p]),
    "tracer_get_size": (ctypes.c_int, [_c_int_p, _c_int_p]),
    "tracer_get_values": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "tracer_finalize": (ctypes.c_int, [ctypes.c_char_p]),
    "tracer_run_workflow": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_double]),
    "tracer_cleanup": (ctypes.c_int, []),
    "tracer_set_mesh_dims": (ctypes.c_int, [ctypes.c_int] * 4),
    "tracer_set_levels": (ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    "tracer_set_thickness": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "tracer_set_partition": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "tracer_allocate_tracers": (ctypes.c_int, [ctypes.c_int] * 4),
    "tracer_set_values": (ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int]),
    "tracer_set_velocity_zero": (ctypes.c_int, [ctypes.c_int] * 3),
    "tracer_set_velocity": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "tracer_init_complete": (ctypes.c_int, []),
    "tracer_load_mesh_partition": (ctypes.c_int, [ctypes.c_char_p]),
    "tracer_load_mesh_from_files": (ctypes.c_int, [ctypes.c_char_p]),
    "tracer_load_mesh_from_files_opts": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_double,
                                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_double]),
    "tracer_init_ale_arrays": (ctypes.c_int, []),
    "tracer_init_for_advection": (ctypes.c_int, []),
    # extensions
    "tracer_init_analytic": (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int] * 2 + [_vp]),
    "tracer_analytic_nodes": (ctypes.c_int, [ctypes.c_int] * 3),
    "tracer_set_mesh_arrays": (ctypes.c_int, [ctypes.c_int] * 5 + [_vp] * 19 + [ctypes.c_double] * 2),
    "tracer_set_scheme": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                         ctypes.c_double, ctypes.c_double]),
    "tracer_set_velocity_elem": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "tracer_set_values_ab": (ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int]),
    "tracer_set_ab_refresh": (ctypes.c_int, [ctypes.c_int]),
    "tracer_set_precision": (ctypes.c_int, [ctypes.c_int]),
    "tracer_set_rounding": (ctypes.c_int, [ctypes.c_int]),
    "tracer_set_step_path": (ctypes.c_int, [ctypes.c_int]),
    "tracer_step_info": (ctypes.c_int, [_vp]),
    "tracer_set_patch_size": (ctypes.c_int, [ctypes.c_int]),
    "tracer_set_cells_per_block": (ctypes.c_int, [ctypes.c_int]),
    "tracer_set_nan_check": (ctypes.c_int, [ctypes.c_int]),
    "tracer_advect_step_io": (ctypes.c_int, [ctypes.c_double, _vp, _vp, ctypes.c_int]),
    "tracer_step_status": (ctypes.c_int, [_vp]),
    "tracer_tile_plan_check": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_host_register": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "tracer_host_unregister": (ctypes.c_int, [_vp]),
    "tracer_storage_offset": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_volume_sum": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_advect_steps": (ctypes.c_int, [ctypes.c_int, ctypes.c_double]),
    "tracer_get_values_id": (ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int]),
    "tracer_get_stats_id": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_analytic_fields": (ctypes.c_int, [_vp] * 4),
    "tracer_synth_bathymetry": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, _vp]),
    "tracer_synth_velocity": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, _vp, _vp]),
    "tracer_synth_bathymetry_smooth": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_double, ctypes.c_uint64, _vp]),
    "tracer_synth_tracer": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_int, _vp]),
    "tracer_mesh_dims": (ctypes.c_int, [_vp]),
    "tracer_mesh_len": (ctypes.c_long, [ctypes.c_char_p]),
    "tracer_mesh_get_int": (ctypes.c_int, [ctypes.c_char_p, _vp]),
    "tracer_mesh_get_dbl": (ctypes.c_int, [ctypes.c_char_p, _vp]),
    "tracer_time_steps": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_float)]),
    "tracer_profile_steps": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, _vp, _vp, ctypes.c_int, _c_int_p]),
    "tracer_set_device": (ctypes.c_int, [ctypes.c_int]),
    "tracer_launches_per_step": (ctypes.c_int, []),
    "tracer_device_bytes": (ctypes.c_longlong, []),
    "tracer_selftest_division": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_uint64, _vp, _vp]),
    "tracer_selftest_sround": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.c_uint32,
                                              ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double)]),
    "tracer_batch_create": (ctypes.c_int, []),
    "tracer_batch_destroy": (ctypes.c_int, []),
    "tracer_batch_add_member": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, _vp,
                                               ctypes.c_int]),
    "tracer_batch_member_dims": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_batch_set_velocity": (ctypes.c_int, [ctypes.c_int, _vp, _vp]),
    "tracer_batch_set_values": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp]),
    "tracer_batch_get_values": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp]),
    "tracer_batch_configure": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                              ctypes.c_double, _vp, ctypes.c_int]),
    "tracer_batch_set_tile": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "tracer_batch_get_tile": (ctypes.c_int, [_vp]),
    "tracer_batch_autotune": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    "tracer_batch_set_path": (ctypes.c_int, [ctypes.c_int]),
    "tracer_batch_learn_set": (ctypes.c_int, [_vp, ctypes.c_int]),
    "tracer_batch_get_path": (ctypes.c_int, []),
    "tracer_batch_steps": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "tracer_batch_time_steps": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "tracer_batch_steps_separate": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "tracer_batch_time_separate": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "tracer_batch_info": (ctypes.c_int, [_vp]),
    "tracer_selftest_barrier_timeout": (ctypes.c_int, [ctypes.c_longlong]),
    "tracer_selftest_umma": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "tracer_mlp_num_params": (ctypes.c_int, []),
    "tracer_mlp_forward": (ctypes.c_int, [_vp, ctypes.c_longlong, _vp, _vp]),
    "tracer_mlp_grads": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _vp, _vp]),
    "tracer_learn_set": (ctypes.c_int, [_vp, ctypes.c_int]),
    "tracer_learn_get": (ctypes.c_int, [_vp]),
    "tracer_learn_grad": (ctypes.c_int, [_vp]),
    "tracer_learn_step": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double)]),
    "tracer_write_mesh": (ctypes.c_int, [ctypes.c_char_p]),
    "tracer_scalar_output_open": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "tracer_scalar_output_write": (ctypes.c_int, []),
    "tracer_scalar_output_close": (ctypes.c_int, []),
    "tracer_advect_device_noalloc": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_double]),
    "tracer_noalloc_scratch_bytes": (ctypes.c_longlong, []),
    "tracer_last_error": (ctypes.c_char_p, []),
    "tracer_partition_read_dist": (ctypes.c_int, [ctypes.c_char_p, _vp, _vp]),
    "tracer_partition_halo": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                             ctypes.c_int]),
    "tracer_partition_part_dims": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "tracer_partition_install_part": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "tracer_partition_part_ids": (ctypes.c_int, [_vp, _vp]),
    "tracer_dd_setup": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int]),
    "tracer_dd_destroy": (ctypes.c_int, []),
    "tracer_dd_part_info": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_dd_allocate_tracers": (ctypes.c_int, [ctypes.c_int]),
    "tracer_dd_set_scheme": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                            ctypes.c_double, ctypes.c_double]),
    "tracer_dd_set_velocity": (ctypes.c_int, [_vp, _vp]),
    "tracer_dd_set_values": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_dd_get_values": (ctypes.c_int, [ctypes.c_int, _vp]),
    "tracer_dd_steps": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "tracer_dd_transfer_nodes": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "tracer_dd_pack": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "tracer_dd_unpack": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
}

REFERENCE_SYMBOLS = [
    "tracer_init_mpi", "tracer_finalize_mpi", "tracer_init", "tracer_finalize",
    "tracer_set_mesh_dims", "tracer_set_levels", "tracer_set_thickness", "tracer_set_partition",
    "tracer_allocate_tracers", "tracer_set_values", "tracer_set_velocity", "tracer_set_velocity_zero",
    "tracer_init_complete", "tracer_load_mesh_partition", "tracer_advect_step", "tracer_get_stats",
    "tracer_get_size", "tracer_get_values", "tracer_cleanup", "tracer_run_workflow",
    "tracer_load_mesh_from_files", "tracer_init_ale_arrays", "tracer_init_for_advection",
]

_LIB = None


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load libfesom_tracer.so once and attach the signatures."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build the CUDA library first (python -c 'import __graft_entry__ as g; g.build()' "
            "or make -C fesom2_tracer_dwarf_b200)")
    lib = ctypes.CDLL(str(p), mode=ctypes.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def ptr(a: np.ndarray | None):
    """Raw pointer of a contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    if not (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]):
        raise ValueError("array must be contiguous")
    return a.ctypes.data_as(ctypes.c_void_p)


def check(lib, rc: int, what: str) -> None:
    if rc != 0:
        msg = lib.tracer_last_error()
        raise RuntimeError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")
