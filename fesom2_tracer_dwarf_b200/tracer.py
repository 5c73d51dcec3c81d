"""Python host of the B200 tracer advection library.

``FESOMTracerAdvection`` keeps the method names, arguments and return values
of the reference's ctypes wrapper (python/demo_tracer.py:40-208 in
suvarchal/fesom2_tracer_dwarf) and adds the analytic-mesh, scheme, velocity
and multi-tracer calls of include/fesom_tracer.h.  Arrays are numpy float64 in
Fortran order, shaped like the reference's: tracers (nl-1, nod2D), element
velocity (2, nl-1, elem2D), vertical velocity (nl, nod2D).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


_INT_MESH_ARRAYS = {"elem2D_nodes", "edges", "edge_tri", "nlevels", "nlevels_nod2D", "nlevels_nod2D_min",
                    "edge_up_dn_tri", "nboundary_lay", "ring_num", "ring_elem"}


def _f64(a, shape):
    a = np.asfortranarray(np.asarray(a, dtype=np.float64))
    if a.shape != tuple(shape):
        raise ValueError(f"expected shape {tuple(shape)}, got {a.shape}")
    return a


class FESOMTracerAdvection:
    """Drop-in for the reference's FESOMTracerAdvection, backed by sm_100a kernels."""

    def __init__(self, lib_path=None):
        self.lib = _lib.load(lib_path)
        self._pinned = {}  # host address -> array kept alive while page-locked

    # ---- methods of python/demo_tracer.py ---------------------------------
    def initialize_mpi(self, mpi_comm=0):
        return self.lib.tracer_init_mpi(mpi_comm)

    def initialize(self, restart_path="./fesom_bin_restart"):
        return self.lib.tracer_init(restart_path.encode())

    def advect_step(self, dt=1.0e-3):
        return self.lib.tracer_advect_step(dt)

    def get_tracer_values(self, tracer_id=1):
        nz, nn = ctypes.c_int(), ctypes.c_int()
        ret = self.lib.tracer_get_size(ctypes.byref(nz), ctypes.byref(nn))
        if ret != 0:
            raise RuntimeError(f"tracer_get_size failed with code {ret}")
        values = np.zeros((nz.value, nn.value), dtype=np.float64, order="F")
        ret = self.lib.tracer_get_values_id(tracer_id, _lib.ptr(values), nz, nn)
        if ret != 0:
            raise RuntimeError(f"tracer_get_values failed with code {ret}")
        return values

    def get_statistics(self, tracer_id=1):
        s = np.zeros(4)
        ret = self.lib.tracer_get_stats_id(tracer_id, _lib.ptr(s))
        if ret != 0:
            raise RuntimeError(f"tracer_get_stats failed with code {ret}")
        return {"min": s[0], "max": s[1], "sum": s[2], "nan": int(s[3])}

    def finalize(self, output_path="./fesom_bin_restart"):
        return self.lib.tracer_finalize(output_path.encode())

    def finalize_mpi(self):
        return self.lib.tracer_finalize_mpi()

    # ---- extensions ---------------------------------------------------------
    def init_analytic(self, nx, ny, nl, Lx=1.0e5, Ly=1.0e5, max_depth=1000.0, periodic=True,
                      full_rings=True, node_K=None, left_oriented=False):
        """Analytic mesh of the reference's generate_analytic_mesh (+ optional bathymetry)."""
        K = None
        if node_K is not None:
            K = np.ascontiguousarray(node_K, dtype=np.int32)
            if K.size != self.lib.tracer_analytic_nodes(nx, ny, int(periodic)):
                raise ValueError("node_K must have one entry per mesh node")
        opts = int(bool(full_rings)) | (2 if left_oriented else 0)
        rc = self.lib.tracer_init_analytic(nx, ny, nl, Lx, Ly, max_depth, int(periodic), opts, _lib.ptr(K))
        _lib.check(self.lib, rc, "tracer_init_analytic")
        self.dims = self.mesh_dims()
        return rc

    def load_mesh_from_files(self, mesh_path, rotate=True, alpha=50.0, beta=15.0, gamma=-90.0, angle_scale=1.0,
                             cyclic_length=360.0):
        """Mesh from a FESOM2 ASCII mesh directory (tracer_load_mesh_from_files).
        The defaults are the reference's conventions; angle_scale=pi/180 and
        cyclic_length=2*pi give FESOM2's (angles in degrees, longitude wrapped
        at the seam)."""
        path = str(mesh_path).encode()
        if (rotate, alpha, beta, gamma, angle_scale, cyclic_length) == (True, 50.0, 15.0, -90.0, 1.0, 360.0):
            rc = self.lib.tracer_load_mesh_from_files(path)
        else:
            rc = self.lib.tracer_load_mesh_from_files_opts(path, int(bool(rotate)), alpha, beta, gamma, angle_scale,
                                                           cyclic_length)
        _lib.check(self.lib, rc, "tracer_load_mesh_from_files")
        self.dims = self.mesh_dims()
        return rc

    def mesh_dims(self):
        d = np.zeros(6, dtype=np.int32)
        _lib.check(self.lib, self.lib.tracer_mesh_dims(_lib.ptr(d)), "tracer_mesh_dims")
        return {"nl": int(d[0]), "nod2D": int(d[1]), "elem2D": int(d[2]), "edge2D": int(d[3]),
                "level_stride": int(d[5])}

    def allocate_tracers(self, num_tracers, ab_order=2):
        d = self.mesh_dims()
        _lib.check(self.lib, self.lib.tracer_allocate_tracers(num_tracers, d["nl"], d["nod2D"], ab_order),
                   "tracer_allocate_tracers")

    def set_values(self, tracer_id, values, values_ab=None):
        d = self.mesh_dims()
        v = _f64(values, (d["nl"] - 1, d["nod2D"]))
        _lib.check(self.lib, self.lib.tracer_set_values(tracer_id, _lib.ptr(v), d["nl"], d["nod2D"]),
                   "tracer_set_values")
        if values_ab is not None:
            a = _f64(values_ab, (d["nl"] - 1, d["nod2D"]))
            _lib.check(self.lib, self.lib.tracer_set_values_ab(tracer_id, _lib.ptr(a), d["nl"], d["nod2D"]),
                       "tracer_set_values_ab")

    def set_scheme(self, tracer_id, hor="MUSCL", ver="PPM", lim="FCT", ph=1.0, pv=1.0):
        rc = self.lib.tracer_set_scheme(tracer_id, hor.encode(), ver.encode(), lim.encode(), ph, pv)
        _lib.check(self.lib, rc, "tracer_set_scheme")

    def set_velocity(self, uv, w):
        """uv (2, nl-1, elem2D) element velocity, w (nl, nod2D)."""
        d = self.mesh_dims()
        u = _f64(uv, (2, d["nl"] - 1, d["elem2D"]))
        ww = _f64(w, (d["nl"], d["nod2D"]))
        rc = self.lib.tracer_set_velocity_elem(_lib.ptr(u), _lib.ptr(ww), d["nl"], d["nod2D"], d["elem2D"])
        _lib.check(self.lib, rc, "tracer_set_velocity_elem")

    PRECISIONS = {"fp64": 0, "fp32": 1, "bf16": 2, "fp16": 3, "fp64fma": 4}

    def set_precision(self, mode):
        """'fp64' (bit-exact), 'fp32', 'bf16' or 'fp16' (16-bit tracer storage, FP32 arithmetic)."""
        _lib.check(self.lib, self.lib.tracer_set_precision(self.PRECISIONS[mode]), "tracer_set_precision")

    def pin(self, array):
        """Page-lock a contiguous numpy array so its transfers take one DMA
        (tracer_host_register).  The array is kept alive until unpin() or
        cleanup(): memory freed while still registered would leave the
        registration behind for whatever the allocator puts there next."""
        if not (array.flags["F_CONTIGUOUS"] or array.flags["C_CONTIGUOUS"]):
            raise ValueError("pin needs a contiguous array")
        addr = array.ctypes.data
        if addr in self._pinned:
            return array
        _lib.check(self.lib, self.lib.tracer_host_register(_lib.ptr(array), array.nbytes), "tracer_host_register")
        self._pinned[addr] = array
        return array

    def unpin(self, array):
        addr = array.ctypes.data
        _lib.check(self.lib, self.lib.tracer_host_unregister(_lib.ptr(array)), "tracer_host_unregister")
        self._pinned.pop(addr, None)

    def unpin_all(self):
        for a in list(self._pinned.values()):
            self.unpin(a)

    ROUNDING = {"nearest": 0, "stochastic": 1}

    def set_rounding(self, mode):
        """Rounding of new values into 16-bit storage: 'nearest' or 'stochastic'."""
        _lib.check(self.lib, self.lib.tracer_set_rounding(self.ROUNDING[mode]), "tracer_set_rounding")

    def storage_offset(self, tracer_id=1):
        """Offset subtracted from the tracer's wet cells in 16-bit storage (0 otherwise)."""
        out = np.zeros(1)
        _lib.check(self.lib, self.lib.tracer_storage_offset(tracer_id, _lib.ptr(out)), "tracer_storage_offset")
        return float(out[0])

    def volume_sum(self, tracer_id=1):
        """(Sum T, Sum T*areasvol*hnode_new) over wet cells, compensated FP64 on the device."""
        out = np.zeros(2)
        _lib.check(self.lib, self.lib.tracer_volume_sum(tracer_id, _lib.ptr(out)), "tracer_volume_sum")
        return float(out[0]), float(out[1])

    def advect_step_io(self, dt, values_in, values_out):
        """One step with host I/O (tracer_advect_step_io): values_in[t] (or None)
        become tracer t+1's values, values_out[t] (or None) receive the new
        values; pipelined across tracers when every array is page-locked
        (pin)."""
        n = len(values_in)
        vin = (ctypes.c_void_p * n)(*[None if a is None else a.ctypes.data for a in values_in])
        vout = (ctypes.c_void_p * n)(*[None if a is None else a.ctypes.data for a in values_out])
        _lib.check(self.lib, self.lib.tracer_advect_step_io(dt, ctypes.cast(vin, ctypes.c_void_p),
                                                            ctypes.cast(vout, ctypes.c_void_p), n),
                   "tracer_advect_step_io")

    def set_step_path(self, path):
        """'five' (default: five kernels) or 'fused' (one patch kernel per tracer where the scheme allows it)."""
        _lib.check(self.lib, self.lib.tracer_set_step_path({"fused": 0, "five": 1}[path]), "tracer_set_step_path")

    def set_cells_per_block(self, cells):
        """Most wet cells per block of the five-kernel schedules (0: the default, 512)."""
        _lib.check(self.lib, self.lib.tracer_set_cells_per_block(int(cells)), "tracer_set_cells_per_block")

    def set_patch_size(self, owned):
        """Owned nodes per patch of the fused kernel (0: the default)."""
        _lib.check(self.lib, self.lib.tracer_set_patch_size(int(owned)), "tracer_set_patch_size")

    def step_info(self):
        """dict(path, fused, patches, node_ratio) of the device state (tracer_step_info)."""
        out = np.zeros(4)
        _lib.check(self.lib, self.lib.tracer_step_info(_lib.ptr(out)), "tracer_step_info")
        return {"path": int(out[0]), "fused": bool(out[1]), "patches": int(out[2]), "node_ratio": float(out[3])}

    def set_ab_refresh(self, on):
        self.lib.tracer_set_ab_refresh(int(bool(on)))

    def advect_steps(self, nsteps, dt):
        _lib.check(self.lib, self.lib.tracer_advect_steps(nsteps, dt), "tracer_advect_steps")

    def analytic_fields(self):
        """T, S, uv, w of the analytic driver (src/fesom_analytic.F90:251-331)."""
        d = self.mesh_dims()
        L, N, T = d["nl"] - 1, d["nod2D"], d["elem2D"]
        Tt = np.zeros((L, N), order="F")
        S = np.zeros((L, N), order="F")
        uv = np.zeros((2, L, T), order="F")
        w = np.zeros((d["nl"], N), order="F")
        _lib.check(self.lib, self.lib.tracer_analytic_fields(_lib.ptr(Tt), _lib.ptr(S), _lib.ptr(uv), _lib.ptr(w)),
                   "tracer_analytic_fields")
        return Tt, S, uv, w

    def synth_velocity(self, seed=0, umax=1.0, mode2=0.5, baro=0.0, mode1=1.0):
        """Seeded layered flow (see tracer_synth_velocity): uv (2, nl-1, elem2D), w (nl, nod2D)."""
        d = self.mesh_dims()
        uv = np.zeros((2, d["nl"] - 1, d["elem2D"]), order="F")
        w = np.zeros((d["nl"], d["nod2D"]), order="F")
        _lib.check(self.lib, self.lib.tracer_synth_velocity(seed, umax, mode1, mode2, baro, _lib.ptr(uv), _lib.ptr(w)),
                   "tracer_synth_velocity")
        return uv, w

    def synth_tracer(self, seed=0, kind=0):
        d = self.mesh_dims()
        v = np.zeros((d["nl"] - 1, d["nod2D"]), order="F")
        _lib.check(self.lib, self.lib.tracer_synth_tracer(seed, kind, _lib.ptr(v)), "tracer_synth_tracer")
        return v

    def mesh_array(self, name):
        n = self.lib.tracer_mesh_len(name.encode())
        if n < 0:
            raise KeyError(name)
        if name in _INT_MESH_ARRAYS:
            out = np.zeros(n, dtype=np.int32)
            _lib.check(self.lib, self.lib.tracer_mesh_get_int(name.encode(), _lib.ptr(out)), "tracer_mesh_get_int")
            return out
        out = np.zeros(n, dtype=np.float64)
        _lib.check(self.lib, self.lib.tracer_mesh_get_dbl(name.encode(), _lib.ptr(out)), "tracer_mesh_get_dbl")
        return out

    def time_steps(self, nsteps, dt):
        ms = ctypes.c_float()
        _lib.check(self.lib, self.lib.tracer_time_steps(nsteps, dt, ctypes.byref(ms)), "tracer_time_steps")
        return ms.value

    def write_mesh(self, output_dir):
        """Mesh files for the reference's plotting scripts (tracer_write_mesh)."""
        _lib.check(self.lib, self.lib.tracer_write_mesh(str(output_dir).encode()), "tracer_write_mesh")

    def open_scalar_output(self, output_dir, nsteps):
        _lib.check(self.lib, self.lib.tracer_scalar_output_open(str(output_dir).encode(), nsteps),
                   "tracer_scalar_output_open")

    def write_scalar_step(self):
        _lib.check(self.lib, self.lib.tracer_scalar_output_write(), "tracer_scalar_output_write")

    def close_scalar_output(self):
        _lib.check(self.lib, self.lib.tracer_scalar_output_close(), "tracer_scalar_output_close")

    def cleanup(self):
        self.unpin_all()
        return self.lib.tracer_cleanup()


def synth_bathymetry_smooth(nx, ny, nl, periodic=True, corr_cells=40.0, seed=0):
    """Smooth seeded bottom level index (uniform marginal on [3, nl]) per node of the analytic grid."""
    lib = _lib.load()
    K = np.zeros(lib.tracer_analytic_nodes(nx, ny, int(periodic)), dtype=np.int32)
    _lib.check(lib, lib.tracer_synth_bathymetry_smooth(nx, ny, int(periodic), nl, corr_cells, seed, _lib.ptr(K)),
               "tracer_synth_bathymetry_smooth")
    return K


def synth_bathymetry(nnodes, nl, seed=0):
    lib = _lib.load()
    K = np.zeros(nnodes, dtype=np.int32)
    _lib.check(lib, lib.tracer_synth_bathymetry(nnodes, nl, seed, _lib.ptr(K)), "tracer_synth_bathymetry")
    return K
