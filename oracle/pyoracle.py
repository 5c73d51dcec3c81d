"""ctypes wrapper of the CPU oracle (oracle/fesom_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py to check / time against the reference algorithm.
The product library never loads it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SERIAL = HERE / "_build" / "libfesom_oracle.so"
OPENMP = HERE / "_build" / "libfesom_oracle_omp.so"

HOR = {"UPW1": 0, "MUSCL": 1, "MFCT": 2}
VER = {"UPW1": 0, "PPM": 1, "QR4C": 2, "CDIFF": 3}
LIM = {"NONE": 0, "FCT": 1}

_INT_FIELDS = {"elem2D_nodes", "edges", "edge_tri", "nlevels", "ulevels", "nlevels_nod2D", "ulevels_nod2D",
               "nlevels_nod2D_min", "ulevels_nod2D_max", "nod_in_elem2D_num", "nod_in_elem2D",
               "edge_up_dn_tri", "nboundary_lay"}


def build() -> None:
    """Compile both oracle flavours (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    def __init__(self, openmp: bool = False):
        path = OPENMP if openmp else SERIAL
        if not path.exists():
            build()
        lib = ctypes.CDLL(str(path))
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        lib.om_mesh_analytic.restype = vp
        lib.om_mesh_analytic.argtypes = [ci, ci, ci, cd, cd, cd, ci, ci, vp]
        lib.om_mesh_free.argtypes = [vp]
        lib.om_mesh_from_files.restype = vp
        lib.om_mesh_from_arrays.restype = vp
        lib.om_mesh_from_arrays.argtypes = [ci, ci, ci, ci, ci, cd, cd] + [vp] * 22
        lib.om_mesh_from_files.argtypes = [ctypes.c_char_p, ci, cd, cd, cd, cd, cd, ctypes.c_char_p, ci]
        lib.om_mesh_dims.argtypes = [vp, vp]
        lib.om_mesh_len.restype = ctypes.c_long
        lib.om_mesh_len.argtypes = [vp, ctypes.c_char_p]
        lib.om_mesh_get_int.argtypes = [vp, ctypes.c_char_p, vp]
        lib.om_mesh_get_dbl.argtypes = [vp, ctypes.c_char_p, vp]
        lib.om_analytic_fields.argtypes = [vp] * 5
        lib.om_tracer_step.argtypes = [vp, ci, ci, ci, cd, cd, cd] + [vp] * 7
        lib.om_run.argtypes = [vp, ci, ci, ci, cd, cd, cd, vp, vp, ci, ci, vp, vp, ci]
        lib.om_stats.argtypes = [vp, vp, vp]
        u64 = ctypes.c_ulonglong
        lib.om_synth_bathymetry_smooth.argtypes = [ci, ci, ci, ci, cd, u64, vp]
        lib.om_synth_velocity.argtypes = [vp, u64, cd, cd, cd, cd, vp, vp]
        lib.om_synth_tracer.argtypes = [vp, u64, ci, vp]
        lib.om_set_threads.argtypes = [ci]
        lib.om_get_threads.restype = ci
        self.lib = lib

    def set_threads(self, n: int) -> None:
        self.lib.om_set_threads(n)

    def threads(self) -> int:
        return self.lib.om_get_threads()


class OracleMesh:
    """An analytic mesh built by the oracle (lib/analytic_mesh.F90 restated)."""

    def __init__(self, oracle: Oracle, nx, ny, nl, Lx=1.0e5, Ly=1.0e5, max_depth=1000.0, periodic=True,
                 full_rings=True, node_K=None, left_oriented=False):
        self.o = oracle
        K = None if node_K is None else np.ascontiguousarray(node_K, dtype=np.int32)
        opts = int(bool(full_rings)) | (2 if left_oriented else 0)
        h = oracle.lib.om_mesh_analytic(nx, ny, nl, Lx, Ly, max_depth, int(periodic), opts, _p(K))
        if not h:
            raise ValueError("oracle mesh construction failed")
        self.h = ctypes.c_void_p(h)
        d = np.zeros(6, dtype=np.int32)
        oracle.lib.om_mesh_dims(self.h, _p(d))
        self.nl, self.nod2D, self.elem2D, self.edge2D, self.max_nie = (int(x) for x in d[:5])

    @classmethod
    def from_files(cls, oracle: Oracle, mesh_dir, rotate=True, alpha=50.0, beta=15.0, gamma=-90.0,
                   angle_scale=1.0, cyclic_length=360.0):
        """A mesh read from the reference's ASCII mesh files (mesh_setup of
        lib/oce_mesh.F90:49-94 restated; defaults are the reference's)."""
        self = cls.__new__(cls)
        self.o = oracle
        err = ctypes.create_string_buffer(512)
        h = oracle.lib.om_mesh_from_files(str(mesh_dir).encode(), int(bool(rotate)), alpha, beta, gamma,
                                          angle_scale, cyclic_length, err, len(err))
        if not h:
            raise ValueError("oracle mesh: " + err.value.decode())
        self.h = ctypes.c_void_p(h)
        d = np.zeros(6, dtype=np.int32)
        oracle.lib.om_mesh_dims(self.h, _p(d))
        self.nl, self.nod2D, self.elem2D, self.edge2D, self.max_nie = (int(x) for x in d[:5])
        return self

    FROM_ARRAYS = ["coord", "elem2D_nodes", "edges", "edge_tri", "nlevels", "nlevels_nod2D", "nlevels_nod2D_min",
                   "ring_num", "ring_elem", "elem_area", "area", "areasvol", "edge_dxdy", "edge_cross_dxdy",
                   "gradient_sca", "elem_cos", "zbar", "hnode", "hnode_new", "helem", "edge_up_dn_tri",
                   "nboundary_lay"]

    @classmethod
    def from_arrays(cls, oracle: Oracle, nl, nod2D, elem2D, edge2D, arrays: dict, periodic=False, Lx=0.0, Ly=0.0):
        """A mesh from arrays (``FROM_ARRAYS``, index arrays 1-based, 0 =
        none), every table taken as given."""
        self = cls.__new__(cls)
        self.o = oracle
        keep = []
        ptrs = []
        for name in cls.FROM_ARRAYS:
            a = arrays[name]
            a = np.ascontiguousarray(a, dtype=np.int32 if name in _INT_FIELDS | {"ring_num", "ring_elem"}
                                     else np.float64)
            keep.append(a)
            ptrs.append(_p(a))
        h = oracle.lib.om_mesh_from_arrays(nl, nod2D, elem2D, edge2D, int(periodic), Lx, Ly, *ptrs)
        if not h:
            raise ValueError("oracle mesh from arrays failed")
        self.h = ctypes.c_void_p(h)
        d = np.zeros(6, dtype=np.int32)
        oracle.lib.om_mesh_dims(self.h, _p(d))
        self.nl, self.nod2D, self.elem2D, self.edge2D, self.max_nie = (int(x) for x in d[:5])
        return self

    def __del__(self):
        try:
            self.o.lib.om_mesh_free(self.h)
        except Exception:
            pass

    def array(self, name: str) -> np.ndarray:
        n = self.o.lib.om_mesh_len(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        if name in _INT_FIELDS:
            a = np.zeros(n, dtype=np.int32)
            self.o.lib.om_mesh_get_int(self.h, name.encode(), _p(a))
        else:
            a = np.zeros(n, dtype=np.float64)
            self.o.lib.om_mesh_get_dbl(self.h, name.encode(), _p(a))
        return a

    def shape_tracer(self):
        return (self.nl - 1, self.nod2D)

    def analytic_fields(self):
        L, N, T = self.nl - 1, self.nod2D, self.elem2D
        Tt = np.zeros((L, N), order="F")
        S = np.zeros((L, N), order="F")
        uv = np.zeros((2, L, T), order="F")
        w = np.zeros((self.nl, N), order="F")
        self.o.lib.om_analytic_fields(self.h, _p(Tt), _p(S), _p(uv), _p(w))
        return Tt, S, uv, w

    def step(self, values, values_ab, uv, w, dt, hor="MUSCL", ver="PPM", lim="FCT", ph=1.0, pv=1.0,
             want_terms=False):
        """One oracle step; values updated in place (Fortran-ordered float64)."""
        for a in (values, values_ab, uv, w):
            assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
        dh = dv = lo = None
        if want_terms:
            dh = np.zeros(self.shape_tracer(), order="F")
            dv = np.zeros(self.shape_tracer(), order="F")
            lo = np.zeros(self.shape_tracer(), order="F")
        self.o.lib.om_tracer_step(self.h, HOR[hor], VER[ver], LIM[lim], ph, pv, dt, _p(uv), _p(w), _p(values),
                                  _p(values_ab), _p(dh), _p(dv), _p(lo))
        return (dh, dv, lo) if want_terms else None

    def run(self, values, values_ab, uv, w, dt, nsteps, hor="MUSCL", ver="PPM", lim="FCT", ph=1.0, pv=1.0,
            refresh_ab=True):
        """nsteps steps of ntracers = values.shape[0] tracers stacked as (ntr, nl-1, nod2D)."""
        ntr = values.shape[0]
        self.o.lib.om_run(self.h, HOR[hor], VER[ver], LIM[lim], ph, pv, dt, _p(uv), _p(w), ntr, nsteps,
                          _p(values), _p(values_ab), int(refresh_ab))

    def synth_velocity(self, seed=0, umax=1.0, mode2=0.5, baro=0.0, mode1=1.0):
        """Seeded layered flow: uv (2, nl-1, elem2D), w (nl, nod2D)."""
        uv = np.zeros((2, self.nl - 1, self.elem2D), order="F")
        w = np.zeros((self.nl, self.nod2D), order="F")
        self.o.lib.om_synth_velocity(self.h, seed, umax, mode1, mode2, baro, _p(uv), _p(w))
        return uv, w

    def synth_tracer(self, seed=0, kind=0):
        v = np.zeros((self.nl - 1, self.nod2D), order="F")
        self.o.lib.om_synth_tracer(self.h, seed, kind, _p(v))
        return v

    def stats(self, values):
        s = np.zeros(4)
        self.o.lib.om_stats(self.h, _p(np.asfortranarray(values)), _p(s))
        return s


def synth_bathymetry_smooth(oracle: Oracle, nx, ny, nl, periodic=True, corr_cells=40.0, seed=0):
    """Smooth seeded bottom level index per analytic grid node (uniform on [3, nl])."""
    n = (nx - 1) * (ny - 1) if periodic else nx * ny
    K = np.zeros(n, dtype=np.int32)
    oracle.lib.om_synth_bathymetry_smooth(nx, ny, int(periodic), nl, corr_cells, seed, _p(K))
    return K


LX = LY = 1.0e5
MAX_DEPTH = 1000.0


def cfl_dt(nx, ny, nl, uv, w, cfl=0.5):
    """dt at CFL `cfl` of the faster of the horizontal and vertical crossings
    on the uniform analytic grid."""
    dx = min(LX / (nx - 1), LY / (ny - 1))
    dz = MAX_DEPTH / (nl - 1)
    umax = float(np.sqrt(uv[0] ** 2 + uv[1] ** 2).max())
    wmax = float(np.abs(w).max())
    rate = max(umax / dx, wmax / dz)
    return cfl / rate if rate > 0.0 else 1.0


def layered_flow_case(oracle: Oracle, nx, nl, seed=0, periodic=True):
    """The benchmark's plain-method-at-scale inputs built by the oracle alone:
    the same mesh, bathymetry, flow, tracers and dt as the library's
    workloads.layered_flow_case for the same arguments.  Returns
    (mesh, K, uv, w, T, S, dt, wet_cells)."""
    corr = max(4.0, nx / 25.0)
    K = synth_bathymetry_smooth(oracle, nx, nx, nl, periodic=periodic, corr_cells=corr, seed=seed)
    m = OracleMesh(oracle, nx, nx, nl, Lx=LX, Ly=LY, max_depth=MAX_DEPTH, periodic=periodic, full_rings=True,
                   node_K=K, left_oriented=True)
    uv, w = m.synth_velocity(seed=seed + 1, umax=1.0, mode2=0.5, baro=1.0)
    T = m.synth_tracer(seed=seed + 2, kind=0)
    S = m.synth_tracer(seed=seed + 3, kind=1)
    nlev = m.array("nlevels_nod2D")[: m.nod2D]
    wet = int(np.maximum(nlev - 1, 0).sum())
    return m, K, uv, w, T, S, cfl_dt(nx, nx, nl, uv, w), wet
