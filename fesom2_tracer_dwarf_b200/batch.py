"""Python host of the multi-member batch (include/fesom_tracer.h, tracer_batch_*).

Many tracers of many ensemble members, each on its own analytic mesh, are
advanced together in FP32: one persistent cooperative kernel launch per step,
replayed from a CUDA graph, with tiles chosen by an autotuner.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class TracerBatch:
    def __init__(self, lib_path=None):
        self.lib = _lib.load(lib_path)
        _lib.check(self.lib, self.lib.tracer_batch_create(), "tracer_batch_create")
        self.members = []

    def close(self):
        self.lib.tracer_batch_destroy()
        self.members = []

    # ---- members -----------------------------------------------------------
    def add_member(self, nx, ny, nl, ntracers, periodic=True, node_K=None, full_rings=True, left_oriented=True,
                   Lx=1.0e5, Ly=1.0e5, max_depth=1000.0):
        K = None if node_K is None else np.ascontiguousarray(node_K, dtype=np.int32)
        opts = int(bool(full_rings)) | (2 if left_oriented else 0)
        m = self.lib.tracer_batch_add_member(nx, ny, nl, Lx, Ly, max_depth, int(periodic), opts, _lib.ptr(K), ntracers)
        _lib.check(self.lib, -1 if m < 0 else 0, "tracer_batch_add_member")
        self.members.append({"nx": nx, "ny": ny, "nl": nl, "ntracers": ntracers, "periodic": bool(periodic)})
        return m

    def member_dims(self, m):
        d = np.zeros(4, dtype=np.int32)
        _lib.check(self.lib, self.lib.tracer_batch_member_dims(m, _lib.ptr(d)), "tracer_batch_member_dims")
        return {"nl": int(d[0]), "nod2D": int(d[1]), "elem2D": int(d[2]), "edge2D": int(d[3])}

    def set_velocity(self, m, uv, w):
        d = self.member_dims(m)
        u = np.asfortranarray(uv, dtype=np.float64)
        ww = np.asfortranarray(w, dtype=np.float64)
        if u.shape != (2, d["nl"] - 1, d["elem2D"]) or ww.shape != (d["nl"], d["nod2D"]):
            raise ValueError("velocity shapes do not match the member's mesh")
        _lib.check(self.lib, self.lib.tracer_batch_set_velocity(m, _lib.ptr(u), _lib.ptr(ww)),
                   "tracer_batch_set_velocity")

    def set_values(self, m, tracer_id, values):
        d = self.member_dims(m)
        v = np.asfortranarray(values, dtype=np.float64)
        if v.shape != (d["nl"] - 1, d["nod2D"]):
            raise ValueError("values shape does not match the member's mesh")
        _lib.check(self.lib, self.lib.tracer_batch_set_values(m, tracer_id, _lib.ptr(v)), "tracer_batch_set_values")

    def get_values(self, m, tracer_id):
        d = self.member_dims(m)
        v = np.zeros((d["nl"] - 1, d["nod2D"]), order="F")
        _lib.check(self.lib, self.lib.tracer_batch_get_values(m, tracer_id, _lib.ptr(v)), "tracer_batch_get_values")
        return v

    # ---- stepping ----------------------------------------------------------
    def configure(self, dt, hor="MUSCL", ver="PPM", lim="FCT", ph=1.0, pv=1.0, refresh_ab=True):
        d = np.ascontiguousarray(dt, dtype=np.float64)
        rc = self.lib.tracer_batch_configure(hor.encode(), ver.encode(), lim.encode(), ph, pv, _lib.ptr(d),
                                             int(bool(refresh_ab)))
        _lib.check(self.lib, rc, "tracer_batch_configure")

    def set_tile(self, cells_per_block=512, threads=256, blocks_per_sm=2, wave=3):
        _lib.check(self.lib, self.lib.tracer_batch_set_tile(cells_per_block, threads, blocks_per_sm, wave),
                   "tracer_batch_set_tile")

    def tile(self):
        t = np.zeros(4, dtype=np.int32)
        _lib.check(self.lib, self.lib.tracer_batch_get_tile(_lib.ptr(t)), "tracer_batch_get_tile")
        return {"cells_per_block": int(t[0]), "threads": int(t[1]), "blocks_per_sm": int(t[2]), "wave": int(t[3])}

    def autotune(self, steps_per_candidate=3):
        buf = ctypes.create_string_buffer(1 << 16)
        _lib.check(self.lib, self.lib.tracer_batch_autotune(steps_per_candidate, buf, len(buf)), "tracer_batch_autotune")
        return buf.value.decode()

    PATHS = {"cooperative": 0, "phases": 1, "separate": 2}

    def set_path(self, path):
        """'phases' (default): one persistent launch per phase and wave;
        'cooperative': the whole step as one cooperative launch; 'separate':
        the members' own per-batch kernel launches on their streams."""
        _lib.check(self.lib, self.lib.tracer_batch_set_path(self.PATHS[path]), "tracer_batch_set_path")

    def path(self):
        rc = self.lib.tracer_batch_get_path()
        _lib.check(self.lib, min(rc, 0), "tracer_batch_get_path")
        return {v: k for k, v in self.PATHS.items()}[rc]

    def learn_set(self, params=None, on=True):
        """The learned antidiffusive flux on every member's MUSCL tracers
        (params: the MLP's packed FP32 parameters; None keeps each member's).
        While on, the batch steps on the 'separate' path."""
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if p is not None and p.shape != (self.lib.tracer_mlp_num_params(),):
            raise ValueError("params must hold tracer_mlp_num_params() floats")
        _lib.check(self.lib, self.lib.tracer_batch_learn_set(_lib.ptr(p), int(bool(on))), "tracer_batch_learn_set")

    def steps(self, n, graph=True):
        _lib.check(self.lib, self.lib.tracer_batch_steps(n, int(bool(graph))), "tracer_batch_steps")

    def time_steps(self, n, graph=True):
        ms = ctypes.c_double()
        _lib.check(self.lib, self.lib.tracer_batch_time_steps(n, int(bool(graph)), ctypes.byref(ms)),
                   "tracer_batch_time_steps")
        return ms.value

    def steps_separate(self, n, graph=False):
        _lib.check(self.lib, self.lib.tracer_batch_steps_separate(n, int(bool(graph))), "tracer_batch_steps_separate")

    def time_separate(self, n, graph=False):
        ms = ctypes.c_double()
        _lib.check(self.lib, self.lib.tracer_batch_time_separate(n, int(bool(graph)), ctypes.byref(ms)),
                   "tracer_batch_time_separate")
        return ms.value

    def info(self):
        i = np.zeros(4, dtype=np.int64)
        _lib.check(self.lib, self.lib.tracer_batch_info(_lib.ptr(i)), "tracer_batch_info")
        return {"members": int(i[0]), "cell_tracers": int(i[1]), "work_bytes": int(i[2]), "graph": bool(i[3])}
