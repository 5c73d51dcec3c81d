"""Domain-decomposed tracer step (tracer_dd_* of the C ABI).

The loaded mesh is split into parts by a node -> part map (a FESOM2 partition
directory ``dist_<n>``, or contiguous strips of node ids); every part
runs the ordinary step on its own local mesh (owned nodes plus three rings of
halo nodes) and the halo values are exchanged after every step.  Owned values
are bit-identical to a step of the whole mesh.

* ``DomainDecomposition`` holds any subset of the parts in this process (all
  of them to run a decomposed mesh on one GPU; the exchange is then a device
  copy between the parts' engines).
* ``DistributedTracer`` is one part per rank: after each step the packed halo
  rows go to the peers with ``torch.distributed`` point-to-point messages
  (NCCL between GPUs), through ``HaloExchange``.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from . import _lib

RINGS = 3


def partition_by_index(nod2D: int, parts: int) -> np.ndarray:
    """Contiguous strips of ascending node id (bands of rows on the analytic mesh)."""
    if not 1 <= parts <= nod2D:
        raise ValueError("need 1 <= parts <= nod2D")
    return (np.arange(nod2D, dtype=np.int64) * parts // nod2D).astype(np.int32)


def read_dist(api, dist_dir) -> tuple[np.ndarray, int]:
    """Node -> part map of a FESOM2 partition directory (dist_<n>: rpart.out
    and my_list<part>.out) for the loaded mesh."""
    part = np.zeros(api.mesh_dims()["nod2D"], dtype=np.int32)
    n = np.zeros(1, dtype=np.int32)
    _lib.check(api.lib, api.lib.tracer_partition_read_dist(str(Path(dist_dir)).encode(), _lib.ptr(part), _lib.ptr(n)),
               "tracer_partition_read_dist")
    return part, int(n[0])


def halo_transfer(api, node_part: np.ndarray, nparts: int, src: int, dst: int, rings: int = RINGS) -> np.ndarray:
    """0-based global ids of the nodes part ``src`` owns in the halo of part ``dst``, ascending."""
    node_part = np.ascontiguousarray(node_part, dtype=np.int32)
    out = np.zeros(node_part.size, dtype=np.int32)
    n = api.lib.tracer_partition_halo(_lib.ptr(node_part), nparts, src, dst, rings, _lib.ptr(out), out.size)
    if n < 0:
        _lib.check(api.lib, n, "tracer_partition_halo")
    return out[:n] - 1


def part_dims(api, node_part: np.ndarray, nparts: int, part: int, rings: int = RINGS) -> dict:
    node_part = np.ascontiguousarray(node_part, dtype=np.int32)
    d = np.zeros(4, dtype=np.int32)
    _lib.check(api.lib, api.lib.tracer_partition_part_dims(_lib.ptr(node_part), nparts, part, rings, _lib.ptr(d)),
               "tracer_partition_part_dims")
    return {"owned": int(d[0]), "nodes": int(d[1]), "elements": int(d[2]), "edges": int(d[3])}


class DomainDecomposition:
    """Parts ``parts`` (default: all) of the decomposition, on this process's GPU."""

    def __init__(self, api, node_part: np.ndarray, nparts: int, parts=None, rings: int = RINGS):
        self.api, self.lib = api, api.lib
        self.node_part = np.ascontiguousarray(node_part, dtype=np.int32)
        self.nparts = nparts
        self.parts = list(range(nparts)) if parts is None else list(parts)
        local = np.asarray(self.parts, dtype=np.int32)
        d = api.mesh_dims()
        self.nl, self.nod2D, self.elem2D = d["nl"], d["nod2D"], d["elem2D"]
        _lib.check(self.lib, self.lib.tracer_dd_setup(_lib.ptr(self.node_part), nparts, _lib.ptr(local), local.size,
                                                      rings), "tracer_dd_setup")

    def part_info(self, i: int) -> dict:
        v = np.zeros(5, dtype=np.int32)
        _lib.check(self.lib, self.lib.tracer_dd_part_info(i, _lib.ptr(v)), "tracer_dd_part_info")
        return {"part": int(v[0]), "owned": int(v[1]), "nodes": int(v[2]), "elements": int(v[3]), "edges": int(v[4])}

    def allocate_tracers(self, n: int) -> None:
        _lib.check(self.lib, self.lib.tracer_dd_allocate_tracers(n), "tracer_dd_allocate_tracers")

    def set_scheme(self, tracer_id, hor="MUSCL", ver="PPM", lim="FCT", ph=1.0, pv=1.0) -> None:
        _lib.check(self.lib, self.lib.tracer_dd_set_scheme(tracer_id, hor.encode(), ver.encode(), lim.encode(), ph, pv),
                   "tracer_dd_set_scheme")

    def set_velocity(self, uv, w) -> None:
        uv = np.asfortranarray(uv, dtype=np.float64)
        w = np.asfortranarray(w, dtype=np.float64)
        if uv.shape != (2, self.nl - 1, self.elem2D) or w.shape != (self.nl, self.nod2D):
            raise ValueError("uv must be (2, nl-1, elem2D) and w (nl, nod2D)")
        _lib.check(self.lib, self.lib.tracer_dd_set_velocity(_lib.ptr(uv), _lib.ptr(w)), "tracer_dd_set_velocity")

    def set_values(self, tracer_id, values) -> None:
        v = np.asfortranarray(values, dtype=np.float64)
        if v.shape != (self.nl - 1, self.nod2D):
            raise ValueError("values must be (nl-1, nod2D)")
        _lib.check(self.lib, self.lib.tracer_dd_set_values(tracer_id, _lib.ptr(v)), "tracer_dd_set_values")

    def get_values(self, tracer_id, out=None) -> np.ndarray:
        """Whole-mesh array with the rows of the nodes the local parts own
        (other rows as in ``out``, zero by default)."""
        if out is None:
            out = np.zeros((self.nl - 1, self.nod2D), order="F")
        _lib.check(self.lib, self.lib.tracer_dd_get_values(tracer_id, _lib.ptr(out)), "tracer_dd_get_values")
        return out

    def steps(self, nsteps: int, dt: float, refresh_ab: bool = True, exchange: bool = True) -> None:
        """nsteps steps of every local part; with exchange, the halos of the
        local parts are refreshed from each other after every step."""
        _lib.check(self.lib, self.lib.tracer_dd_steps(nsteps, dt, int(refresh_ab), int(exchange)), "tracer_dd_steps")

    def transfer_nodes(self, i: int, peer: int, send: bool) -> int:
        n = self.lib.tracer_dd_transfer_nodes(i, peer, int(send))
        if n < 0:
            _lib.check(self.lib, n, "tracer_dd_transfer_nodes")
        return n

    def destroy(self) -> None:
        self.lib.tracer_dd_destroy()


class HaloExchange:
    """Point-to-point halo exchange between ranks with ``torch.distributed``.

    ``send[peer]`` / ``recv[peer]``: FP64 values this rank sends to / receives
    from each peer per tracer.  ``exchange(pack, unpack)`` posts every receive
    and send in one batch (no ordering deadlock), waits, then unpacks; every
    rank must call it the same number of times."""

    def __init__(self, send: dict, recv: dict, device):
        self.send = {p: n for p, n in send.items() if n > 0}
        self.recv = {p: n for p, n in recv.items() if n > 0}
        self.device = device

    def exchange(self, pack, unpack) -> None:
        import torch
        import torch.distributed as dist
        ops, bufs = [], {}
        for peer in sorted(self.recv):
            bufs[peer] = torch.empty(self.recv[peer], dtype=torch.float64, device=self.device)
            ops.append(dist.P2POp(dist.irecv, bufs[peer], peer))
        for peer in sorted(self.send):
            t = pack(peer)
            if t.numel() != self.send[peer]:
                raise ValueError("packed halo of the wrong size")
            ops.append(dist.P2POp(dist.isend, t, peer))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for peer in sorted(bufs):
            unpack(peer, bufs[peer])


class DistributedTracer:
    """One part per rank (part = rank, nparts = world size) on this rank's
    GPU; ``steps`` advances every tracer and exchanges the halos with the
    peers after each step, one message per peer holding every tracer's rows.
    The halo rows are packed on the GPU; with the NCCL backend they travel
    from device memory, with gloo through host memory."""

    def __init__(self, api, node_part: np.ndarray, rank: int, world: int, device, rings: int = RINGS):
        import torch.distributed as dist
        self.dd = DomainDecomposition(api, node_part, world, parts=[rank], rings=rings)
        self.rank, self.world, self.device = rank, world, device
        self.L = self.dd.nl - 1
        self.send_nodes = {p: self.dd.transfer_nodes(0, p, True) for p in range(world) if p != rank}
        self.recv_nodes = {p: self.dd.transfer_nodes(0, p, False) for p in range(world) if p != rank}
        backend = dist.get_backend() if dist.is_available() and dist.is_initialized() else None
        if world > 1 and backend is None:
            raise RuntimeError("DistributedTracer: initialise torch.distributed for more than one rank")
        self.wire = device if backend == "nccl" else "cpu"
        self.ntr = 0
        self.halo = None

    def allocate_tracers(self, n: int) -> None:
        self.dd.allocate_tracers(n)
        self.ntr = n
        self.halo = HaloExchange({p: c * self.L * n for p, c in self.send_nodes.items()},
                                 {p: c * self.L * n for p, c in self.recv_nodes.items()}, self.wire)

    def exchange(self) -> None:
        """Halo rows of every tracer, tracer after tracer in one buffer per peer."""
        import torch
        lib = self.dd.lib

        def pack(peer):
            per = self.send_nodes[peer] * self.L
            buf = torch.empty(per * self.ntr, dtype=torch.float64, device=self.device)
            for t in range(self.ntr):
                _lib.check(lib, lib.tracer_dd_pack(0, t + 1, peer, buf[t * per:(t + 1) * per].data_ptr()),
                           "tracer_dd_pack")
            return buf.to(self.wire)

        def unpack(peer, buf):
            per = self.recv_nodes[peer] * self.L
            dev = buf.to(self.device).contiguous()
            for t in range(self.ntr):
                _lib.check(lib, lib.tracer_dd_unpack(0, t + 1, peer, dev[t * per:(t + 1) * per].data_ptr()),
                           "tracer_dd_unpack")

        self.halo.exchange(pack, unpack)

    def steps(self, nsteps: int, dt: float, refresh_ab: bool = True) -> None:
        for _ in range(nsteps):
            self.dd.steps(1, dt, refresh_ab, exchange=False)
            self.exchange()
