"""Domain decomposition on the host: part maps (the reference's METIS
partitions of the pi mesh and index strips of the analytic mesh), halo
transfer lists, local part sizes, and the point-to-point halo exchange with
two gloo ranks on the CPU."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from test_replicas import _launch

ROOT = Path(__file__).resolve().parents[1]


def _check_plans(api, part, nparts):
    from fesom2_tracer_dwarf_b200 import decomp
    owned = [set(np.flatnonzero(part == p)) for p in range(nparts)]
    assert sum(len(o) for o in owned) == part.size
    for q in range(nparts):
        dims = decomp.part_dims(api, part, nparts, q)
        assert dims["owned"] == len(owned[q])
        into_q = 0
        for p in range(nparts):
            if p == q:
                continue
            t = decomp.halo_transfer(api, part, nparts, p, q)
            assert np.all(np.diff(t) > 0)                  # ascending global ids
            assert set(t.tolist()) <= owned[p]             # only nodes p owns
            into_q += t.size
        assert dims["nodes"] == dims["owned"] + into_q      # the halo is exactly what the peers send
        assert into_q > 0 and dims["elements"] > 0 and dims["edges"] > 0


@pytest.mark.parametrize("n", [2, 8])
def test_pi_mesh_metis_partitions(api, pi_mesh_dir, n):
    from fesom2_tracer_dwarf_b200 import decomp
    api.load_mesh_from_files(pi_mesh_dir)
    part, nparts = decomp.read_dist(api, pi_mesh_dir / f"dist_{n}")
    assert nparts == n
    _check_plans(api, part, nparts)


@pytest.mark.parametrize("n", [2, 3, 5])
def test_analytic_strips(api, n):
    from fesom2_tracer_dwarf_b200 import decomp
    api.init_analytic(30, 24, 8, periodic=True, full_rings=True)
    part = decomp.partition_by_index(api.mesh_dims()["nod2D"], n)
    _check_plans(api, part, n)


def test_bad_partition_files_fail_cleanly(api, pi_mesh_dir, tmp_path):
    import shutil
    from fesom2_tracer_dwarf_b200 import decomp
    api.load_mesh_from_files(pi_mesh_dir)
    d = tmp_path / "dist_2"
    shutil.copytree(pi_mesh_dir / "dist_2", d)
    (d / "my_list00001.out").unlink()
    with pytest.raises(RuntimeError, match="my_list00001"):
        decomp.read_dist(api, d)
    shutil.copy(pi_mesh_dir / "dist_2" / "my_list00000.out", d / "my_list00001.out")
    with pytest.raises(RuntimeError, match="bad header|disagrees|owned twice"):
        decomp.read_dist(api, d)


WORKER = r'''
import json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, torch
import torch.distributed as dist
from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection, decomp
from fesom2_tracer_dwarf_b200.replicas import from_env
r = from_env("gloo", timeout_s=60)
api = FESOMTracerAdvection()
api.init_analytic(20, 16, 6, periodic=True, full_rings=True)
N, L = api.mesh_dims()["nod2D"], 5
part = decomp.partition_by_index(N, r.world)
send_ids = {p: decomp.halo_transfer(api, part, r.world, r.rank, p) for p in range(r.world) if p != r.rank}
recv_ids = {p: decomp.halo_transfer(api, part, r.world, p, r.rank) for p in range(r.world) if p != r.rank}
# every rank's copy of the field: its own rows hold 1000 * node + level, halo rows -1
field = np.full((N, L), -1.0)
mine = np.flatnonzero(part == r.rank)
field[mine] = 1000.0 * mine[:, None] + np.arange(L)[None, :]
hx = decomp.HaloExchange({p: v.size * L for p, v in send_ids.items()}, {p: v.size * L for p, v in recv_ids.items()}, "cpu")
def pack(peer):
    return torch.from_numpy(np.ascontiguousarray(field[send_ids[peer]]).ravel())
def unpack(peer, buf):
    field[recv_ids[peer]] = buf.numpy().reshape(-1, L)
hx.exchange(pack, unpack)
hx.exchange(pack, unpack)  # idempotent
halo = np.concatenate([v for v in recv_ids.values()])
ok = bool(np.array_equal(field[halo], 1000.0 * halo[:, None] + np.arange(L)[None, :]))
print(json.dumps({"rank": r.rank, "ok": ok, "halo": int(halo.size)}))
r.close()
'''


def test_halo_exchange_two_gloo_ranks():
    import json
    outs = _launch(["-c", WORKER, str(ROOT)])
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert all(d["ok"] for d in res)
    assert all(d["halo"] > 0 for d in res)


def test_decomposition_refuses_unsupported_setups(api):
    """16-bit storage (per-part storage offsets would differ) and fewer than
    three halo rings are refused before any device work."""
    from fesom2_tracer_dwarf_b200.decomp import DomainDecomposition, partition_by_index
    api.init_analytic(20, 16, 6, periodic=True, full_rings=True)
    part = partition_by_index(api.mesh_dims()["nod2D"], 2)
    with pytest.raises(RuntimeError, match="at least 3 halo rings"):
        DomainDecomposition(api, part, 2, rings=2)
    with pytest.raises(RuntimeError, match="outside"):
        DomainDecomposition(api, np.where(part == 1, 5, 0).astype(np.int32), 2)
    with pytest.raises(RuntimeError, match="listed twice"):
        DomainDecomposition(api, part, 2, parts=[1, 1])
    api.set_precision("bf16")
    try:
        with pytest.raises(RuntimeError, match="FP64 and FP32"):
            DomainDecomposition(api, part, 2)
    finally:
        api.set_precision("fp64")


@pytest.mark.parametrize("n", [2, 8])
def test_one_ring_halos_equal_the_reference_partition_lists(api, pi_mesh_dir, n):
    """The reference's my_list<part>.out files list each part's halo nodes
    (eDim_nod2D: the nodes of its elements that other parts own, one ring);
    the library's one-ring halo (union of the transfers into the part) is
    exactly that set, for every part of both partitions."""
    from fesom2_tracer_dwarf_b200 import decomp
    api.load_mesh_from_files(pi_mesh_dir)
    part, nparts = decomp.read_dist(api, pi_mesh_dir / f"dist_{n}")
    for r in range(nparts):
        words = (pi_mesh_dir / f"dist_{n}" / f"my_list{r:05d}.out").read_text().split()
        my, halo = int(words[1]), int(words[2])
        ref = set(int(v) - 1 for v in words[3 + my:3 + my + halo])
        ours = set()
        for q in range(nparts):
            if q != r:
                ours |= set(decomp.halo_transfer(api, part, nparts, q, r, rings=1).tolist())
        assert ours == ref, f"part {r}"


def _com_nod2D(path):
    """Node receive / send structure of a com_info<part>.out file
    (lib/oce_mesh.F90:686-702): {peer: local 1-based indices} for both."""
    w = [int(v) for v in path.read_text().split()]
    i = 1
    out = []
    for _ in range(2):  # receive, then send
        npe = w[i]; i += 1
        pes = w[i:i + npe]; i += npe
        ptr = w[i:i + npe + 1]; i += npe + 1
        lst = w[i:i + ptr[-1] - 1]; i += ptr[-1] - 1
        out.append({pe: lst[ptr[k] - 1:ptr[k + 1] - 1] for k, pe in enumerate(pes)})
    return out


@pytest.mark.parametrize("n", [2, 8])
def test_one_ring_transfers_equal_the_reference_communication_lists(api, pi_mesh_dir, n):
    """Per peer, the nodes a part receives and sends (the reference's
    com_nod2D lists, local indices into its my_list order) are the library's
    one-ring halo transfers."""
    from fesom2_tracer_dwarf_b200 import decomp
    api.load_mesh_from_files(pi_mesh_dir)
    part, nparts = decomp.read_dist(api, pi_mesh_dir / f"dist_{n}")
    for r in range(nparts):
        words = (pi_mesh_dir / f"dist_{n}" / f"my_list{r:05d}.out").read_text().split()
        my, halo = int(words[1]), int(words[2])
        local = [int(v) - 1 for v in words[3:3 + my + halo]]  # local -> global, 0-based
        recv, send = _com_nod2D(pi_mesh_dir / f"dist_{n}" / f"com_info{r:05d}.out")
        for q in range(nparts):
            if q == r:
                continue
            ours_in = set(decomp.halo_transfer(api, part, nparts, q, r, rings=1).tolist())
            ours_out = set(decomp.halo_transfer(api, part, nparts, r, q, rings=1).tolist())
            assert ours_in == set(local[i - 1] for i in recv.get(q, [])), f"part {r} from {q}"
            assert ours_out == set(local[i - 1] for i in send.get(q, [])), f"part {r} to {q}"
