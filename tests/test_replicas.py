"""Multi-rank host logic of the replica runs (bench.py --gpus N) with two gloo
ranks on the CPU: barriers, the maximum over ranks, the job-wide rate, and
the reference arm leaving the work to rank 0."""
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

WORKER = r'''
import os, sys, json
sys.path.insert(0, sys.argv[1])
from fesom2_tracer_dwarf_b200.replicas import from_env, job_rate
r = from_env("gloo", timeout_s=60)
r.barrier()
mine = 10.0 + 5.0 * r.rank
worst = r.max(mine)
rate = job_rate(1000.0, r.world, worst)
r.barrier()
print(json.dumps({"rank": r.rank, "world": r.world, "worst": worst, "rate": rate}))
r.close()
'''


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _launch(code_args, world=2):
    port = _port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable] + code_args, env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_two_gloo_ranks_max_and_rate():
    import json
    outs = _launch(["-c", WORKER, str(ROOT)])
    res = sorted((json.loads(o.strip().splitlines()[-1]) for o in outs), key=lambda d: d["rank"])
    assert [d["world"] for d in res] == [2, 2]
    assert all(d["worst"] == 15.0 for d in res)          # the slowest rank's time on every rank
    assert all(abs(d["rate"] - 2 * 1000.0 / 15.0) < 1e-12 for d in res)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun, `bench.py --impl reference` does its CPU work on rank 0
    and the other ranks leave at once with status 0 and no output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=240)
    assert p.returncode == 0 and p.stdout.strip() == ""
