"""The multi-GPU form is N independent replicas (no data-path collective): each rank sorts
its own copy of the workload, the job's time is the slowest rank's (a MAX all-reduce), and
the reported rate is all ranks' units over that time.  Checked here with two gloo ranks on
the CPU (127.0.0.1 rendezvous), and the reference arm's rule that only rank 0 runs."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, datetime
sys.path.insert(0, %r)
import torch.distributed as dist
import bench
rank, world, _ = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
secs = [0.25, 0.5][rank]                  # rank 1 is the slow replica
m = bench.reduce_max(secs, world, "cpu")
rate = bench.replica_rate(1000, world, m)
print("RANK", rank, m, rate, flush=True)
dist.barrier()
dist.destroy_process_group()
""" % ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_replicas_max_time_and_rate(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        out, _ = p.communicate(timeout=120)
        assert p.returncode == 0, out
        outs.append([l for l in out.splitlines() if l.startswith("RANK")][0].split())
    for _, rank, m, rate in outs:
        assert float(m) == 0.5                     # both ranks see the slowest replica's time
        assert float(rate) == pytest.approx(4000.0)  # 2 ranks x 1000 units / 0.5 s


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""              # no work and no JSON line on the other ranks
