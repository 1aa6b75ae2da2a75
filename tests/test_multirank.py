"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1) agree on the
slowest rank's times, and the reference arm prints only on rank 0.  The operator
itself does not shard ("replicas only"): each rank runs its own copy."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import datetime, os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank={rank}, world_size=2,
                        timeout=datetime.timedelta(seconds=60))
r = dist.get_rank()
out = bench.max_over_ranks([1.0 + r, 10.0 - r, 0.5 * r], dist)
print("RESULT", out, flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def test_max_over_ranks_gloo_two_ranks():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [subprocess.Popen([sys.executable, "-c", WORKER.format(root=ROOT, port=port, rank=r)],
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=120)
        finally:
            if p.poll() is None:
                p.kill()
        assert p.returncode == 0, e
        outs.append(o)
    for o in outs:
        line = [l for l in o.splitlines() if l.startswith("RESULT")][0]
        assert line == "RESULT [2.0, 10.0, 0.5]"


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks([3, 4.5]) == [3.0, 4.5]


def test_reference_arm_only_rank0_prints(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
