"""The multi-rank plumbing of bench.py on the CPU with two gloo ranks: every rank takes the
same collective steps, the timing is the maximum over ranks, and under `--impl reference`
only rank 0 works and prints (the others exit 0 at once).  The GPU path runs one replica per
rank with no data-path collective, so these steps are all it has."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys, json, datetime
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
world, rank, local = bench.dist_setup()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
times = [0.25, 0.75]
got = bench.max_over_ranks(times[rank], world, device="cpu")
dist.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": rank, "max": got}))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn(code, world, extra=None):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r),
                   WORLD_SIZE=str(world), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, "-c", code, ROOT] + (extra or []),
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    out = []
    for p in procs:
        o, e = p.communicate(timeout=240)
        assert p.returncode == 0, e[-2000:]
        out.append(o)
    return out


def test_max_over_ranks_gloo():
    outs = spawn(CHILD, 2)
    for o in outs:
        rec = json.loads(o.strip().splitlines()[-1])
        assert rec["max"] == 0.75


def test_max_over_ranks_single():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(1.5, 1) == 1.5


def test_reference_arm_other_ranks_exit():
    """Rank 1 of a two-rank `--impl reference` launch returns 0 without work or output."""
    code = r"""
import sys
sys.path.insert(0, sys.argv[1])
sys.argv = ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
import bench
sys.exit(bench.run_reference(bench.parse()))
"""
    port = free_port()
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="1",
               WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, "-c", code, ROOT], env=env, capture_output=True,
                       text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
