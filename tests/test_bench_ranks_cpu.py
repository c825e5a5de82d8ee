"""The multi-process plumbing of bench.py on CPU: two ranks over gloo on
127.0.0.1 (one process per rank, as torchrun starts them on GPUs) take the
maximum of their elapsed times, pass the barrier, and report the whole-job
seconds per update for the updates all ranks ran. The replicas share no data
path, so nothing else crosses between ranks."""
import json
import os
import socket
import subprocess
import sys
import textwrap

from conftest import ROOT

CHILD = textwrap.dedent("""
    import json, sys
    sys.path.insert(0, {root!r})
    import bench
    world, rank, local = bench.dist_setup(2, backend="gloo")
    elapsed = [40.0, 55.0][rank]          # ms of K updates on this rank
    bench.barrier(world)
    worst = bench.max_over_ranks(world, elapsed)
    value = bench.job_seconds_per_update(worst, 10, world)
    print(json.dumps({{"rank": rank, "world": world, "max_ms": worst, "value": value}}))
    import torch.distributed as dist
    dist.destroy_process_group()
""")


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_max_and_the_job_value():
    port = _port()
    code = CHILD.format(root=str(ROOT))
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["max_ms"] == 55.0                     # the slowest rank bounds the job
        assert abs(o["value"] - 55.0e-3 / 20) < 1e-15  # 2 ranks x 10 updates in 55 ms
    assert sorted(o["rank"] for o in outs) == [0, 1]
