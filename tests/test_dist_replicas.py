"""Multi-rank plumbing of bench.py on the CPU (gloo, world size 2): every
rank runs an independent replica; the job's time is the max over ranks and
its work the sum, as the driver's scaling runs compute them."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(backend="gloo")
    d.barrier()
    t = d.max(1.0 + rank)          # per-rank "device time"
    w = d.sum(10.0 * (rank + 1))   # per-rank work
    d.close()
    q.put((rank, t, w))


def test_replicas_max_time_sum_work():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r[1] for r in res] == [2.0, 2.0]
    assert [r[2] for r in res] == [30.0, 30.0]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "librefemu.so")),
                    reason="oracle/_ref not built")
def test_reference_arm_line():
    """bench.py --impl reference prints one JSON line with the contract's keys"""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "3", "--n", "256"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "impl", "cpu_baseline", "e2e"):
        assert k in line
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
