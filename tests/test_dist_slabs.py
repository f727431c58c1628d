"""Row-slab decomposition of one grid across ranks, on the CPU (gloo): the
multi-GPU split of a single large scenario, with the FP64 oracle's
arithmetic.  Each rank updates one slab of rows; after phase 1 it sends its
first and last two rows of the new depth to its neighbours and receives
theirs (the stencil reaches two rows), after phase 2 the same for the
discharges, and every rank steps with the minimum of the ranks' next dt (one
all-reduce per step).  The decomposed run must give bitwise the state of the
same stepper updating every row in one process, which in turn gives the
oracle's own run (thy_oracle_run) bitwise."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 40
FIELDS = ("h", "qx", "qy", "eta_max", "t_arr")


def _problem():
    sys.path.insert(0, os.path.join(ROOT, "tsunami-hysea_b200"))
    from thysea import synth

    # open borders (sponges at the top and bottom slabs' outer rows), a
    # shelf with dry land, one fault at t = 0
    p = synth.plain_small(nx=96, ny=83, seed=11, sim_time=3600.0, save_time=-1.0, npoints=0)
    p.name = "slabs"
    return p


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      OMP_NUM_THREADS="1")
    for d in (ROOT, os.path.join(ROOT, "oracle")):
        sys.path.insert(0, d)
    import datetime

    import torch
    import torch.distributed as dist

    import oracle

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    p = _problem()

    def exchange(name, arr, lo, hi):
        # rows lo, lo+1 go up to rank-1 (its lower halo), rows hi-2, hi-1 down
        # to rank+1 (its upper halo); the halos come back the same way
        reqs, bufs = [], []
        if rank > 0:
            reqs.append(dist.isend(torch.from_numpy(arr[lo:lo + 2].copy()), rank - 1))
            up = torch.empty((2, arr.shape[1]), dtype=torch.float64)
            reqs.append(dist.irecv(up, rank - 1))
            bufs.append((lo - 2, up))
        if rank < world - 1:
            reqs.append(dist.isend(torch.from_numpy(arr[hi - 2:hi].copy()), rank + 1))
            down = torch.empty((2, arr.shape[1]), dtype=torch.float64)
            reqs.append(dist.irecv(down, rank + 1))
            bufs.append((hi, down))
        for r in reqs:
            r.wait()
        for row, b in bufs:
            arr[row:row + 2] = b.numpy()

    def allreduce_min(v):
        t = torch.tensor([v], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        return float(t.item())

    s = oracle.run_slabs(p, rank, world, STEPS, exchange, allreduce_min)
    q.put((rank, s.row_lo, s.row_hi, {k: s.field(k)[s.row_lo:s.row_hi].copy() for k in FIELDS}, s.t))
    s.close()
    dist.barrier()
    dist.destroy_process_group()


def _single():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    p = _problem()
    s = oracle.run_slabs(p, 0, 1, STEPS, lambda *a: None, lambda v: v)
    return p, s


@pytest.mark.parametrize("world", [2, 3])
def test_row_slabs_match_one_process_bitwise(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    p, ref = _single()
    times = {g[4] for g in got}
    assert times == {ref.t}   # every rank took the same time steps as the single process
    rows = sorted((g[1], g[2]) for g in got)
    assert rows[0][0] == 0 and rows[-1][1] == p.ny and all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
    for rank, lo, hi, fields, _ in got:
        for k in FIELDS:
            assert np.array_equal(fields[k], ref.field(k)[lo:hi]), (world, rank, k)
    # the wave has moved: the comparison is not of an untouched state
    assert np.abs(ref.field("qx")).max() > 0
    ref.close()


def test_single_process_slab_is_the_oracle_run():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    p, s = _single()
    r = oracle.run_oracle(p, max_iterations=STEPS)
    assert r["iterations"] == STEPS
    assert abs(r["final_time"] - s.t * s.Ts) <= 1e-9 * r["final_time"]
    em = s.field("eta_max")
    maxh = np.where(em < -1e20, -9999.0, (em - s.Hmin) * s.Hs).astype(np.float32)
    assert np.array_equal(maxh, r["max_height"])
    s.close()
