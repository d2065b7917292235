"""Replica jobs across ranks (feicar3d_3.0_febio_b200/replicas.py), run as
two gloo processes on the CPU: the split of a batch's problems between
ranks covers every problem once and balances the ranks, and the
measurement collectives (barrier, maximum and sum over ranks) give every
rank the same job time and total.  On GPUs the same calls run over NCCL in
bench.py (--gpus N), one process per GPU."""
import datetime
import importlib.util
import multiprocessing as mp
import os
import socket

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
_spec = importlib.util.spec_from_file_location(
    "fg_replicas", os.path.join(HERE, "..", "feicar3d_3.0_febio_b200", "replicas.py"))
replicas = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(replicas)

COSTS = [float(e) ** 3 for e in (81, 96, 63, 45, 32, 37, 59, 36, 43, 35, 38, 53, 55, 133, 70, 61, 48, 166,
                                 93, 47, 90, 63, 32, 59, 57, 139, 43, 34, 138, 143, 49, 111)]


def test_shard_balanced_covers_and_balances():
    for world in (1, 2, 3, 8):
        sh = replicas.shard_balanced(COSTS, world)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(COSTS)))
        loads = [sum(COSTS[i] for i in s) for s in sh]
        # greedy largest-first: no rank exceeds the mean by more than the largest problem
        assert max(loads) <= sum(COSTS) / world + max(COSTS)
    assert replicas.shard_balanced(COSTS, 2) == replicas.shard_balanced(list(COSTS), 2)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    spec = importlib.util.spec_from_file_location(
        "fg_replicas", os.path.join(HERE, "..", "feicar3d_3.0_febio_b200", "replicas.py"))
    rp = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rp)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    R = rp.Ranks(dist)
    mine = rp.shard_balanced(COSTS, R.world)[R.rank]
    R.barrier()
    t_mine = sum(COSTS[i] for i in mine) * 1e-6  # this rank's stand-in "time"
    t_job = R.max(t_mine)
    n_job = R.sum(len(mine))
    R.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, t_mine, t_job, n_job))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_split_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(2):
            rank, mine, t_mine, t_job, n_job = q.get(timeout=120)
            out[rank] = (mine, t_mine, t_job, n_job)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert sorted(out) == [0, 1]
    assert sorted(out[0][0] + out[1][0]) == list(range(len(COSTS)))
    assert out[0][2] == out[1][2] == pytest.approx(max(out[0][1], out[1][1]))
    assert out[0][3] == out[1][3] == len(COSTS)
