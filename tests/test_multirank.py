"""Sharding across ranks, as bench.py runs it under torchrun: every rank plans
its own seeded batch (no data exchange), and the job's throughput is the sum
of the ranks' samples over the maximum of their times.  Two gloo ranks on the
CPU, planning in host-only contexts."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

N_SRC = 6


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _plan_rank(rank):
    import emri_kludge_suite_b200 as E
    from emri_kludge_suite_b200.workloads import NMODES, SEED, config1

    src, _ = config1(SEED + rank, N_SRC)
    src = [dict(p, length=min(p["length"], 40000)) for p in src]  # keep the host planning short
    wb = E.WaveBatch(-1)
    wb.plan(src, nmodes=NMODES, nthreads=2)
    return wb.total_samples, wb.status.copy(), src


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    n, status, src = _plan_rank(rank)
    fake_ms = 100.0 + 10.0 * rank  # a rank's device time
    t = torch.tensor([fake_ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tot = torch.tensor([float(n)], dtype=torch.float64)
    dist.all_reduce(tot)
    first = torch.tensor([src[0]["M"]], dtype=torch.float64)
    gathered = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(gathered, first)
    q.put((rank, n, int(np.sum(status != 0)), float(t.item()), float(tot.item()), [float(g.item()) for g in gathered]))
    dist.destroy_process_group()


def test_two_ranks_shard_without_exchange():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    per_rank = {r: n for r, n, *_ in res}
    assert all(failed == 0 for _, _, failed, *_ in res)
    for _, _, _, tmax, tsum, firsts in res:
        assert tmax == 110.0  # max over ranks, as the bench reports
        assert tsum == float(per_rank[0] + per_rank[1])  # whole-job samples
        assert firsts[0] != firsts[1]  # each rank has its own seeded shard
    # a rank's shard does not depend on the others: same totals planned alone
    assert _plan_rank(1)[0] == per_rank[1]
