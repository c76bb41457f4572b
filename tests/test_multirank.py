"""Several ranks, one process each, two gloo ranks on the CPU (host-only
contexts plan without a GPU): independent per-rank batches reduced to the
job's throughput (the sum of the ranks' samples over the maximum of their
times), and one caller batch split over the ranks by LPT with the per-unit
results gathered back in the caller's order."""
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


# ----------------------------------------------------------------------------- one batch split over ranks
def test_lpt_partition_balances_and_is_deterministic():
    from emri_kludge_suite_b200 import shard

    rng = np.random.default_rng(5)
    for parts in (2, 3, 8):
        c = rng.pareto(1.5, 200) + 0.1
        a, load = shard.lpt_partition(c, parts)
        assert a.min() >= 0 and a.max() < parts
        assert np.allclose(load, [c[a == k].sum() for k in range(parts)])
        a2, _ = shard.lpt_partition(c, parts)
        assert np.array_equal(a, a2)  # a pure function of the costs
        lower = max(c.max(), c.sum() / parts)
        assert load.max() <= 4.0 / 3.0 * lower + 1e-9 or load.max() <= c.max() + c.sum() / parts
    # equal costs (templates of one likelihood batch): counts differ by at most one
    a, _ = shard.lpt_partition(np.ones(4097), 8)
    counts = np.bincount(a, minlength=8)
    assert counts.max() - counts.min() <= 1
    # ties go to the lowest index; decreasing cost order
    a, load = shard.lpt_partition([5.0, 3.0, 3.0, 2.0, 2.0, 2.0, 1.0], 2)
    assert list(a) == [0, 1, 1, 0, 1, 0, 1] and list(load) == [9.0, 9.0]


SPLIT_N = 7


def _split_batch():
    from emri_kludge_suite_b200.workloads import SEED, config1

    src, _ = config1(SEED, SPLIT_N)
    return [dict(p, length=min(p["length"], 30000 + 5000 * k)) for k, p in enumerate(src)]


def _plan_rows(params, nthreads=2):
    """Per-source plan results of a host-only context: length, status, i_plunge, i_buffer."""
    import emri_kludge_suite_b200 as E
    from emri_kludge_suite_b200.workloads import NMODES

    wb = E.WaveBatch(-1)
    wb.plan(params, nmodes=NMODES, nthreads=nthreads)
    lens = np.diff(wb.offsets)
    return np.stack([lens, wb.status, wb.i_plunge, wb.i_buffer], axis=1).astype(np.float64)


def _template_rows(params):
    """(4<h|d>, 4<h|h>) of short templates on the CPU (the product's host front
    end, the oracle waveform, an rFFT inner product with a fixed data vector):
    stands in for a rank's device likelihoods, which gather the same way."""
    import emri_kludge_suite_b200 as E
    from oracle import oracle as O

    out = []
    for p in params:
        q = dict(p, length=2000)
        q["T"] = q["length"] * q["dt"] / O.YEAR
        m = E.front_end(q)
        mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
        _, hI, hII, _, _ = O.oracle_genwave(q, mt, 10)
        fI, fII = np.fft.rfft(hI), np.fft.rfft(hII)
        d = np.cos(np.arange(len(fI)) * 0.01) + 0j
        out.append([4.0 * np.real(np.vdot(fI, d) + np.vdot(fII, d)), 4.0 * np.real(np.vdot(fI, fI) + np.vdot(fII, fII))])
    return np.array(out)


def _split_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    from emri_kludge_suite_b200 import shard
    from emri_kludge_suite_b200.workloads import NMODES

    params = _split_batch()
    costs = shard.source_costs(params, NMODES)
    idx = shard.rank_indices(costs, rank, world)
    mine = [params[i] for i in idx]
    plan = shard.gather_rows(_plan_rows(mine) if mine else np.zeros((0, 4)), idx, len(params))
    like = shard.gather_rows(_template_rows(mine) if mine else np.zeros((0, 2)), idx, len(params))
    q.put((rank, idx.tolist(), plan, like))
    dist.destroy_process_group()


def test_two_ranks_split_one_batch_and_gather():
    """The union of the ranks' LPT shards is the caller's batch, and the
    gathered per-source plan rows and per-template likelihood rows equal a
    single process's results for the same list, in the caller's order."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    idx0, idx1 = set(res[0][1]), set(res[1][1])
    assert idx0 and idx1 and not (idx0 & idx1) and idx0 | idx1 == set(range(SPLIT_N))
    params = _split_batch()
    single_plan = _plan_rows(params)
    single_like = _template_rows(params)
    for _, _, plan, like in res:
        assert np.array_equal(plan, single_plan)
        assert np.array_equal(like, single_like)
