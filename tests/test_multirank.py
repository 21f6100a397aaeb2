"""The multi-GPU decomposition of bench.py, run as two gloo ranks on the CPU
with the oracle standing in for each rank's GPU: the disjoint realisation
ranges of the ranks, all-reduced, give the same sums as one solve of all of
them (the realisation streams are keyed by realisation id), and the timing
reduction takes the max over ranks. Then the library's own merge: the
ranks' tally vectors all-reduced over gloo and turned into one estimator by
ssol_b200_estimator_create_from_tallies, which needs no GPU."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "solstice-solver_b200"))

N = 40000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sums(est):
    """(sum w, sum w^2) of every global estimate, from (E, V, SE)."""
    n = est.count("realisation_count")
    out = []
    for k, (e, v, se) in sorted(est.globals().items()):
        out += [e * n, (v + e * e) * n]
    return out


def _rank(rank, world, port, oracle_path, q):
    import torch
    import torch.distributed as dist
    import bench
    import pyssol as P
    import workloads as W
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port,
                            rank=rank, world_size=world)
    lib = P.Lib(oracle_path)
    s, _ = W.single_mirror(lib)
    rng = s.rng(seed=7, position=bench.shard_first(0, rank, world, N))
    est = s.solve(N, rng=rng)
    t = torch.tensor(_sums(est), dtype=torch.float64)
    dist.all_reduce(t)
    ms = torch.tensor([10.0 * (rank + 1)], dtype=torch.float64)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    suns = bench.shard_suns(list(range(256)), rank, world)
    cover = torch.zeros(256, dtype=torch.int64)
    cover[suns] = 1
    dist.all_reduce(cover)
    if rank == 0:
        q.put((t.tolist(), float(ms[0]), cover.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_match_one_solve(oracle):
    import torch.multiprocessing as mp
    import pyssol as P
    import workloads as W
    from conftest import ORACLE_LIB
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, ORACLE_LIB, q)) for r in range(2)]
    for p in procs:
        p.start()
    sums, ms, cover = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    s, _ = W.single_mirror(oracle)
    ref = _sums(s.solve(2 * N, rng=s.rng(seed=7)))
    for a, b in zip(sums, ref):
        assert a == pytest.approx(b, rel=1e-9, abs=1e-6)
    assert ms == 20.0
    assert cover == [1] * 256


def _merge_rank(rank, world, port, product_path, q):
    """One rank of the tally merge through the library's own entries: the
    rank's tally vectors (pairs of sum w and sum w^2, here drawn from seeded
    weights, as a GPU's plan would hold them) are all-reduced over gloo and
    rank 0 builds the merged estimator with
    ssol_b200_estimator_create_from_tallies."""
    import random
    import torch
    import torch.distributed as dist
    import pyssol as P
    import workloads as W
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port,
                            rank=rank, world_size=world)
    lib = P.Lib(product_path)
    s, h = W.heliostat_field(lib, n_helio=30, receiver_cells=4)
    ns, nc = P.tallies_size(s)
    rnd = random.Random(1000 + rank)
    sums = []
    for _ in range(ns // 2):
        w = [rnd.uniform(0.0, 10.0) for _ in range(3)]
        sums += [sum(w), sum(x * x for x in w)]
    t = torch.tensor(sums, dtype=torch.float64)
    c = torch.zeros(nc, dtype=torch.int64)
    gathered = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(gathered, t)
    dist.all_reduce(t)
    dist.all_reduce(c)
    if rank == 0:
        rng = s.rng(seed=3)
        n_rank = 1000
        merged = P.estimator_from_tallies(s, rng, world * n_rank, t.tolist(), c.tolist())
        parts = [P.estimator_from_tallies(s, rng, n_rank, g.tolist(), c.tolist())
                 for g in gathered]
        q.put((merged.count("realisation_count"), merged.globals(),
               merged.receiver(h["receiver"]), [p.globals() for p in parts],
               [p.receiver(h["receiver"]) for p in parts], t[:12].tolist(), n_rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_merge_tallies_through_the_library(product):
    """The merged estimator of two ranks' all-reduced tallies: N = N0 + N1
    realisations, E the pooled mean (N0 E0 + N1 E1) / N, and every global
    estimate equal to the one computed from the summed vectors."""
    import torch.multiprocessing as mp
    import pyssol as P
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_merge_rank, args=(r, 2, port, P.PRODUCT_LIB, q))
             for r in range(2)]
    for p in procs:
        p.start()
    count, g, rcv, pg, prcv, gsum, n = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert count == 2 * n
    for i, k in enumerate(P.GLOBAL_FIELDS):
        assert g[k][0] == pytest.approx(gsum[2 * i] / (2 * n), rel=1e-12)
        assert g[k][0] == pytest.approx((pg[0][k][0] + pg[1][k][0]) / 2, rel=1e-12)
    for k in rcv:
        assert rcv[k][0] == pytest.approx((prcv[0][k][0] + prcv[1][k][0]) / 2, rel=1e-12)
