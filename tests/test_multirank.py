"""The multi-GPU decomposition of bench.py, run as two gloo ranks on the CPU
with the oracle standing in for each rank's GPU: the disjoint realisation
ranges of the ranks, all-reduced, give the same sums as one solve of all of
them (the realisation streams are keyed by realisation id), and the timing
reduction takes the max over ranks."""
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
