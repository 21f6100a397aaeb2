"""Batched form: several sun positions (each its own re-aimed field) in one
persistent launch replayed from a CUDA graph must give, item by item, the
estimates of a plain ssol_solve of the same scene on the same realisation
streams (3 combined standard errors, 1e-6 relative floor)."""
import math

import pytest

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu


def close(a, b):
    return abs(a[0] - b[0]) <= 3 * math.hypot(a[2], b[2]) + 1e-6 * max(1.0, abs(b[0]))


def test_batch_matches_plain_solves(product):
    suns = [{"elevation": 30.0, "azimuth": 180.0, "dni": 900.0},
            {"elevation": 60.0, "azimuth": 90.0, "dni": 700.0},
            {"elevation": 15.0, "azimuth": 270.0, "dni": 400.0},
            {"elevation": 80.0, "azimuth": 0.0, "dni": 1000.0}]
    fields = W.batched_fields(product, suns, n_helio=60, receiver_cells=8)
    scenes = [f[0] for f in fields]
    batch = P.Batch(product, scenes)
    rng = scenes[0].rng(seed=21)
    budgets = [30000, 100000, 50000, 20000]
    batch.launch(rng, budgets)
    extra = [10000, 0, 25000, 5000]
    batch.launch(rng, extra)
    ests = batch.finish(rng)
    for (s, h), est, n0, n1 in zip(fields, ests, budgets, extra):
        n = n0 + n1
        assert est.count("realisation_count") == n
        ref = s.solve(n, rng=rng)
        g, gr = est.globals(), ref.globals()
        bad = [k for k in g if not close(g[k], gr[k])]
        assert not bad, (bad, g, gr)
        r, rr = est.receiver(h["receiver"]), ref.receiver(h["receiver"])
        bad = [k for k in r if not close(r[k], rr[k])]
        assert not bad, (bad, r, rr)
        # same streams: means agree far below one standard error
        assert abs(r["absorbed_flux"][0] - rr["absorbed_flux"][0]) <= \
            0.05 * rr["absorbed_flux"][2] + 1e-9 * abs(rr["absorbed_flux"][0])
    batch.reset()
    batch.launch(rng, budgets)
    again = batch.finish(rng)
    for est, n in zip(again, budgets):
        assert est.count("realisation_count") == n
    batch.close()


def test_autotune_picks_a_valid_shape(product):
    """ssol_b200_autotune returns one of its candidate shapes, and a solve
    with it agrees with the default shape within 3 combined SE."""
    s, h = W.heliostat_field(product, n_helio=120, receiver_cells=16)
    opt, ms = P.autotune(s, 500000)
    assert ms > 0
    assert opt.block_size in (128, 256)
    assert opt.min_blocks_per_sm in (1, 2, 3)
    assert opt.waves in (1, 2)
    assert opt.bvh_leaf_size in (1, 2, 4)
    # the builder is the caller's choice, kept as given (default: by solve size)
    assert opt.bvh_builder == P.BVH_AUTO
    a = s.solve(2000000, seed=4, options=opt).globals()
    b = s.solve(2000000, seed=4).globals()
    for k in b:
        assert P.combined_ok(a[k], b[k], floor=1e-6 * abs(b[k][0])), k


def test_batch_coherent_order_equals_plain_solves(product):
    """Launches of at least 2^22 realisations run in the coherent order
    (per item, sorted by sampled primitive, handed out in strided segments);
    each realisation keeps its stream and primary draw, so the items must
    equal plain solves of the same realisations to the order of the FP64
    sums. The second, small launch runs in id order through another
    captured graph and adds to the same tallies."""
    suns = [{"elevation": 30.0, "azimuth": 180.0, "dni": 900.0},
            {"elevation": 60.0, "azimuth": 90.0, "dni": 700.0},
            {"elevation": 15.0, "azimuth": 270.0, "dni": 400.0},
            {"elevation": 80.0, "azimuth": 0.0, "dni": 1000.0}]
    fields = W.batched_fields(product, suns, n_helio=60, receiver_cells=8)
    scenes = [f[0] for f in fields]
    batch = P.Batch(product, scenes)
    rng = scenes[0].rng(seed=33)
    budgets = [1_500_000, 1_000_000, 1_200_000, 800_123]
    assert sum(budgets) >= 1 << 22
    batch.launch(rng, budgets)
    extra = [50000, 0, 7, 31000]
    batch.launch(rng, extra)
    ests = batch.finish(rng)
    for (s, h), est, n0, n1 in zip(fields, ests, budgets, extra):
        n = n0 + n1
        ref = s.solve(n, rng=rng, max_failed=1 << 40)
        # the same paths: the same failures (a path that meets the segment
        # budget or overflows its receiver entries) as the plain solve
        for q in ("realisation_count", "failed_count"):
            assert est.count(q) == ref.count(q), (q, est.count(q), ref.count(q))
        assert est.count("realisation_count") + est.count("failed_count") == n
        for got, want in ((est.globals(), ref.globals()),
                          (est.receiver(h["receiver"]), ref.receiver(h["receiver"]))):
            for q in want:
                assert abs(got[q][0] - want[q][0]) <= \
                    1e-9 * max(1.0, abs(want[q][0])) + 1e-3 * want[q][2], (q, got[q], want[q])
        pg = est.primitives(h["receiver"], h["receiver_shape"])
        pr = ref.primitives(h["receiver"], h["receiver_shape"])
        for a, b in zip(pg, pr):
            for q in b:
                assert abs(a[q][0] - b[q][0]) <= 1e-9 * max(1.0, abs(b[q][0])) + 1e-3 * b[q][2]
    batch.close()
