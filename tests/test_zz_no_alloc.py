"""The no-allocation batched launch (ssol_b200_batch_launch_noalloc).

It exists for callers that must not have device memory allocated for them
while they launch: code that owns every device allocation through its own
pool, or a real-time loop whose rules forbid allocating. Its kernel scratch
sits in a static device array sized for at most 4096 items. Through the
C-ABI, calls in a row must reproduce what the regular ssol_b200_batch_launch
gives on the same batch and streams, item by item, within the tolerance of
the other GPU tests (3 combined standard errors with a 1e-6 relative floor),
also when batches of different sizes take turns in the shared array; a batch
above the limit gets RES_BAD_ARG. Collected last so that a failure here never
hides the other tests' results."""
import math

import pytest

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu

NOALLOC_MAX_ITEMS = 4096


def close(a, b):
    return abs(a[0] - b[0]) <= 3 * math.hypot(a[2], b[2]) + 1e-6 * max(1.0, abs(b[0]))


def assert_items_match(fields, got, ref, budgets, what):
    for (s, h), a, b, n in zip(fields, got, ref, budgets):
        assert a.count("realisation_count") == b.count("realisation_count") == n
        ga, gb = a.globals(), b.globals()
        bad = [k for k in gb if not close(ga[k], gb[k])]
        assert not bad, (what, bad, ga, gb)
        ra, rb = a.receiver(h["receiver"]), b.receiver(h["receiver"])
        bad = [k for k in rb if not close(ra[k], rb[k])]
        assert not bad, (what, bad, ra, rb)


SUNS = [{"elevation": 35.0, "azimuth": 170.0, "dni": 850.0},
        {"elevation": 55.0, "azimuth": 120.0, "dni": 650.0},
        {"elevation": 20.0, "azimuth": 220.0, "dni": 500.0},
        {"elevation": 70.0, "azimuth": 300.0, "dni": 950.0}]


def test_noalloc_launch_matches_regular_launch(product):
    fields = W.batched_fields(product, SUNS[:3], n_helio=40, receiver_cells=8)
    scenes = [f[0] for f in fields]
    regular = P.Batch(product, scenes)
    noalloc = P.Batch(product, scenes)
    rng = scenes[0].rng(seed=33)
    budgets = [40000, 15000, 25000]
    for call in range(2):
        regular.reset()
        noalloc.reset()
        regular.launch(rng, budgets)
        noalloc.launch_noalloc(rng, budgets)
        assert_items_match(fields, noalloc.finish(rng), regular.finish(rng), budgets,
                           "call %d" % call)
    regular.close()
    noalloc.close()


def test_noalloc_batches_of_different_sizes_in_turn(product):
    """A 4-item batch, then a 2-item batch, then the 4-item one again, all
    through the shared array: a stale prefix, first id or work counter left
    by the previous call would show as a wrong realisation count or estimate."""
    big_f = W.batched_fields(product, SUNS, n_helio=30, receiver_cells=8)
    small_f = W.batched_fields(product, SUNS[2:0:-1], n_helio=30, receiver_cells=8)
    big_s, small_s = [f[0] for f in big_f], [f[0] for f in small_f]
    big_budgets, small_budgets = [30000, 5000, 20000, 12000], [7000, 26000]
    rng = big_s[0].rng(seed=71)
    runs = []
    for fields, scenes, budgets in ((big_f, big_s, big_budgets),
                                    (small_f, small_s, small_budgets),
                                    (big_f, big_s, big_budgets)):
        noalloc = P.Batch(product, scenes)
        noalloc.launch_noalloc(rng, budgets)
        runs.append((fields, scenes, budgets, noalloc.finish(rng)))
        noalloc.close()
    for k, (fields, scenes, budgets, got) in enumerate(runs):
        regular = P.Batch(product, scenes)
        regular.launch(rng, budgets)
        assert_items_match(fields, got, regular.finish(rng), budgets, "run %d" % k)
        regular.close()


def test_noalloc_rejects_batches_above_its_limit(product):
    """NOALLOC_MAX_ITEMS + 1 items (one small scene repeated): RES_BAD_ARG,
    and the regular launch of the same batch still works."""
    s, h = W.single_mirror(product)
    batch = P.Batch(product, [s] * (NOALLOC_MAX_ITEMS + 1))
    rng = s.rng(seed=5)
    budgets = (P.C.c_uint64 * (NOALLOC_MAX_ITEMS + 1))(*([1] * (NOALLOC_MAX_ITEMS + 1)))
    res = product.raw("ssol_b200_batch_launch_noalloc", batch.h, rng, budgets, None)
    assert res == P.RES_BAD_ARG
    batch.close()
    small = P.Batch(product, [s] * 3)
    small.launch_noalloc(rng, [1000, 2000, 3000])
    ests = small.finish(rng)
    assert [e.count("realisation_count") for e in ests] == [1000, 2000, 3000]
    small.close()
