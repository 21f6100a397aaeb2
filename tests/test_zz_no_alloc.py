"""The no-allocation batched launch (ssol_b200_batch_launch_noalloc).

It exists for callers that must not have device memory allocated for them
while they launch (their own memory pool, a capture region or a real-time
loop): its kernel scratch sits in a static device array sized for at most
4096 items. Through the C-ABI, two calls in a row must reproduce what the
regular ssol_b200_batch_launch gives on the same batch and streams, item by
item, within the tolerance of the other GPU tests (3 combined standard
errors with a 1e-6 relative floor). Collected last so that a failure here
never hides the other tests' results."""
import math

import pytest

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu


def close(a, b):
    return abs(a[0] - b[0]) <= 3 * math.hypot(a[2], b[2]) + 1e-6 * max(1.0, abs(b[0]))


def test_noalloc_launch_matches_regular_launch(product):
    suns = [{"elevation": 35.0, "azimuth": 170.0, "dni": 850.0},
            {"elevation": 55.0, "azimuth": 120.0, "dni": 650.0},
            {"elevation": 20.0, "azimuth": 220.0, "dni": 500.0}]
    fields = W.batched_fields(product, suns, n_helio=40, receiver_cells=8)
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
        ref = regular.finish(rng)
        got = noalloc.finish(rng)
        for (s, h), a, b, n in zip(fields, got, ref, budgets):
            assert a.count("realisation_count") == b.count("realisation_count") == n
            ga, gb = a.globals(), b.globals()
            bad = [k for k in gb if not close(ga[k], gb[k])]
            assert not bad, ("call %d" % call, bad, ga, gb)
            ra, rb = a.receiver(h["receiver"]), b.receiver(h["receiver"])
            bad = [k for k in rb if not close(ra[k], rb[k])]
            assert not bad, ("call %d" % call, bad, ra, rb)
    regular.close()
    noalloc.close()
