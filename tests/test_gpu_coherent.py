"""Coherent order: a plain launch of at least 6e6 realisations is presorted
by sampled primitive (in chunks of 2^24) and handed to warps in strided
segments. It must trace exactly the realisations of the launch, each once with
its own stream, so the estimates equal those of the same range launched in id
order (launches below 6e6), up to the rounding of the FP64 sums in another
order."""
import ctypes as C

import pytest

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu

CHUNK = 1 << 24


def _run(lib, s, launches, nreal):
    opt = P.options(P.FP32, count=1)
    plan = C.c_void_p()
    lib.call("ssol_b200_plan_create", s.scn, C.byref(opt), C.byref(plan))
    try:
        rng = s.rng(seed=11)
        for first, count in launches:
            lib.call("ssol_b200_plan_launch", plan, rng, first, count, None)
        est = C.c_void_p()
        lib.call("ssol_b200_plan_finish", plan, rng, nreal, 0, None, C.byref(est))
        e = P.Estimator(s, est, P.RES_OK)
        return e
    finally:
        lib.raw("ssol_b200_plan_ref_put", plan)


def test_sorted_launch_equals_id_order(product):
    s, h = W.heliostat_field(product)
    n = CHUNK + 12345  # two sorted chunks, the second one short
    sorted_est = _run(product, s, [(0, n)], n)
    step = (1 << 20) - 1  # below the sort threshold: id order
    id_est = _run(product, s, [(f, min(step, n - f)) for f in range(0, n, step)], n)
    g1, g2 = sorted_est.globals(), id_est.globals()
    for k in g1:
        e1, _, se1 = g1[k]
        e2, _, se2 = g2[k]
        assert e1 == pytest.approx(e2, rel=1e-10, abs=1e-9), k
        assert se1 == pytest.approx(se2, rel=1e-6, abs=1e-7 * abs(e1) + 1e-9), k
    r1, r2 = sorted_est.receiver(h["receiver"]), id_est.receiver(h["receiver"])
    for k in r1:
        assert r1[k][0] == pytest.approx(r2[k][0], rel=1e-10, abs=1e-9), k
    p1 = sorted_est.primitives(h["receiver"], h["receiver_shape"])
    p2 = id_est.primitives(h["receiver"], h["receiver_shape"])
    for a, b in zip(p1, p2):
        assert a["absorbed_flux"][0] == pytest.approx(b["absorbed_flux"][0], rel=1e-9,
                                                      abs=1e-6)
    st1, st2 = sorted_est.stats(), id_est.stats()
    assert st1["paths"] == st2["paths"] == n
    for k in ("rays", "node_visits", "triangle_tests", "bounces"):
        assert st1[k] == st2[k], k
    s.close()
