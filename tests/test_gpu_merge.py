"""Merging tallies across GPUs through the library: two plans of the
1000-heliostat field trace disjoint realisation ranges, as two GPUs of a
multi-GPU solve would. Their device tally vectors (ssol_b200_plan_get_tallies)
added in place, as an all-reduce over NVLink leaves them, give through
ssol_b200_plan_finish the estimator of one plan that traced both ranges; the
host route (vectors copied out, added, ssol_b200_estimator_create_from_tallies)
gives the same. Only the order of the FP64 sums differs: 1e-10 relative."""
import ctypes as C

import pytest
import torch

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu


def _plan(lib, s):
    plan = C.c_void_p()
    lib.call("ssol_b200_plan_create", s.scn, None, C.byref(plan))
    return plan


def _finish(lib, s, plan, rng, n):
    est = C.c_void_p()
    res = lib.raw("ssol_b200_plan_finish", plan, rng, n, 0, None, C.byref(est))
    assert res == P.RES_OK
    return P.Estimator(s, est, res)


def _same(a, b, what):
    for k in b:
        assert a[k][0] == pytest.approx(b[k][0], rel=1e-10, abs=1e-9), (what, k)
        assert a[k][2] == pytest.approx(b[k][2], rel=1e-6, abs=1e-9), (what, k)


def test_merged_plans_equal_one_plan(product):
    s, h = W.heliostat_field(product, receiver_cells=32)
    rng = s.rng(seed=17)
    n = 3_000_000
    a, b, ref = _plan(product, s), _plan(product, s), _plan(product, s)
    product.call("ssol_b200_plan_launch", a, rng, 0, n, None)
    product.call("ssol_b200_plan_launch", b, rng, n, n, None)
    product.call("ssol_b200_plan_launch", ref, rng, 0, 2 * n, None)
    torch.cuda.synchronize()
    sa, ca = (torch.as_tensor(x, device="cuda") for x in P.plan_tallies(product, a))
    sb, cb = (torch.as_tensor(x, device="cuda") for x in P.plan_tallies(product, b))
    host_sums = (sa + sb).cpu().tolist()
    host_counts = (ca + cb).cpu().tolist()
    sa += sb
    ca += cb
    torch.cuda.synchronize()
    merged = _finish(product, s, a, rng, 2 * n)
    one = _finish(product, s, ref, rng, 2 * n)
    assert merged.count("realisation_count") == one.count("realisation_count") == 2 * n
    _same(merged.globals(), one.globals(), "globals")
    _same(merged.receiver(h["receiver"]), one.receiver(h["receiver"]), "receiver")
    pm = merged.primitives(h["receiver"], h["receiver_shape"])
    po = one.primitives(h["receiver"], h["receiver_shape"])
    for i in range(0, len(po), 97):
        _same(pm[i], po[i], "primitive %d" % i)
    for k in (0, 500, 999):
        assert merged.sampled(h["heliostats"][k])["nb_samples"] == \
            one.sampled(h["heliostats"][k])["nb_samples"]
    via_host = P.estimator_from_tallies(s, rng, 2 * n, host_sums, host_counts)
    assert via_host.count("realisation_count") == 2 * n
    _same(via_host.globals(), one.globals(), "host globals")
    _same(via_host.receiver(h["receiver"]), one.receiver(h["receiver"]), "host receiver")
    for p in (a, b, ref):
        product.raw("ssol_b200_plan_ref_put", p)
