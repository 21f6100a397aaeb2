"""Boundary cases of ssol_solve on the B200 library, against the oracle and
exact identities:
- realisation ids that cross 2^32 (the 64-bit Philox counter split into two
  words on the device);
- ragged realisation counts (1, 33, a prime above a million) and their
  exact realisation and sample counts;
- a scene without receivers (warning only; nothing is absorbed by receivers);
- the failure rule (src/ssol_solver.c:1240-1245, 1340): every path meets a
  dielectric whose outside medium is not the air; RES_BAD_OP with a valid
  estimator whatever max_failed_count, as on the oracle; once the limit is
  reached no new realisation is scheduled (src/ssol_solver.c:1229);
- a host-side abort of a running plan (ssol_b200_plan_abort);
- a 256 x 256 per-primitive receiver map (131072 triangles): the primitive
  estimates integrate to the receiver's, to rounding."""
import math

import pytest

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu


def close(a, b, k=3.0, floor=1e-6):
    return abs(a[0] - b[0]) <= k * math.hypot(a[2], b[2]) + floor * abs(b[0])


def test_realisation_ids_across_2_32(product, oracle):
    n = 120000
    start = (1 << 32) - n // 2
    outs = []
    for lib in (product, oracle):
        s, h = W.single_mirror(lib)
        rng = s.rng(seed=4, position=start)
        e = s.solve(n, rng=rng)
        outs.append((e.globals(), e.receiver(h["receiver"])))
    (gp, rp), (go, ro) = outs
    for k in go:
        assert close(gp[k], go[k]), k
    for k in ro:
        assert close(rp[k], ro[k]), k
    # the same ids give the same estimates (FP64 sums in another order)
    s, h = W.single_mirror(product)
    a = s.solve(n, rng=s.rng(seed=4, position=start)).receiver(h["receiver"])
    b = s.solve(n, rng=s.rng(seed=4, position=start)).receiver(h["receiver"])
    assert a["incoming_flux"][0] == pytest.approx(b["incoming_flux"][0], rel=1e-12)


@pytest.mark.parametrize("n", [1, 33, 1000003])
def test_ragged_counts(product, n):
    s, h = W.single_mirror(product)
    e = s.solve(n, seed=3)
    assert e.count("realisation_count") == n
    assert e.sampled(h["heliostat"])["nb_samples"] == n
    assert e.stats()["paths"] == n


def test_scene_without_receiver(product, oracle):
    outs = []
    for lib in (product, oracle):
        s = P.Scene(lib)
        m = s.mirror(0.9, 0.0)
        s.instance(s.object([(s.rectangle(5, 5), m, m)]))
        s.set_sun("directional", (0.3, 0.0, -1.0), 1000.0)
        outs.append(s.solve(50000, seed=6).globals())
    gp, go = outs
    assert gp["absorbed_by_receivers"][0] == 0.0
    for k in go:
        assert close(gp[k], go[k]), k


def _failing_scene(lib):
    """A virtual sampled plane above a plate whose material's outside medium is
    glass: a ray from the air meets it and fails (src/ssol_material.c:97-101)."""
    s = P.Scene(lib)
    air = s.medium(0.0, 1.0)
    glass = s.medium(0.0, 1.5)
    wrong = s.dielectric(glass, air)
    v = s.virtual()
    s.instance(s.object([(s.rectangle(5, 5), v, v)]), P.transform_from(None, (0, 0, 2.0)))
    s.instance(s.object([(s.rectangle(5, 5), wrong, wrong)]),
               P.transform_from(None, (0, 0, 1.0)), sample=0)
    s.set_sun("directional", (0, 0, -1), 1000.0)
    return s


@pytest.mark.parametrize("max_failed", [0, 10, 1 << 40])
def test_failure_rule(product, oracle, max_failed):
    n = 20000
    codes = []
    for lib in (product, oracle):
        s = _failing_scene(lib)
        e = s.solve(n, seed=2, max_failed=max_failed, check=False)
        assert e is not None
        codes.append(e.res)
        assert e.count("failed_count") > 0
    assert codes[0] == codes[1]
    assert codes[0] == (P.RES_BAD_OP if max_failed <= n else P.RES_OK)


def test_large_primitive_map(product):
    s2 = P.Scene(product)
    mirror = s2.mirror(0.9, 0.0)
    s2.instance(s2.object([(s2.rectangle(5, 5), mirror, mirror)]))
    shape = W.grid_mesh(s2, 4.0, 4.0, 256, 256)
    absorber = s2.matte(0.0)
    # sun 0.3 rad off the vertical; the receiver faces the mirror 20 m along
    # the reflected axis, out of the sun's way
    a = 0.3
    r = (-math.sin(a), 0.0, math.cos(a))  # reflection of the sun direction
    rcv = s2.instance(s2.object([(shape, absorber, absorber)]),
                      P.transform_from(W.frame_z_to(tuple(-c for c in r)),
                                       tuple(20.0 * c for c in r)),
                      receiver=P.SSOL_FRONT, per_primitive=1, sample=0)
    s2.set_sun("directional", (r[0], 0.0, -r[2]), 1000.0)
    e = s2.solve(2_000_000, seed=8)
    total = e.receiver(rcv)["incoming_flux"][0]
    prims = e.primitives(rcv, shape)
    assert len(prims) == 2 * 256 * 256
    cell = (4.0 / 256) ** 2 / 2
    integral = sum(p["incoming_flux"][0] for p in prims) * cell
    assert total > 0
    assert integral == pytest.approx(total, rel=1e-9)


def test_failure_limit_stops_the_work_fetch(product, oracle):
    """src/ssol_solver.c:1229, 1240-1248: once max_failed_count paths have
    failed, no new realisation is scheduled; the call returns RES_BAD_OP with
    an estimator counting only what ran. Every path of this scene fails."""
    n = 4_000_000
    for lib in (product, oracle):
        s = _failing_scene(lib)
        e = s.solve(n, seed=3, max_failed=10, check=False)
        assert e is not None and e.res == P.RES_BAD_OP
        failed, ran = e.count("failed_count"), e.count("realisation_count")
        assert failed >= 10
        assert failed + ran < n // 4, (failed, ran)
    # no limit reached: every realisation runs
    s = _failing_scene(product)
    e = s.solve(50000, seed=3, max_failed=1 << 40, check=False)
    assert e.res == P.RES_OK
    assert e.count("failed_count") == 50000 and e.count("realisation_count") == 0


def test_host_abort_of_a_running_plan(product):
    """ssol_b200_plan_abort while a long launch runs: its warps stop taking
    realisations within milliseconds, ssol_b200_plan_finish returns
    RES_BAD_OP with the estimator of what ran, and a reset clears it."""
    import threading
    import time
    s, h = W.single_mirror(product)
    plan = P.C.c_void_p()
    product.call("ssol_b200_plan_create", s.scn, None, P.C.byref(plan))
    rng = s.rng(seed=4)
    n = 8_000_000_000
    t0 = time.perf_counter()
    # The launch enqueues its chunks of 2^24 realisations from this thread
    # (it may block on the launch queue); the abort comes from another one
    th = threading.Thread(target=product.call,
                          args=("ssol_b200_plan_launch", plan, rng, 0, n, None))
    th.start()
    time.sleep(0.2)
    product.call("ssol_b200_plan_abort", plan)
    th.join()
    est = P.C.c_void_p()
    res = product.raw("ssol_b200_plan_finish", plan, rng, n, 0, None, P.C.byref(est))
    dt = time.perf_counter() - t0
    e = P.Estimator(s, est, res)
    assert res == P.RES_BAD_OP
    ran = e.count("realisation_count")
    assert 0 < ran < n // 2, ran
    assert dt < 5.0, dt
    g = e.globals()
    assert g["cos_factor"][0] > 0
    del e
    product.call("ssol_b200_plan_reset", plan, None)
    product.call("ssol_b200_plan_launch", plan, rng, 0, 100000, None)
    est = P.C.c_void_p()
    res = product.raw("ssol_b200_plan_finish", plan, rng, 100000, 0, None, P.C.byref(est))
    e = P.Estimator(s, est, res)
    assert res == P.RES_OK and e.count("realisation_count") == 100000
    del e
    product.raw("ssol_b200_plan_ref_put", plan)
