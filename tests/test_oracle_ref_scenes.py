"""The CPU oracle against the closed forms of the reference's solver tests
2 to 9 and the by-receiver integration test, with the reference's own
realisation counts and tolerances (the assertions live in ref_checks)."""
import ctypes as C

import pytest

import ref_checks as K
import ref_scenes as R


@pytest.mark.parametrize("name,builder,kw,n", [
    ("solver2", R.solver2, {}, 10000),
    ("solver2b", R.solver2, {"punched_heliostats": True}, 50000),
    ("solver3", R.solver3, {}, 20000),
    ("solver4", R.solver4, {}, 100000),
    ("solver5", R.solver5, {}, 10000),
    ("solver6", R.solver6, {}, 10000),
    ("solver7", R.solver7, {}, 10000),
    ("solver8", R.solver8, {}, 100000),
    ("solver9", R.solver9, {}, 100000),
])
def test_reference_closed_form(oracle, name, builder, kw, n):
    s, h = builder(oracle, **kw)
    est = s.solve(n, seed=11)
    getattr(K, name)(est, h, n)


def test_solver3_area(oracle):
    """src/test_ssol_solver3.c:161-162: the punched 20x20 plane has area 400."""
    s, h = R.solver3(oracle)
    a = C.c_double()
    oracle.call("ssol_instance_get_area", h["heliostat"], C.byref(a))
    assert abs(a.value - 400) <= 2.3e-16 * 400


def test_solver6_continuation(oracle):
    """The reference's checks here are 2-sigma ones on a fixed seed; about one
    seed in ten fails them, so the seed is fixed too."""
    s, h = R.solver6(oracle)
    n = 10000
    est = s.solve(n, seed=6)
    state = C.c_void_p()
    oracle.call("ssol_estimator_get_rng_state", est.h, C.byref(state))
    est2 = s.solve(3 * n, rng=state)
    K.solver6_continuation(est, est2, n)


def test_by_receiver_integration(oracle):
    """src/test_ssol_by_receiver_integration.c:134-162: the same RNG carried
    through three solves; the heliostat becomes a receiver after the first."""
    s, h = R.solver3(oracle, heliostat_receiver=False)
    rng = s.rng(seed=3)
    K.by_receiver(s.solve(10000, rng=rng), h)
    oracle.call("ssol_instance_set_receiver", h["heliostat"], 1, 0)
    K.by_receiver(s.solve(80000, rng=rng), h)
    K.by_receiver(s.solve(30000, rng=rng), h, sampled_x=True)
