"""Tracking batches (ssol_b200_batch_create_tracking): one snapshot of a
heliostat field, its heliostats re-aimed per sun and its BVH refitted on the
device. Item i must be the field a host snapshot gives for sun i
(workloads.heliostat_field re-aims with the same rule): against ssol_solve of
that host-built scene on the same realisation streams, every global and
receiver estimate within 3 combined standard errors, and the means within a
tenth of a standard error (the paths are the same ones). Then a few items
against the oracle's solve of the host-built scene."""
import math

import pytest

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu


def close(a, b, k=3.0):
    return abs(a[0] - b[0]) <= k * math.hypot(a[2], b[2]) + 1e-6 * max(1.0, abs(b[0]))


def _suns(k):
    grid = W.sun_grid()
    return [grid[i * 16 + (i * 7) % 16] for i in range(0, 16, 16 // k)]


@pytest.mark.parametrize("precision,scale", [(P.FP32, 1), (P.FP64, 1), (P.FP32, 2)])
def test_tracking_items_equal_host_built_fields(product, precision, scale):
    """scale 2 takes the launch above 2^22 realisations: the coherent order"""
    suns = _suns(8)
    kw = dict(n_helio=300, receiver_cells=16)
    s, h = W.heliostat_field(product, **kw)
    hel, aims, sp = W.tracking_inputs(h, suns)
    opts = P.options(precision)
    batch = P.Batch.tracking(s, hel, aims, sp, opts)
    rng = s.rng(seed=5)
    budgets = [scale * (300000 + 50000 * i) for i in range(len(suns))]
    batch.launch(rng, budgets)
    ests = batch.finish(rng)
    for sun, est, n in zip(suns, ests, budgets):
        what = "el %.1f az %.1f" % (sun["elevation"], sun["azimuth"])
        sh, hh = W.heliostat_field(product, elevation=sun["elevation"], azimuth=sun["azimuth"],
                                   dni=sun["dni"], **kw)
        ref = sh.solve(n, seed=5, options=opts)
        assert est.count("realisation_count") == n
        for got, want in ((est.globals(), ref.globals()),
                          (est.receiver(h["receiver"]), ref.receiver(hh["receiver"]))):
            for q in want:
                assert close(got[q], want[q]), (what, q, got[q], want[q])
                assert abs(got[q][0] - want[q][0]) <= 0.1 * want[q][2] + 1e-9 * abs(want[q][0]), \
                    (what, q, got[q], want[q])
        sh.close()
    batch.close()


def test_tracking_items_vs_oracle(product, oracle):
    suns = _suns(4)
    s, h = W.heliostat_field(product)
    hel, aims, sp = W.tracking_inputs(h, suns)
    batch = P.Batch.tracking(s, hel, aims, sp)
    rng = s.rng(seed=9)
    budgets = [1_000_000] * len(suns)
    batch.launch(rng, budgets)
    ests = batch.finish(rng)
    for sun, est, n in zip(suns, ests, budgets):
        so, ho = W.heliostat_field(oracle, elevation=sun["elevation"], azimuth=sun["azimuth"],
                                   dni=sun["dni"])
        ref = so.solve(n, seed=9)
        for got, want in ((est.globals(), ref.globals()),
                          (est.receiver(h["receiver"]), ref.receiver(ho["receiver"]))):
            for q in want:
                assert close(got[q], want[q]), (sun, q, got[q], want[q])
        so.close()
    batch.close()


def test_tracking_noalloc_launch(product):
    """The no-allocation launch on a tracking batch gives what the regular
    launch gives."""
    suns = _suns(4)
    s, h = W.heliostat_field(product, n_helio=100, receiver_cells=8)
    hel, aims, sp = W.tracking_inputs(h, suns)
    a = P.Batch.tracking(s, hel, aims, sp)
    b = P.Batch.tracking(s, hel, aims, sp)
    rng = s.rng(seed=2)
    budgets = [100000, 20000, 70000, 40000]
    a.launch(rng, budgets)
    b.launch_noalloc(rng, budgets)
    for x, y in zip(a.finish(rng), b.finish(rng)):
        gx, gy = x.globals(), y.globals()
        for q in gy:
            assert close(gx[q], gy[q]), q
    a.close()
    b.close()


def test_batch_globals_equal_the_estimators(product):
    """ssol_b200_batch_get_mc_global gives, item by item, the global
    estimates of the estimators ssol_b200_batch_finish builds."""
    suns = _suns(4)
    s, h = W.heliostat_field(product, n_helio=100, receiver_cells=8)
    batch = P.Batch.tracking(s, *W.tracking_inputs(h, suns))
    rng = s.rng(seed=3)
    batch.launch(rng, [50000, 10000, 30000, 20000])
    batch.launch(rng, [5000, 0, 7000, 1000])
    quick = batch.globals()
    full = batch.finish(rng)
    for g, e in zip(quick, full):
        for k, v in e.globals().items():
            assert g[k][0] == pytest.approx(v[0], rel=1e-14, abs=1e-12), k
            assert g[k][2] == pytest.approx(v[2], rel=1e-12, abs=1e-12), k
    batch.close()


def test_tracking_receiver_sums_repeat(product):
    """Receiver sums go through per-warp shared-memory slots that are
    flushed and cleared whenever a warp moves to another item. Many small
    items of ragged budgets make many such moves; three launches of the
    same realisations must give the same receiver sums (to the order of the
    FP64 additions) and the same per-primitive map."""
    suns = W.sun_grid()[::4]
    kw = dict(n_helio=300, receiver_cells=16)
    s, h = W.heliostat_field(product, **kw)
    hel, aims, sp = W.tracking_inputs(h, suns)
    budgets = [20000 + 7919 * (i % 13) for i in range(len(suns))]
    runs = []
    for rep in range(3):
        batch = P.Batch.tracking(s, hel, aims, sp)
        rng = s.rng(seed=21)
        batch.launch(rng, budgets)
        ests = batch.finish(rng)
        runs.append([(e.receiver(h["receiver"]),
                      [c["incoming_flux"][0] for c in e.primitives(h["receiver"],
                                                                   h["receiver_shape"])])
                     for e in ests])
        del ests
        batch.close()
    for i in range(len(suns)):
        r0, m0 = runs[0][i]
        for rep in (1, 2):
            r, m = runs[rep][i]
            for q in r0:
                assert abs(r[q][0] - r0[q][0]) <= 1e-9 * max(1.0, abs(r0[q][0])), \
                    (i, rep, q, r[q], r0[q])
            assert max(abs(a - b) for a, b in zip(m, m0)) <= 1e-9 * max(1.0, max(map(abs, m0)))
    s.close()
