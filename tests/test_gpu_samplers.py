"""The B200 library's sun-direction and microfacet samplers against their
analytic distributions (sampler_scenes), through the device path tracker,
in both precisions: Kolmogorov-Smirnov distance below the 0.1 % critical
value."""
import pytest

import pyssol as P
import sampler_scenes as S

pytestmark = pytest.mark.gpu

N = 50000
PREC = [P.FP64, P.FP32]
IDS = ["fp64", "fp32"]


@pytest.mark.parametrize("precision", PREC, ids=IDS)
@pytest.mark.parametrize("kind,param,cdf", [
    ("pillbox", 4.65e-3, S.pillbox_cdf(4.65e-3)),
    ("pillbox", 0.2, S.pillbox_cdf(0.2)),
    ("gaussian", 2.5e-3, S.gaussian_cdf(2.5e-3)),
    ("buie", 0.1, S.buie_cdf(0.1)),
    ("buie", 0.02, S.buie_cdf(0.02)),
], ids=["pillbox-4.65mrad", "pillbox-0.2rad", "gaussian-2.5mrad", "buie-csr0.1",
        "buie-csr0.02"])
def test_gpu_sun_directions(product, kind, param, cdf, precision):
    s = S.sun_scene(product, kind, param)
    e = s.solve(N, seed=21, tracker=(100.0, 100.0), options=P.options(precision=precision))
    th = S.sun_angles(e)
    assert th.size == N
    assert S.ks_distance(th, cdf) < S.ks_bound(N)


@pytest.mark.parametrize("precision", PREC, ids=IDS)
@pytest.mark.parametrize("distrib,m,cdf", [
    (P.BECKMANN, 0.05, S.beckmann_cdf(0.05)),
    (P.PILLBOX, 0.05, S.pillbox_slope_cdf(0.05)),
], ids=["beckmann", "pillbox"])
def test_gpu_microfacet_lobe(product, distrib, m, cdf, precision):
    s = S.lobe_scene(product, distrib, m)
    e = s.solve(N, seed=22, tracker=(100.0, 100.0), options=P.options(precision=precision))
    t2 = S.lobe_tan2(e)
    assert S.ks_distance(t2, cdf) < S.ks_bound(N)
    mean = m * m if distrib == P.BECKMANN else 0.5 * m * m
    assert abs(t2.mean() - mean) < 4 * t2.std() / N ** 0.5
