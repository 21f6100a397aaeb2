"""Distributions of the sun-direction and microfacet samplers, read back
through the path tracker, against their analytic CDFs.

No reference test pins these samplers (src/test_ssol_sun.c checks the API
only; every solver test uses roughness 0), so each gets its published
distribution:
- pillbox (src/ssol_ranst_sun_dir.c:265-283): sin^2(theta) ~ U[0, sin^2(a)],
  P(theta <= t) = sin^2 t / sin^2 a;
- Gaussian (src/ssol_ranst_sun_dir.c:285-310): sin(theta) = sigma
  sqrt(-2 ln u), P(sin theta <= s) = 1 - exp(-s^2 / (2 sigma^2));
- Buie (src/ssol_ranst_sun_dir.c:177-241, 362-419; Buie, Monger and Dey,
  Solar Energy 74, 2003): density in theta proportional to phi(theta)
  sin(theta), phi = cos(0.326 t) / cos(0.308 t) inside the disk (t in mrad,
  t <= 4.65) and e^k t^gamma in the circumsolar region (4.65 < t <= 43.6),
  k and gamma from the CSR through chi (calibration polynomial of
  src/ssol_ranst_sun_dir.c:89-107); the CDF is integrated numerically;
- microfacet normals (Walter et al. 2007): Beckmann tan^2(theta_h) ~
  Exp(mean m^2), pillbox tan^2(theta_h) ~ U[0, m^2]; at normal incidence
  the reflected direction makes 2 theta_h with the normal.
"""
import math

import numpy as np

import pyssol as P


def ks_distance(samples, cdf):
    """Kolmogorov-Smirnov distance of the samples to a vectorised CDF."""
    x = np.sort(np.asarray(samples, dtype=np.float64))
    n = x.size
    f = cdf(x)
    i = np.arange(1, n + 1)
    return float(max(np.max(i / n - f), np.max(f - (i - 1) / n)))


def ks_bound(n, alpha_coef=1.95):
    """Critical KS distance at the 0.1 % level (1.95 / sqrt(n))."""
    return alpha_coef / math.sqrt(n)


def sun_scene(lib, kind, param):
    """A 100 x 100 matte plane under a sun along -z; the tracker's sun
    segment gives each path's sampled direction."""
    s = P.Scene(lib)
    m = s.matte(0.5)
    s.instance(s.object([(s.rectangle(50, 50), m, m)]))
    s.set_sun(kind, (0.0, 0.0, -1.0), 1000.0, param=param)
    return s


def sun_angles(est):
    """Angle of each tracked path's incoming direction to -z."""
    out = []
    for _, verts in est.paths():
        (x0, _), (x1, _) = verts[0], verts[1]
        d = np.subtract(x1, x0)
        d /= np.linalg.norm(d)
        out.append(math.acos(max(-1.0, min(1.0, -d[2]))))
    return np.array(out)


def pillbox_cdf(a):
    return lambda t: np.sin(t) ** 2 / math.sin(a) ** 2


def gaussian_cdf(sigma):
    return lambda t: 1.0 - np.exp(-np.sin(t) ** 2 / (2 * sigma * sigma))


def buie_chi(csr):
    c = csr
    if c > 0.145:
        return -0.04419909985804843 + c * (1.401323894233574 + c * (
            -0.3639746714505299 + c * (-0.9579768560161194 + 1.1550475450828657 * c)))
    if c > 0.035:
        return 0.022652077593662934 + c * (0.5252380349996234 + c * (
            2.5484334534423887 - 0.8763755326550412 * c))
    return 0.004733749294807862 + c * (4.716738065192151 + c * (-463.506669149804 + c * (
        24745.88727411664 + c * (-606122.7511711778 + 5521693.445014727 * c))))


def buie_cdf(csr, n=200001):
    chi = buie_chi(csr)
    k = 0.9 * math.log(13.5 * chi) * chi ** -0.3
    g = 2.2 * math.log(0.52 * chi) * chi ** 0.43 - 0.1
    t_sd, t_cs = 4.65e-3, 43.6e-3
    t = np.linspace(0.0, t_cs, n)
    tm = t * 1e3
    phi = np.where(t <= t_sd, np.cos(0.326 * tm) / np.cos(0.308 * tm),
                   math.exp(k) * np.power(np.maximum(tm, 1e-30), g))
    pdf = phi * np.sin(t)
    c = np.concatenate([[0.0], np.cumsum(0.5 * (pdf[1:] + pdf[:-1]) * np.diff(t))])
    c /= c[-1]
    return lambda x: np.interp(x, t, c)


def lobe_scene(lib, distrib, m):
    """A 100 x 100 mirror of roughness m under a vertical directional sun;
    the tracker's segment to infinity gives the reflected direction."""
    s = P.Scene(lib)
    mir = s.mirror(1.0, m, distrib)
    s.instance(s.object([(s.rectangle(50, 50), mir, mir)]))
    s.set_sun("directional", (0.0, 0.0, -1.0), 1000.0)
    return s


def lobe_tan2(est):
    """tan^2 of half the reflected direction's angle to +z, per path."""
    out = []
    for _, verts in est.paths():
        (x1, _), (x2, _) = verts[1], verts[2]
        d = np.subtract(x2, x1)
        d /= np.linalg.norm(d)
        th = 0.5 * math.acos(max(-1.0, min(1.0, d[2])))
        out.append(math.tan(th) ** 2)
    return np.array(out)


def beckmann_cdf(m):
    return lambda x: 1.0 - np.exp(-x / (m * m))


def pillbox_slope_cdf(m):
    return lambda x: np.clip(x / (m * m), 0.0, 1.0)
