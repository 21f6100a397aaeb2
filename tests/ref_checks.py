"""The assertions of the reference's solver tests, restated once and applied
to any estimator: the CPU oracle (exact reference tolerances), the B200
library in FP64 (exact reference tolerances) and in FP32 (the same plus a
relative floor `rel` for FP32 ray geometry; the tallies stay FP64).

Each function cites the CHK lines it restates; `eps` arguments are the
reference's absolute eq_eps tolerances."""
import math

import ref_scenes as R

DNI = R.DNI
COS45 = R.COS45


def near(x, m, eps, rel=0.0):
    return abs(x - m) <= eps + rel * abs(m)


def solver2(est, h, n, rel=0.0):
    """src/test_ssol_solver2.c:183-197: shadowed 0, missing and target
    incoming 4 DNI cos45 (the target sees the whole beam: SE 0)."""
    g = est.globals()
    m = 4 * DNI * COS45
    assert est.count("realisation_count") == n
    assert near(g["shadowed"][0], 0, 1e-4)
    assert near(g["missing"][0], m, 1e-4, rel)
    assert near(g["cos_factor"][0], COS45, 1e-4, rel)
    r = est.receiver(h["target"])["incoming_flux"]
    assert near(r[0], m, 1e-8, rel)
    assert near(r[2], 0, 1e-4, rel * m)


def solver2b(est, h, n, rel=0.0):
    """src/test_ssol_solver2b.c:183-206: the 1x2 target gets half the beam:
    E = 2 DNI cos45 within 2 std, SE = std within 1e-3,
    std = sqrt(((4 DNI cos45)^2 / 2 - (2 DNI cos45)^2) / N)."""
    g = est.globals()
    m = 2 * DNI * COS45
    std = math.sqrt(((4 * DNI * COS45) ** 2 / 2 - m * m) / n)
    assert near(g["shadowed"][0], 0, 1e-4)
    assert near(g["missing"][0], 4 * DNI * COS45, 1e-4, rel)
    assert near(g["cos_factor"][0], COS45, 1e-4, rel)
    r = est.receiver(h["target"])["incoming_flux"]
    assert near(r[0], m, 2 * std)
    assert near(r[2], std, 1e-3, rel * 1e3)
    assert est.count("failed_count") == 0


def solver3(est, h, n, rel=0.0, lib=None):
    """src/test_ssol_solver3.c:138-163: the 2x2 target above a 20x20 mirror
    gets 4 DNI cos45 within 2 std, SE = std within 10,
    std = sqrt(((400 DNI cos45)^2 / 100 - (4 DNI cos45)^2) / N); missing
    400 DNI cos45; instance area exactly 400."""
    g = est.globals()
    m = 4 * DNI * COS45
    std = math.sqrt(((400 * DNI * COS45) ** 2 / 100 - m * m) / n)
    assert near(g["shadowed"][0], 0, 1e-4)
    assert near(g["missing"][0], 400 * DNI * COS45, 1e-4, rel)
    assert near(g["cos_factor"][0], COS45, 1e-4, rel)
    r = est.receiver(h["target"])["incoming_flux"]
    assert near(r[0], m, 2 * std)
    assert near(r[2], std, 10)
    assert est.count("failed_count") == 0


def solver4(est, h, n, rel=0.0):
    """src/test_ssol_solver4.c:151-172: both targets at the focus get
    400 DNI within 1e-2 with SE within 1e-2; missing 400 DNI (1e-2)."""
    g = est.globals()
    m = 400 * DNI
    assert near(g["shadowed"][0], 0, 1e-4)
    assert near(g["missing"][0], m, 1e-2, rel)
    for t in ("target1", "target2"):
        r = est.receiver(h[t])["incoming_flux"]
        assert near(r[0], m, 1e-2, rel)
        assert near(r[2], 0, 1e-2, rel * m)
    assert est.count("failed_count") == 0


def solver5(est, h, n, rel=0.0):
    """src/test_ssol_solver5.c:143-157: the focal-line target gets 400 DNI
    (1e-8, SE 1e-4); missing 400 DNI (1e-4)."""
    g = est.globals()
    m = 400 * DNI
    assert near(g["shadowed"][0], 0, 1e-4)
    assert near(g["missing"][0], m, 1e-4, rel)
    r = est.receiver(h["target"])["incoming_flux"]
    assert near(r[0], m, 1e-8, rel)
    assert near(r[2], 0, 1e-4, rel * m)


def solver6(est, h, n, rel=0.0):
    """src/test_ssol_solver6.c:183-202: shadowed 1e5 within 2e5/sqrt(N);
    missing exactly 0; target 1 front gets 1e5 within 2e5/sqrt(N) (incoming
    == absorbed); target 2 back gets 0 (within 1)."""
    g = est.globals()
    tol = 2 * 100000 / math.sqrt(n)
    assert near(g["shadowed"][0], 100000, tol)
    assert g["missing"][0] == 0
    r1 = est.receiver(h["target1"])
    assert near(r1["incoming_flux"][0], 100000, tol)
    assert r1["incoming_flux"][0] == r1["absorbed_flux"][0]
    r2 = est.receiver(h["target2"], 2)
    assert near(r2["incoming_flux"][0], 0, 1)
    assert r2["incoming_flux"][0] == r2["absorbed_flux"][0]


def solver6_continuation(est, est2, n):
    """src/test_ssol_solver6.c:204-236: a second solve of 3N from the first
    one's RNG state is independent: its SE is the first one's / sqrt3
    (within 0.1), its estimates differ, and merging gives half the SE."""
    g, g2 = est.globals(), est2.globals()
    assert est2.count("realisation_count") == 3 * n
    assert near(g2["shadowed"][0], 100000, 2 * 100000 / math.sqrt(n))
    assert near(g["shadowed"][2] / math.sqrt(3), g2["shadowed"][2], 1e-1)
    assert g["shadowed"][0] != g2["shadowed"][0]
    assert g["shadowed"][2] != g2["shadowed"][2]
    sum_w = g["shadowed"][0] * n + g2["shadowed"][0] * 3 * n
    v1 = g["shadowed"][2] ** 2 * n
    sum_w2 = (v1 + g["shadowed"][0] ** 2) * n
    v2 = g2["shadowed"][2] ** 2 * 3 * n
    sum_w2 += (v2 + g2["shadowed"][0] ** 2) * 3 * n
    e = sum_w / (4 * n)
    v = sum_w2 / (4 * n) - e * e
    se = math.sqrt(v / (4 * n))
    assert near(e, 100000, 3 * se)
    assert near(se, g["shadowed"][2] / 2, se * 1e-2)


def solver7(est, h, n, rel=0.0):
    """src/test_ssol_solver7.c:188-211: sampled area x DNI = 16 DNI (1e-4
    relative); the target receives 16 DNI (1e-4 relative) and absorbs 0.9 of
    it; SE within 1e-2."""
    total = h["total"]
    assert near(est.sampled_area() * DNI, total, total * 1e-4)
    r = est.receiver(h["target"])
    assert near(r["incoming_flux"][0], total, total * 1e-4)
    assert near(r["absorbed_flux"][0], 0.9 * total, 0.9 * total * 1e-4)
    assert near(r["incoming_flux"][2], 0, 1e-2, rel * total)


def solver8(est, h, n, rel=0.0):
    """src/test_ssol_solver8.c:141-160: shadowed 0, missing sqrt2 40 DNI
    within 3 SE, target incoming the same within 2 SE."""
    g = est.globals()
    m = h["S"] * DNI
    assert est.count("failed_count") == 0
    assert near(g["shadowed"][0], 0, 1e-4)
    assert near(g["missing"][0], m, 3 * g["missing"][2])
    r = est.receiver(h["target"])["incoming_flux"]
    assert near(r[0], m, 2 * r[2])


def solver9(est, h, n, rel=0.0):
    """src/test_ssol_solver9.c:135-156: cos_factor 1/3, shadowed DNI x 100,
    missing max(DNI x 100, DNI x 60), incoming min(...), all within 3 SE."""
    g = est.globals()
    assert est.count("failed_count") == 0
    assert near(g["cos_factor"][0], 1 / 3, 3 * g["cos_factor"][2])
    assert near(g["shadowed"][0], h["DNI_S"], 3 * g["shadowed"][2])
    assert near(g["missing"][0], max(h["DNI_S"], h["DNI_TGT_S"]), 3 * g["missing"][2])
    r = est.receiver(h["target"])["incoming_flux"]
    assert near(r[0], min(h["DNI_S"], h["DNI_TGT_S"]), 3 * r[2])


def by_receiver(est, h, rel=0.0, sampled_x=False):
    """src/test_ssol_by_receiver_integration.c:138-162: the target gets
    4 DNI cos45 within 3 SE, and so does the sampled x receiver view."""
    m = 4 * DNI * COS45
    r = est.receiver(h["target"])["incoming_flux"]
    assert near(r[0], m, 3 * r[2])
    if sampled_x:
        r = est.sampled_x_receiver(h["heliostat"], h["target"])["incoming_flux"]
        assert near(r[0], m, 3 * r[2])
