"""Closed forms for the dielectric, thin dielectric and Russian roulette rows
on the CPU oracle (no reference test pins them; the expectations follow from
Fresnel reflectance at normal incidence and from energy conservation)."""
import pytest

import material_scenes as M


def test_glass_slab(oracle):
    s, h = M.glass_slab(oracle)
    est = s.solve(200000, seed=1)
    r = est.receiver(h["receiver"])["incoming_flux"]
    assert abs(r[0] - h["expected"]) <= 3 * r[2] + 1e-9 * h["expected"]
    g = est.globals()
    total = sum(g[k][0] for k in ("absorbed_by_receivers", "missing", "other_absorbed",
                                  "extinguished_by_atmosphere", "shadowed"))
    assert total == pytest.approx(M.DNI * M.AREA, rel=1e-9)
    assert est.count("failed_count") == 0


def test_thin_slab(oracle):
    s, h = M.thin_slab(oracle)
    est = s.solve(200000, seed=2)
    r = est.receiver(h["receiver"])["incoming_flux"]
    assert abs(r[0] - h["expected"]) <= 3 * r[2] + 1e-9 * h["expected"]


def test_light_trap_roulette(oracle):
    s, h = M.light_trap(oracle)
    est = s.solve(20000, seed=3)
    g = est.globals()
    assert est.count("failed_count") == 0
    assert abs(g["missing"][0] - h["expected_missing"]) <= 3 * g["missing"][2]
    assert abs(g["cos_factor"][0] - h["cos"]) <= 3 * g["cos_factor"][2]
    # the roulette adds variance: paths are killed (0) or survive (x 2^k)
    assert g["missing"][2] > 1e-3 * g["missing"][0]
