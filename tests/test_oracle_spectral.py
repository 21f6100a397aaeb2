"""The CPU oracle on the wavelength-dependent scenes of spectral_scenes: a
four-node sun spectrum with spectral reflectivity, extinction, refractive
index and slab absorption, against closed forms integrated over the sun's
piecewise-linear spectrum (4 standard errors). No reference test solves with
these, so the closed forms pin the oracle here, as the monochromatic
spectral-extinction pin (src/test_ssol_solver1.c:491-528) does for one
wavelength."""
import pytest

import spectral_scenes as SP


@pytest.mark.parametrize("name", sorted(SP.BUILDERS))
def test_oracle_spectral_closed_form(oracle, name):
    s, h = SP.BUILDERS[name](oracle)
    est = s.solve(200000, seed=8)
    assert est.count("failed_count") == 0
    inc = est.receiver(h["receiver"])["incoming_flux"]
    assert abs(inc[0] - h["expected"]) <= 4 * inc[2] + 1e-6 * h["expected"], (inc, h["expected"])
    assert inc[2] > 1e-4 * h["expected"]
