"""The oracle on spatially varying shaders and vertex normals: the shaders of
a material that varies over its mesh are called at every hit's surface
fragment (reference semantics), and the BSDF follows the interpolated
vertex normal. Closed forms in attr_scenes."""
import pytest

import attr_scenes as A


@pytest.mark.parametrize("kind", ["P", "uv"])
def test_oracle_varying_reflectivity(oracle, kind):
    s, h = A.ramp_mirror(oracle, kind)
    e = s.solve(40000, seed=2)
    r = e.receiver(h["receiver"])["incoming_flux"]
    assert abs(r[0] - h["expected"]) <= 3 * r[2]
    assert r[2] > 0  # the weight varies from path to path


def test_oracle_texcoord_shader_exact(oracle):
    """The oracle calls u^2 at each hit's texcoords: the exact mean 1/3, not
    the piecewise-linear mean the device's per-vertex baking gives."""
    s, h = A.ramp_mirror(oracle, "tex")
    e = s.solve(500000, seed=4)
    r = e.receiver(h["receiver"])["incoming_flux"]
    assert abs(r[0] - h["exact"]) <= 3 * r[2]
    assert abs(h["expected"] - h["exact"]) > 5 * r[2]  # the two are told apart


@pytest.mark.parametrize("turn_z", [False, True], ids=["plain", "turned"])
def test_oracle_vertex_normals(oracle, turn_z):
    s, h = A.tilted_normals(oracle, turn_z=turn_z)
    e = s.solve(20000, seed=3)
    r = e.receiver(h["receiver"])["incoming_flux"]
    assert r[0] == pytest.approx(h["expected"], rel=1e-9)
