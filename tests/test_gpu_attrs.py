"""Spatially varying shaders and vertex normals on the B200 library. Shaders
of a material that varies over its mesh are evaluated at the vertices of
every triangle when the scene is snapshot and interpolated with the hit's
barycentric weights on the device: exact for shaders affine in position and
texcoords (compared with the oracle, which calls the shaders at each hit,
within 3 combined SE), linear inside each triangle otherwise (checked
against the piecewise-linear closed form). Vertex normals are interpolated
and normalised on the device like Star-3D's attributes."""
import math

import pytest

import attr_scenes as A
import pyssol as P

pytestmark = pytest.mark.gpu


def close(a, b, k=3.0):
    return abs(a[0] - b[0]) <= k * math.hypot(a[2], b[2]) + 1e-6 * abs(b[0])


@pytest.mark.parametrize("kind", ["P", "uv"])
@pytest.mark.parametrize("precision", [P.FP64, P.FP32], ids=["fp64", "fp32"])
def test_gpu_varying_reflectivity(product, oracle, kind, precision):
    s, h = A.ramp_mirror(product, kind)
    n = 1000000
    e = s.solve(n, seed=2, options=P.options(precision=precision))
    r = e.receiver(h["receiver"])["incoming_flux"]
    assert abs(r[0] - h["expected"]) <= 3 * r[2] + 1e-6 * h["expected"]
    so, ho = A.ramp_mirror(oracle, kind)
    ro = so.solve(200000, seed=2).receiver(ho["receiver"])["incoming_flux"]
    assert close(r, ro)


def test_gpu_baked_texcoord_shader(product):
    s, h = A.ramp_mirror(product, "tex")
    e = s.solve(2000000, seed=4)
    r = e.receiver(h["receiver"])["incoming_flux"]
    assert abs(r[0] - h["expected"]) <= 3 * r[2] + 1e-6 * h["expected"]


@pytest.mark.parametrize("turn_z", [False, True], ids=["plain", "turned"])
@pytest.mark.parametrize("precision", [P.FP64, P.FP32], ids=["fp64", "fp32"])
def test_gpu_vertex_normals(product, oracle, precision, turn_z):
    s, h = A.tilted_normals(product, turn_z=turn_z)
    e = s.solve(200000, seed=3, options=P.options(precision=precision))
    r = e.receiver(h["receiver"])["incoming_flux"]
    assert r[0] == pytest.approx(h["expected"], rel=1e-6)
    so, ho = A.tilted_normals(oracle, turn_z=turn_z)
    ro = so.solve(20000, seed=3).receiver(ho["receiver"])["incoming_flux"]
    assert close(r, ro)
