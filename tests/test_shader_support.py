"""Shaders the device cannot evaluate are refused, not approximated.

The reference evaluates the material shaders per hit fragment
(src/ssol_material.c:551-655): position P, normals, the incoming direction.
The B200 library tabulates them per material (at the sun's wavelength nodes)
and bakes them per vertex on meshes where they vary. Three kinds of shader
fit neither form and make ssol_solve return RES_BAD_ARG when the scene is
snapshot (on the host, so these checks need no GPU):
- a mirror or matte shader that varies over a punched (quadric) surface;
- a mirror or matte shader that reads the incoming direction `dir`;
- a normal shader that returns anything but the shading normal Ns.
The oracle evaluates all three per hit and solves these scenes."""
import ctypes as C

import pytest

import pyssol as P
import ref_scenes as R


def _paraboloid_scene(lib, refl):
    s = P.Scene(lib)
    poly = [(-5, -5), (-5, 5), (5, 5), (5, -5)]
    shape = s.punched(P.Q_PARABOL, (10.0,), [(P.SSOL_AND, poly)])
    m = s.mirror(refl, 0.0)
    s.instance(s.object([(shape, m, m)]))
    tgt = s.matte(0.0)
    s.instance(s.object([(s.rectangle(1, 1), tgt, tgt)]), P.transform_from(None, (0, 0, 10)),
               receiver=P.SSOL_FRONT, sample=0)
    s.set_sun("directional", (0, 0, -1), R.DNI)
    return s


def _solve_code(s):
    est = C.c_void_p()
    rng = s.rng(seed=1)
    res = s.lib.raw("ssol_solve", s.scn, rng, 1000, 0, None, C.byref(est))
    if est:
        s.lib.raw("ssol_estimator_ref_put", est)
    return res


def test_shader_varying_over_a_punched_surface_is_refused(product, oracle):
    def varying(wl, frag):
        return 0.5 + 0.04 * frag.P[0]
    assert _solve_code(_paraboloid_scene(product, varying)) == P.RES_BAD_ARG
    assert _solve_code(_paraboloid_scene(oracle, varying)) == P.RES_OK
    # a constant shader on the same surface passes the snapshot (without a
    # GPU the solve then stops at the device: RES_UNKNOWN_ERR)
    assert _solve_code(_paraboloid_scene(product, lambda wl, frag: 0.9)) != P.RES_BAD_ARG


def test_shader_reading_the_direction_is_refused(product, oracle):
    def view_dependent(wl, frag):
        return 0.5 + 0.4 * abs(frag.dir[2])
    for lib, want in ((product, P.RES_BAD_ARG), (oracle, P.RES_OK)):
        s = P.Scene(lib)
        m = s.mirror(view_dependent, 0.0)
        s.instance(s.object([(s.rectangle(5, 5), m, m)]))
        tgt = s.matte(0.0)
        s.instance(s.object([(s.rectangle(5, 5), tgt, tgt)]), P.transform_from(None, (0, 0, 5)),
                   receiver=P.SSOL_BACK, sample=0)
        s.set_sun("directional", (0.1, 0, -1), R.DNI)
        assert _solve_code(s) == want


def test_normal_shader_other_than_ns_is_refused(product, oracle):
    def fixed_normal(dev, buf, wl, frag, out):
        out[0], out[1], out[2] = 0.0, 0.0, 1.0
    for lib, want in ((product, P.RES_BAD_ARG), (oracle, P.RES_OK)):
        s = P.Scene(lib)
        h = s._new("ssol_material_create_mirror", "ssol_material_ref_put", s.dev)
        shader = P.MirrorShader(P.SHADER(fixed_normal), s._const(0.9), s._const(0.0))
        s._keep.append(shader)
        lib.call("ssol_mirror_setup", h, C.byref(shader), P.BECKMANN)
        s.instance(s.object([(s.rectangle(5, 5), h, h)]))
        tgt = s.matte(0.0)
        s.instance(s.object([(s.rectangle(5, 5), tgt, tgt)]), P.transform_from(None, (0, 0, 5)),
                   receiver=P.SSOL_BACK, sample=0)
        s.set_sun("directional", (0.1, 0, -1), R.DNI)
        assert _solve_code(s) == want
