"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares; the setup half of the API behaves like the reference's
argument checks (src/test_ssol_*.c API-contract tests)."""
import ctypes as C
import os
import re

import pytest

import pyssol as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = "\n".join(ln for ln in text.splitlines() if not ln.lstrip().startswith("#"))
        for m in re.finditer(r"(?:SSOL_API|SSP_API)\s+[^;(]*?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported(product):
    names = declared_symbols()
    assert len(names) > 100
    missing = [n for n in names if not hasattr(product.dll, n)]
    assert not missing, missing


def test_oracle_exports_the_hot_subset(oracle):
    for n in ("ssol_solve", "ssol_estimator_get_mc_global", "ssol_estimator_get_mc_receiver",
              "ssol_estimator_get_rng_state", "ssol_mc_shape_get_mc_primitive"):
        assert hasattr(oracle.dll, n)


@pytest.fixture(params=["product", "oracle"])
def lib(request, product, oracle):
    return product if request.param == "product" else oracle


def test_setup_argument_checks(lib):
    s = P.Scene(lib)
    h = C.c_void_p()
    assert lib.raw("ssol_device_create", None, None, 0, 0, C.byref(h)) == P.RES_BAD_ARG
    assert lib.raw("ssol_scene_create", None, C.byref(h)) == P.RES_BAD_ARG
    assert lib.raw("ssol_shape_create_mesh", s.dev, None) == P.RES_BAD_ARG
    sun = s.set_sun("pillbox", (0, 0, -1), 1000.0, param=0.1)
    assert lib.raw("ssol_sun_set_dni", sun, 0.0) == P.RES_BAD_ARG
    assert lib.raw("ssol_sun_pillbox_set_half_angle", sun, 2.0) == P.RES_BAD_ARG
    assert lib.raw("ssol_sun_gaussian_set_std_dev", sun, 0.1) == P.RES_BAD_ARG
    zero = (C.c_double * 3)(0, 0, 0)
    assert lib.raw("ssol_sun_set_direction", sun, zero) == P.RES_BAD_ARG
    atm = C.c_void_p()
    lib.call("ssol_atmosphere_create", s.dev, C.byref(atm))
    d = s.data(1.5)
    assert lib.raw("ssol_atmosphere_set_extinction", atm, C.byref(d)) == P.RES_BAD_ARG
    lib.call("ssol_atmosphere_ref_put", atm)
    # punched surface with no carving is invalid unless hemisphere
    with pytest.raises(P.SsolError):
        s.punched(P.Q_PARABOL, (10.0,), [])
    with pytest.raises(P.SsolError):
        s.punched(P.Q_PARABOL, (-1.0,), [(P.SSOL_AND, [(-1, -1), (-1, 1), (1, 1), (1, -1)])])
    s.close()


def test_solve_argument_checks(lib):
    """src/test_ssol_solver1.c:127-136: NULL scene / rng / zero realisations,
    no sun, no geometry are RES_BAD_ARG (no GPU work is reached)."""
    s = P.Scene(lib)
    rng = s.rng()
    est = C.c_void_p()
    assert lib.raw("ssol_solve", None, rng, 10, 0, None, C.byref(est)) == P.RES_BAD_ARG
    assert lib.raw("ssol_solve", s.scn, None, 10, 0, None, C.byref(est)) == P.RES_BAD_ARG
    assert lib.raw("ssol_solve", s.scn, rng, 0, 0, None, C.byref(est)) == P.RES_BAD_ARG
    assert lib.raw("ssol_solve", s.scn, rng, 10, 0, None, None) == P.RES_BAD_ARG
    # no sun
    assert lib.raw("ssol_solve", s.scn, rng, 10, 0, None, C.byref(est)) == P.RES_BAD_ARG
    s.set_sun("directional", (1, 0, -1), 1000.0)
    # no geometry to sample
    assert lib.raw("ssol_solve", s.scn, rng, 10, 0, None, C.byref(est)) == P.RES_BAD_ARG
    sq = s.rectangle(1, 1)
    m = s.mirror(1.0)
    inst = s.instance(s.object([(sq, m, m)]), sample=0)
    assert lib.raw("ssol_solve", s.scn, rng, 10, 0, None, C.byref(est)) == P.RES_BAD_ARG
    s.close()


def test_plan_option_checks(product):
    """Options are checked before any snapshot or GPU work: an unknown BVH
    builder, a negative leaf size and an unknown precision are RES_BAD_ARG."""
    s = P.Scene(product)
    plan = C.c_void_p()
    for o in (P.options(bvh=7), P.options(bvh=-1), P.options(leaf=-1), P.options(precision=5)):
        assert product.raw("ssol_b200_plan_create", s.scn, C.byref(o), C.byref(plan)) == P.RES_BAD_ARG
    scenes = (C.c_void_p * 1)(s.scn.value)
    batch = C.c_void_p()
    assert product.raw("ssol_b200_batch_create", scenes, 1, C.byref(P.options(bvh=7)),
                       C.byref(batch)) == P.RES_BAD_ARG
    s.close()


def test_areas_and_tessellation(lib):
    """Areas of meshes and punched surfaces (src/test_ssol_solver3.c:138-163:
    a 20x20 punched plane has area 400)."""
    s = P.Scene(lib)
    poly = [(-10, -10), (-10, 10), (10, 10), (10, -10)]
    plane = s.punched(P.Q_PLANE, (), [(P.SSOL_AND, poly)])
    m = s.mirror(1.0)
    obj = s.object([(plane, m, m)])
    a = C.c_double()
    lib.call("ssol_object_get_area", obj, C.byref(a))
    assert a.value == pytest.approx(400.0, rel=1e-12)
    par = s.punched(P.Q_PARABOL, (10.0,), [(P.SSOL_AND, [(-5, -5), (-5, 5), (5, 5), (5, -5)])])
    obj2 = s.object([(par, m, m)])
    lib.call("ssol_object_get_area", obj2, C.byref(a))
    # paraboloid 10x10, f = 10: the tessellated area exceeds the flat 100
    assert 100.0 < a.value < 103.0
    # a circular carving: polygon with the area of a unit-radius disk
    import math
    nv = 36
    r = math.sqrt(2 * math.pi / (math.sin(2 * math.pi / nv) * nv))
    circ = [(r * math.cos(-k * 2 * math.pi / nv), r * math.sin(-k * 2 * math.pi / nv))
            for k in range(nv)]
    disk = s.punched(P.Q_PLANE, (), [(P.SSOL_AND, circ)])
    lib.call("ssol_object_get_area", s.object([(disk, m, m)]), C.byref(a))
    assert a.value == pytest.approx(math.pi, rel=1e-6)  # float vertices
    # SUB carving: 20x20 minus a centred 4x4 hole
    holed = s.punched(P.Q_PLANE, (), [(P.SSOL_AND, poly),
                                      (P.SSOL_SUB, [(-2, -2), (-2, 2), (2, 2), (2, -2)])])
    lib.call("ssol_object_get_area", s.object([(holed, m, m)]), C.byref(a))
    assert a.value == pytest.approx(384.0, rel=1e-6)
    s.close()


def test_rng_shim_matches_between_libraries(product, oracle):
    """Both libraries implement the same Philox shim: identical draws."""
    outs = []
    for lib in (product, oracle):
        r = C.c_void_p()
        lib.call("ssp_rng_create", None, P.SSP_RNG_THREEFRY, C.byref(r))
        lib.call("ssp_rng_set", r, 42)
        outs.append([lib.dll.ssp_rng_get(r) for _ in range(8)])
        lib.call("ssp_rng_ref_put", r)
    assert outs[0] == outs[1]


def test_batch_host_path(product):
    """Batch creation validates and snapshots every scene on the host; without
    a GPU it stops at device binding (RES_UNKNOWN_ERR), with bad arguments at
    RES_BAD_ARG."""
    import workloads as W
    fields = W.batched_fields(product, [{"elevation": 30.0, "azimuth": 180.0, "dni": 900.0},
                                        {"elevation": 50.0, "azimuth": 90.0, "dni": 600.0}],
                              n_helio=10, receiver_cells=4)
    arr = (C.c_void_p * 2)(*[f[0].scn.value for f in fields])
    h = C.c_void_p()
    assert product.raw("ssol_b200_batch_create", None, 2, None, C.byref(h)) == P.RES_BAD_ARG
    assert product.raw("ssol_b200_batch_create", C.cast(arr, P.PVP), 0, None,
                       C.byref(h)) == P.RES_BAD_ARG
    res = product.raw("ssol_b200_batch_create", C.cast(arr, P.PVP), 2, None, C.byref(h))
    import conftest
    if conftest.gpu_available():
        assert res == P.RES_OK
        product.raw("ssol_b200_batch_ref_put", h)
    else:
        assert res == P.RES_UNKNOWN_ERR


def test_native_constant_shaders(product):
    """ssol_b200_shader_param0/1 read the material's parameter buffer,
    ssol_b200_shader_Ns returns the fragment's shading normal"""
    import ctypes as C
    import pyssol as P
    s = P.Scene(product)
    dll = product.dll
    buf = C.c_void_p()
    product.call("ssol_param_buffer_create", s.dev, 16, C.byref(buf))
    mem = dll.ssol_param_buffer_allocate(buf, 16, 8, None)
    arr = C.cast(mem, C.POINTER(C.c_double))
    arr[0], arr[1] = 0.7, 0.003
    frag = P.SurfaceFragment()
    frag.Ns[0], frag.Ns[1], frag.Ns[2] = 0.6, 0.0, 0.8
    out = (C.c_double * 3)()
    for name, want in (("ssol_b200_shader_param0", 0.7), ("ssol_b200_shader_param1", 0.003)):
        f = P.SHADER((name, dll))
        f(s.dev, buf, 500.0, C.byref(frag), out)
        assert out[0] == want
        f(s.dev, None, 500.0, C.byref(frag), out)
        assert out[0] == 0.0
    P.SHADER(("ssol_b200_shader_Ns", dll))(s.dev, None, 500.0, C.byref(frag), out)
    assert tuple(out) == (0.6, 0.0, 0.8)
    product.call("ssol_param_buffer_ref_put", buf)
    s.close()


def test_tracking_batch_argument_checks(product):
    """ssol_b200_batch_create_tracking refuses bad arguments on the host,
    before any device work: no suns, a DNI <= 0, a zero direction, a punched
    heliostat, a heliostat outside the scene."""
    import workloads as W
    s, h = W.heliostat_field(product, n_helio=10, receiver_cells=2)
    hel, aims, sp = W.tracking_inputs(h, [{"elevation": 40.0, "azimuth": 90.0, "dni": 800.0}])
    ha = (C.c_void_p * len(hel))(*[x.value for x in hel])
    aa = (C.c_double * (3 * len(aims)))(*[c for a in aims for c in a])
    out = C.c_void_p()

    def call(suns, heliostats=ha, n=len(hel)):
        arr = (P.SunPosition * max(1, len(suns)))()
        for i, (d, dni) in enumerate(suns):
            arr[i].direction[:] = d
            arr[i].dni = dni
        return product.raw("ssol_b200_batch_create_tracking", s.scn, C.cast(heliostats, P.PVP),
                           n, aa, arr, len(suns), None, C.byref(out))
    assert call([]) == P.RES_BAD_ARG
    assert call([(sp[0][0], 0.0)]) == P.RES_BAD_ARG
    assert call([((0.0, 0.0, 0.0), 900.0)]) == P.RES_BAD_ARG
    other = P.Scene(product)
    stray = other.instance(other.object([(other.rectangle(1, 1), other.matte(0.0),
                                          other.matte(0.0))]))
    assert call(sp, (C.c_void_p * 1)(stray.value), 1) == P.RES_BAD_ARG
    poly = [(-1, -1), (-1, 1), (1, 1), (1, -1)]
    par = s.instance(s.object([(s.punched(P.Q_PARABOL, (10.0,), [(P.SSOL_AND, poly)]),
                                s.mirror(0.9, 0.0), s.matte(0.0))]),
                     P.transform_from(None, (0, 300, 5)), sample=0)
    assert call(sp, (C.c_void_p * 1)(par.value), 1) == P.RES_BAD_ARG
