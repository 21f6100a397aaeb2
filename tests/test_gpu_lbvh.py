"""The device-built linear BVH (ssol_b200_options.bvh_builder = LBVH) against
the host binned-SAH tree.

Both trees hold the same primitive boxes and the traversal reports the
closest accepted hit whatever the tree, so a solve traces the same paths with
either: on the same seed every estimate agrees to the order of the FP64
reductions (1e-10 relative). This is the device replacement of the
reference's per-solve Star-3D view build (src/ssol_scene.c:347-433), checked
through the estimates the reference's own tests read. The stats say which
builder ran and how deep its tree is."""
import pytest

import pyssol as P
import workloads as W

pytestmark = pytest.mark.gpu


def _same(a, b, what, rel=1e-10):
    """Estimates equal to the FP64 summation order. A zero-variance estimate
    (every path with the same weight) has an SE made of that rounding alone,
    hence the SE's floor relative to the estimate."""
    for k in b:
        assert a[k][0] == pytest.approx(b[k][0], rel=rel, abs=1e-9), (what, k)
        assert a[k][2] == pytest.approx(b[k][2], rel=1e-6, abs=1e-7 * abs(b[k][0]) + 1e-9), \
            (what, k)


def _solve_pair(s, n, seed, precision=P.FP32):
    sah = s.solve(n, seed=seed, options=P.options(precision=precision, bvh=P.BVH_SAH, count=1))
    lbvh = s.solve(n, seed=seed, options=P.options(precision=precision, bvh=P.BVH_LBVH,
                                                   count=1))
    return sah, lbvh


def test_lbvh_full_field_equals_sah(product):
    """1000-heliostat field with its 64x64 receiver map (10,192 triangles),
    4e6 paths: globals, receiver and all 8192 per-primitive estimates."""
    s, h = W.heliostat_field(product)
    sah, lbvh = _solve_pair(s, 4_000_000, seed=5)
    st, sl = sah.stats(), lbvh.stats()
    assert st["bvh_device"] == 0 and sl["bvh_device"] == 1
    assert sl["bvh_nodes"] == 2 * 1000 + 2 * 64 * 64 - 1
    assert 1 <= sl["bvh_depth"] <= 30
    assert sl["rays"] == st["rays"] and sl["bounces"] == st["bounces"]
    assert sl["triangle_tests"] > 0 and sl["node_visits"] > 0
    _same(lbvh.globals(), sah.globals(), "globals")
    _same(lbvh.receiver(h["receiver"]), sah.receiver(h["receiver"]), "receiver")
    pl = lbvh.primitives(h["receiver"], h["receiver_shape"])
    ps = sah.primitives(h["receiver"], h["receiver_shape"])
    assert len(pl) == len(ps) == 2 * 64 * 64
    for i, (a, b) in enumerate(zip(pl, ps)):
        _same(a, b, ("primitive", i))
    s.close()


def test_lbvh_beam_down_equals_sah(product):
    """Beam-down scene: 5000 punched paraboloids, a hyperboloid, the glass
    window and the receiver grid (quadric patches in the device build), 1e6
    paths with the roulette in FP32, 2e5 in FP64."""
    s, h = W.beam_down(product)
    sah, lbvh = _solve_pair(s, 1_000_000, seed=9)
    assert lbvh.stats()["bvh_device"] == 1
    assert lbvh.stats()["killed"] == sah.stats()["killed"]
    _same(lbvh.globals(), sah.globals(), "globals")
    _same(lbvh.receiver(h["receiver"]), sah.receiver(h["receiver"]), "receiver")
    # the FP64 build's device tree (boxes and Morton codes in FP64)
    sah, lbvh = _solve_pair(s, 200_000, seed=10, precision=P.FP64)
    assert lbvh.stats()["bvh_device"] == 1
    _same(lbvh.globals(), sah.globals(), "fp64 globals")
    _same(lbvh.receiver(h["receiver"]), sah.receiver(h["receiver"]), "fp64 receiver")
    s.close()


def test_lbvh_fp64_and_single_mirror(product):
    """The FP64 build of a reduced field, and the single-mirror scene (four
    triangles), with either builder."""
    s, h = W.heliostat_field(product, n_helio=200, receiver_cells=16)
    sah, lbvh = _solve_pair(s, 1_000_000, seed=3, precision=P.FP64)
    assert lbvh.stats()["bvh_device"] == 1
    _same(lbvh.globals(), sah.globals(), "fp64 globals")
    _same(lbvh.receiver(h["receiver"]), sah.receiver(h["receiver"]), "fp64 receiver")
    s.close()
    s, h = W.single_mirror(product)
    sah, lbvh = _solve_pair(s, 1_000_000, seed=0)
    assert lbvh.stats()["bvh_nodes"] == 3
    _same(lbvh.globals(), sah.globals(), "mirror globals")
    _same(lbvh.receiver(h["receiver"]), sah.receiver(h["receiver"]), "mirror receiver")
    s.close()


def test_lbvh_two_primitives(product):
    """The smallest scene the device builds: one 10x10 matte rectangle (two
    triangles), sampled and receiving on its front, under a tilted sun."""
    s = P.Scene(product)
    sq = s.rectangle(5, 5)
    m = s.matte(0.6)
    inst = s.instance(s.object([(sq, m, m)]), receiver=P.SSOL_FRONT)
    s.set_sun("directional", (0.2, 0.1, -1.0), 1000.0)
    sah, lbvh = _solve_pair(s, 500_000, seed=2)
    assert lbvh.stats()["bvh_device"] == 1 and lbvh.stats()["bvh_nodes"] == 1
    assert lbvh.stats()["bvh_depth"] == 1
    _same(lbvh.globals(), sah.globals(), "globals")
    _same(lbvh.receiver(inst, P.SSOL_FRONT), sah.receiver(inst, P.SSOL_FRONT), "front")
    s.close()


def _deep_layout(lib):
    """36 small horizontal matte triangles whose Morton codes are 0 (five of
    them), each single bit of the 30 (one triangle per axis and bit) and all
    ones: the linear hierarchy peels one triangle off per level, 33 levels
    deep, more than the traversal stack holds."""
    s = P.Scene(lib)
    centres = [(0.1 * k, 0.0, 0.0) for k in range(5)]
    for lvl in range(10):
        v = 2.0 ** lvl + 0.5
        centres += [(v, 0.0, 0.0), (0.0, v, 0.0), (0.0, 0.0, v)]
    centres.append((1024.0, 1024.0, 1024.0))
    a = 0.04
    verts, ids = [], []
    for (x, y, z) in centres:
        b = len(verts)
        verts += [(x - a, y - a, z), (x + a, y - a, z), (x, y + a, z)]
        ids.append((b, b + 1, b + 2))
    mesh = s.mesh(verts, ids)
    m = s.matte(0.5)
    inst = s.instance(s.object([(mesh, m, m)]), receiver=P.SSOL_FRONT | P.SSOL_BACK)
    s.set_sun("directional", (0.1, 0.2, -1.0), 1000.0)
    return s, inst


def test_lbvh_chain_layout_is_restructured(product):
    """The treelet restructuring balances the 33-level chain of the linear
    hierarchy to about half that depth, so the tree is built on the device and
    traced as is, with the SAH tree's results."""
    s, inst = _deep_layout(product)
    sah, lbvh = _solve_pair(s, 200_000, seed=1)
    st, sl = sah.stats(), lbvh.stats()
    assert sl["bvh_device"] == 1 and st["bvh_device"] == 0
    assert 1 <= sl["bvh_depth"] <= 20
    assert sl["bvh_nodes"] == 35
    _same(lbvh.globals(), sah.globals(), "globals")
    _same(lbvh.receiver(inst, P.SSOL_FRONT), sah.receiver(inst, P.SSOL_FRONT), "front")
    s.close()


def test_default_builder_by_solve_size(product):
    """With the default options, ssol_solve builds the tree on the device for
    solves of at most 2^24 realisations and on the host above; a plan, which
    does not know its solve size, gets the host tree."""
    import ctypes as C
    s, h = W.single_mirror(product)
    assert s.solve(100_000, seed=1).stats()["bvh_device"] == 1
    assert s.solve((1 << 24) + 1, seed=1).stats()["bvh_device"] == 0
    assert s.solve(100_000, seed=1, options=P.options()).stats()["bvh_device"] == 1
    plan = C.c_void_p()
    product.call("ssol_b200_plan_create", s.scn, None, C.byref(plan))
    st = P.B200Stats()
    product.call("ssol_b200_plan_get_stats", plan, C.byref(st))
    assert st.bvh_device == 0 and st.bvh_nodes >= 1
    product.call("ssol_b200_plan_ref_put", plan)
    s.close()


def test_work_counters_are_optional(product):
    """FP32 solves count rays, node visits and primitive tests only when the
    options ask for it; the estimates are the same either way, and so are
    the counters that are always kept (paths, bounces)."""
    s, h = W.heliostat_field(product, n_helio=200, receiver_cells=16)
    off = s.solve(2_000_000, seed=6)
    on = s.solve(2_000_000, seed=6, options=P.options(count=1))
    so, sn = off.stats(), on.stats()
    for k in ("rays", "node_visits", "triangle_tests", "quadric_tests"):
        assert so[k] == 0, k
    assert sn["rays"] > 0 and sn["node_visits"] > sn["rays"] and sn["triangle_tests"] > 0
    assert so["paths"] == sn["paths"] == 2_000_000 and so["bounces"] == sn["bounces"]
    _same(off.globals(), on.globals(), "globals")
    _same(off.receiver(h["receiver"]), on.receiver(h["receiver"]), "receiver")
    s.close()


def test_large_default_solve_switches_trees(product):
    """A default ssol_solve above 2^24 realisations traces its first 2^24 on
    the device-built tree and the rest on the host SAH tree built meanwhile:
    the same estimates as a solve on either tree alone, and the stats name
    the tree it ended on."""
    s, h = W.heliostat_field(product, n_helio=300, receiver_cells=16)
    n = (1 << 24) + 3_000_000
    both = s.solve(n, seed=21)
    sah = s.solve(n, seed=21, options=P.options(bvh=P.BVH_SAH))
    lbvh = s.solve(n, seed=21, options=P.options(bvh=P.BVH_LBVH))
    sb = both.stats()
    assert sb["bvh_device"] == 0 and sb["paths"] == n and sb["kernel_ms"] > 0
    assert both.count("realisation_count") == n
    for other in (sah, lbvh):
        _same(both.globals(), other.globals(), "globals")
        _same(both.receiver(h["receiver"]), other.receiver(h["receiver"]), "receiver")
    s.close()
