"""ssol_solve_adjoint: its primal objective against the CPU oracle's
restatement (same Philox streams), and its gradients against central finite
differences with common random numbers, on a scene without edge terms and on
one whose spots straddle the receiver's edge (the edge term).

Scene: four 2x2 heliostats around the foot of a 100 m tower, aimed at a
12x12 receiver; their spots (about 3 m) stay inside the receiver and no
heliostat shadows or blocks another, so nothing the adjoint leaves out
(changes of shadowing, blocking, the receiver's edges) contributes, and the
adjoint must equal the derivative of the estimator itself."""
import ctypes as C
import math
import os
import sys

import pytest

import pyssol as P
import workloads as W

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "solstice-solver_b200"))
import adjoint as A  # noqa: E402

pytestmark = pytest.mark.gpu

LOWER, UPPER, NX, NY = (-6.0, -6.0), (6.0, 6.0), 24, 24


def four_heliostats(lib):
    """Four 2x2 heliostats 3 m around the origin, aimed at a 12x12 receiver
    100 m above them (facing down). The heliostats sit near the origin so
    that the FP32 rounding of their vertices (about 1e-7 x 4 m) stays far
    below the 1e-4 m that a 1e-4 rad turn moves them."""
    s = P.Scene(lib)
    sun = W.to_sun(45.0, 135.0)
    aim = (0.0, 0.0, 100.0)
    front = s.mirror(0.9, 2e-3, P.BECKMANN)
    back = s.matte(0.0)
    obj = s.object([(s.rectangle(1, 1), front, back)])
    helios, xfs = [], []
    for p in ((3.0, 0.0, 1.0), (-3.0, 0.0, 1.0), (0.0, 3.0, 1.0), (0.0, -3.0, 1.0)):
        a = W._unit((aim[0] - p[0], aim[1] - p[1], aim[2] - p[2]))
        n = W._unit((sun[0] + a[0], sun[1] + a[1], sun[2] + a[2]))
        xfs.append(P.transform_from(W.frame_z_to(n), p))
        helios.append(s.instance(obj, xfs[-1]))
    rmtl = s.mirror(0.05, 0.0)
    rcv = s.instance(s.object([(W.grid_mesh(s, 12.0, 12.0, 4, 4), rmtl, rmtl)]),
                     P.transform_from(P.rotation_pitch_pi(), aim),
                     receiver=P.SSOL_FRONT, sample=0)
    s.set_sun("pillbox", tuple(-x for x in sun), 1000.0, param=4.65e-3)
    s.atmosphere(1e-4)
    return s, {"heliostats": helios, "transforms": xfs, "receiver": rcv}


def oracle_first_bounce(lib, s, rcv, n, seed):
    fn = lib.dll.ssol_oracle_first_bounce
    fn.argtypes = [P.VP, P.VP, C.c_size_t, P.VP, C.POINTER(C.c_double),
                   C.POINTER(C.c_double), C.c_uint, C.c_uint, C.POINTER(C.c_double),
                   C.POINTER(C.c_double), C.POINTER(C.c_ulonglong), C.POINTER(C.c_double)]
    a, se, h = C.c_double(), C.c_double(), C.c_ulonglong()
    m = (C.c_double * (NX * NY))()
    assert fn(s.scn, s.rng(seed=seed), n, rcv, (C.c_double * 2)(*LOWER),
              (C.c_double * 2)(*UPPER), NX, NY, C.byref(a), C.byref(se), C.byref(h), m) == 0
    return a.value, se.value, h.value, list(m)


@pytest.mark.parametrize("builder", ["four", "field"])
def test_adjoint_primal_matches_oracle(product, oracle, builder):
    if builder == "four":
        sg, hg = four_heliostats(product)
        sc, hc = four_heliostats(oracle)
    else:
        sg, hg = W.heliostat_field(product, n_helio=100, receiver_cells=16)
        sc, hc = W.heliostat_field(oracle, n_helio=100, receiver_cells=16)
    n = 2000000
    r = A.solve_adjoint(sg, hg["heliostats"], hg["receiver"], LOWER, UPPER, NX, NY, 0.0, n,
                        seed=3, want_map=True)
    a, se, hits, m = oracle_first_bounce(oracle, sc, hc["receiver"], n, 3)
    assert abs(r["absorbed"] - a) <= 3 * math.hypot(r["absorbed_se"], se) + 1e-6 * a
    assert abs(r["hits"] - hits) <= 1e-4 * hits + 2
    peak = max(m)
    assert max(abs(x - y) for x, y in zip(r["map"], m)) <= 1e-3 * peak
    spill = sum(x * x for x in m)
    assert abs(r["spillage"] - spill) <= 1e-3 * spill
    # device work of both passes: every sample that reaches the reflection
    # cast a shadow ray first, and each ray visits at least the root
    c = r["counters"]
    assert c["rays"] >= 2 * r["hits"] and c["node_visits"] >= c["rays"]
    assert c["triangle_tests"] > 0


def test_adjoint_matches_finite_differences(product):
    """h = 3e-3 rad keeps the turn far above the FP32 rounding of the vertices
    (the spot moves 0.6 m, about one cell); 4e7 paths keep the noise of the
    map-derivative estimator (tent kernels on a sharp spot) near 1 %."""
    s, h = four_heliostats(product)
    n = 40000000
    base = A.solve_adjoint(s, h["heliostats"], h["receiver"], LOWER, UPPER, NX, NY, 0.0,
                           n, seed=5, want_map=True)
    target = sum(base["map"]) / len(base["map"])
    field = A.AimField(s, h["heliostats"], h["transforms"], h["receiver"], LOWER, UPPER,
                       NX, NY, target, n, seed=5)
    params = [(i, k) for i in range(4) for k in range(2)]
    res, rows = A.finite_difference_check(field, params, h=3e-3)
    adj = [r["adjoint_spillage"] for r in rows]
    fd = [r["fd_spillage"] for r in rows]
    scale = max(abs(x) for x in fd)
    l2 = math.sqrt(sum((a - b) ** 2 for a, b in zip(adj, fd)) / sum(b * b for b in fd))
    assert l2 <= 0.05, rows
    for a, b in zip(adj, fd):
        assert abs(a - b) <= 0.06 * scale, rows
    for r in rows:
        # absorbed power: cosine and extinction terms only, smooth in theta
        assert abs(r["adjoint_absorbed"] - r["fd_absorbed"]) <= 1e-3 * abs(r["fd_absorbed"]), r


def test_torch_autograd_function(product):
    torch = pytest.importorskip("torch")
    s, h = four_heliostats(product)
    field = A.AimField(s, h["heliostats"], h["transforms"], h["receiver"], LOWER, UPPER,
                       NX, NY, 1000.0, 1000000, seed=7)
    theta = torch.zeros(4, 2, dtype=torch.float64, requires_grad=True)
    J = A.aim_objective().apply(theta, field)
    J[1].backward()
    direct = field.evaluate(gradients=True)
    assert torch.allclose(theta.grad.view(-1),
                          torch.tensor(direct["d_spillage"], dtype=torch.float64))
    assert J[1].item() == pytest.approx(direct["spillage"])


def edge_heliostats(lib, offset=5.0):
    """The four heliostats of four_heliostats, each aimed `offset` metres
    off the receiver's centre toward one of its sides, so that their spots
    (about 3 m) straddle the receiver's edge: turning one moves flux across
    the boundary, the receiver-edge term of the adjoint."""
    s = P.Scene(lib)
    sun = W.to_sun(45.0, 135.0)
    front = s.mirror(0.9, 2e-3, P.BECKMANN)
    back = s.matte(0.0)
    obj = s.object([(s.rectangle(1, 1), front, back)])
    helios, xfs = [], []
    for p, aim in (((3.0, 0.0, 1.0), (offset, 0.0, 100.0)),
                   ((-3.0, 0.0, 1.0), (-offset, 0.0, 100.0)),
                   ((0.0, 3.0, 1.0), (0.0, offset, 100.0)),
                   ((0.0, -3.0, 1.0), (1.0, -offset, 100.0))):
        a = W._unit((aim[0] - p[0], aim[1] - p[1], aim[2] - p[2]))
        n = W._unit((sun[0] + a[0], sun[1] + a[1], sun[2] + a[2]))
        xfs.append(P.transform_from(W.frame_z_to(n), p))
        helios.append(s.instance(obj, xfs[-1]))
    rmtl = s.mirror(0.05, 0.0)
    rcv = s.instance(s.object([(W.grid_mesh(s, 12.0, 12.0, 4, 4), rmtl, rmtl)]),
                     P.transform_from(P.rotation_pitch_pi(), (0.0, 0.0, 100.0)),
                     receiver=P.SSOL_FRONT, sample=0)
    s.set_sun("pillbox", tuple(-x for x in sun), 1000.0, param=4.65e-3)
    s.atmosphere(1e-4)
    return s, {"heliostats": helios, "transforms": xfs, "receiver": rcv}


def test_adjoint_receiver_edge_term(product):
    """Spots across the receiver's edge: the derivative of the absorbed power
    is mostly the flux crossing the boundary. The smoothed-boundary edge term
    (band of half a cell) must give the finite differences (h = 1e-3 rad,
    common random numbers, 2e7 paths) of both objectives: absorbed power to
    2 % and spillage to 5 % relative L2, cosine above 0.99."""
    s, h = edge_heliostats(product)
    n = 20000000
    base = A.solve_adjoint(s, h["heliostats"], h["receiver"], LOWER, UPPER, NX, NY, 0.0,
                           n, seed=5, want_map=True)
    target = sum(base["map"]) / len(base["map"])
    field = A.AimField(s, h["heliostats"], h["transforms"], h["receiver"], LOWER, UPPER,
                       NX, NY, target, n, seed=5)
    params = [(i, k) for i in range(4) for k in range(2)]
    _, rows = A.finite_difference_check(field, params, h=1e-3)
    for key, tol in (("absorbed", 0.02), ("spillage", 0.05)):
        a = [r["adjoint_" + key] for r in rows]
        b = [r["fd_" + key] for r in rows]
        nb = math.sqrt(sum(x * x for x in b))
        na = math.sqrt(sum(x * x for x in a))
        l2 = math.sqrt(sum((x - y) ** 2 for x, y in zip(a, b))) / nb
        cos = sum(x * y for x, y in zip(a, b)) / (na * nb)
        assert l2 <= tol and cos >= 0.99, (key, l2, cos, rows)
