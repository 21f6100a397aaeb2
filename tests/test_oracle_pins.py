"""The CPU oracle against the closed-form answers of the reference's solver
tests. These pins are what makes the oracle trustworthy as the checker of the
B200 library: each assertion restates one CHK of a reference test file."""
import math

import pytest

import pyssol as P
import ref_scenes as R

N = 10000


def test_solver1_sample_all(oracle):
    """src/test_ssol_solver1.c:312-351: sampling all three squares; the
    target is shadowed by the secondary and receives 4 DNI cos45."""
    s, h = R.solver1_base(oracle)
    est = s.solve(N, seed=1)
    assert est.count("realisation_count") == N
    assert est.count("failed_count") == 0
    m = 4 * R.DNI * R.COS45
    std = math.sqrt(((12 * R.DNI * R.COS45) ** 2 / 3 - (4 * R.DNI * R.COS45) ** 2) / N)
    g = est.globals()
    assert abs(g["shadowed"][0] - m) <= 2 * std
    assert abs(g["missing"][0] - 2 * m) <= 2 * g["missing"][2]
    rcv = est.receiver(h["target"])
    assert abs(rcv["incoming_flux"][0] - m) <= 3 * std
    assert abs(rcv["incoming_flux"][2] - std) <= std * 1e-2
    assert est.sampled_area() == pytest.approx(12, abs=1e-12)
    assert est.count("sampled_count") == 3


def test_solver1_sample_primary(oracle):
    """src/test_ssol_solver1.c:354-373: only the primary is sampled; the
    incoming flux on the target is exactly 4 DNI cos45 with zero variance."""
    s, h = R.solver1_base(oracle)
    oracle.call("ssol_instance_sample", h["target"], 0)
    oracle.call("ssol_instance_sample", h["secondary"], 0)
    est = s.solve(N, seed=2)
    m = 4 * R.DNI * R.COS45
    g = est.globals()
    assert abs(g["shadowed"][0]) <= 1e-4
    assert g["missing"][0] == pytest.approx(m, rel=1e-4)
    assert g["cos_factor"][0] == pytest.approx(R.COS45, rel=1e-4)
    rcv = est.receiver(h["target"])
    assert rcv["incoming_flux"][0] == pytest.approx(m, rel=1e-8)
    assert abs(rcv["incoming_flux"][2]) <= 1e-4


def test_solver1_atmosphere(oracle):
    """src/test_ssol_solver1.c:402-485: reflectivity 0.87 and k = 0.03 give
    incoming = 0.87 4 e^(-0.03 4 sqrt2) DNI cos45; energy is conserved and the
    per-primitive flux integrates to the receiver flux."""
    s, h = R.solver1_base(oracle)
    oracle.call("ssol_instance_sample", h["target"], 0)
    oracle.call("ssol_instance_sample", h["secondary"], 0)
    oracle.call("ssol_scene_detach_instance", s.scn, h["heliostat"])
    m_mtl2 = s.mirror(0.87, 0.0)
    obj2 = s.object([(h["square"], m_mtl2, m_mtl2)])
    s.instance(obj2, receiver=P.SSOL_FRONT)
    s.atmosphere(0.03)
    oracle.call("ssol_instance_set_receiver", h["target"], P.SSOL_FRONT, 1)
    est = s.solve(N, seed=3)
    k = math.exp(-0.03 * 4 * math.sqrt(2))
    a_m = 0.87 * 4 * k * R.DNI * R.COS45
    m = 4 * R.DNI * R.COS45
    g = est.globals()
    total = sum(g[q][0] for q in ("missing", "shadowed", "absorbed_by_receivers",
                                  "extinguished_by_atmosphere", "other_absorbed"))
    assert total == pytest.approx(m, rel=1e-4)
    assert g["cos_factor"][0] == pytest.approx(R.COS45, rel=1e-4)
    rcv = est.receiver(h["target"])
    assert rcv["incoming_flux"][0] == pytest.approx(a_m, rel=1e-4)
    prims = est.primitives(h["target"], h["square"])
    area = 2.0  # each triangle of the 2x2 square
    assert sum(p["incoming_flux"][0] * area for p in prims) == pytest.approx(a_m, rel=1e-4)


def test_solver1_monochromatic_spectral_extinction(oracle):
    """src/test_ssol_solver1.c:491-528: a sun at wavelength 1.21 through an
    extinction spectrum {1, 2} x {0.1, 0.2} interpolates k = 0.121."""
    s, h = R.solver1_base(oracle)
    oracle.call("ssol_instance_sample", h["target"], 0)
    oracle.call("ssol_instance_sample", h["secondary"], 0)
    mono = s.spectrum([1.21], [1.0])
    s.set_sun("directional", (1, 0, -1), R.DNI, spectrum=mono)
    ext = s.spectrum([1, 2], [0.1, 0.2])
    s.atmosphere(ext)
    est = s.solve(N, seed=4)
    k2 = math.exp(-0.121 * 4 * math.sqrt(2))
    m = 4 * k2 * R.DNI * R.COS45
    g = est.globals()
    assert g["missing"][0] == pytest.approx(m, rel=1e-4)
    rcv = est.receiver(h["target"])
    assert rcv["incoming_flux"][0] == pytest.approx(m, rel=1e-4)
    assert abs(rcv["incoming_flux"][2]) <= 1e-4


@pytest.mark.parametrize("kind,param", [("pillbox", 1.0), ("gaussian", 0.01),
                                        ("buie", 0.1)])
def test_solver10_12_flat_exact(oracle, kind, param):
    """src/test_ssol_solver10.c:128-181 (and 11, 12): whatever the sunshape,
    the flat absorbing square gets exactly DNI x 100 with zero variance; the
    paraboloid gets DNI x 100 within 3 standard errors."""
    s, h = R.flat_and_parabol(oracle, kind, param)
    est = s.solve(N, seed=5)
    g = est.globals()
    assert g["cos_factor"][0] == 1.0
    assert g["cos_factor"][2] == 0.0
    assert g["absorbed_by_receivers"][0] == R.DNI * 100
    assert g["absorbed_by_receivers"][2] == 0.0
    geom2 = R.add_parabol_10(s, h["matte"])
    oracle.call("ssol_scene_detach_instance", s.scn, h["geom1"])
    est = s.solve(100000, seed=6)
    g = est.globals()
    assert abs(g["absorbed_by_receivers"][0] - R.DNI * 100) <= \
        3 * g["absorbed_by_receivers"][2]
    assert est.count("failed_count") == 0
    del geom2


def test_oracle_tracked_paths(oracle):
    """src/test_ssol_solver1.c:177-207: a tracked solve of one realisation
    records one path with vertices; the sun and infinite segments follow the
    tracker lengths (negative: 0.75 x the scene's largest extent)."""
    s, h = R.solver1_base(oracle)
    e = s.solve(1, seed=0, tracker=(-1, -1))
    paths = e.paths()
    assert len(paths) == 1 and len(paths[0][1]) != 0
    e = s.solve(200, seed=3, tracker=(2.0, 5.0))
    paths = e.paths()
    assert len(paths) == 200
    for kind, verts in paths:
        (x0, w0), (x1, w1) = verts[0], verts[1]
        assert w0 == 1000.0  # the sun end carries the DNI
        assert math.dist(x0, x1) == pytest.approx(2.0, rel=1e-9)
        if kind == "shadow":
            assert len(verts) == 2
        else:
            assert kind in ("success", "missing")
            xl, _ = verts[-1]
            assert math.dist(xl, verts[-2][0]) == pytest.approx(5.0, rel=1e-9)
