"""Scenes of the reference's own solver tests, restated on the ssol API.

Each builder reproduces the geometry, materials, sun and receivers of one
reference test (paths relative to the reference tree) and returns the handles
the assertions need. The closed-form expectations live in the tests that use
these builders.
"""
import math

import pyssol as P

DNI = 1000.0
COS45 = math.cos(math.pi / 4)


def solver1_base(lib):
    """src/test_ssol_solver1.c:96-175: 2x2 heliostat at the origin, a flipped
    2x2 secondary at (2, 0, 2), a virtual 2x2 target at (4, 0, 0); sun
    (1, 0, -1), DNI 1000, spectrum {1, 2, 3} x {1, 0.8, 1}."""
    s = P.Scene(lib)
    square = s.rectangle(1, 1)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    m_obj = s.object([(square, m_mtl, m_mtl)])
    t_obj = s.object([(square, v_mtl, v_mtl)])
    heliostat = s.instance(m_obj, receiver=P.SSOL_FRONT)
    secondary = s.instance(m_obj, P.transform_from(P.rotation_pitch_pi(), (2, 0, 2)),
                           receiver=P.SSOL_FRONT)
    target = s.instance(t_obj, P.transform_from(None, (4, 0, 0)), receiver=P.SSOL_FRONT)
    spec = s.spectrum([1, 2, 3], [1, 0.8, 1])
    s.set_sun("directional", (1, 0, -1), DNI, spectrum=spec)
    return s, dict(square=square, heliostat=heliostat, secondary=secondary,
                   target=target, m_obj=m_obj, spec=spec)


def flat_and_parabol(lib, sun_kind, param):
    """src/test_ssol_solver10.c (pillbox 1 rad), 11.c (Buie CSR 0.1), 12.c
    (Gaussian 0.01): a 10x10 absorbing matte square at x = -10 seen by a
    vertical sun; then a 10x10 punched paraboloid f = 10 at x = +10."""
    s = P.Scene(lib)
    square = s.rectangle(5, 5)
    matte = s.matte(0.0)
    obj = s.object([(square, matte, matte)])
    geom1 = s.instance(obj, P.transform_from(None, (-10, 0, 0)), receiver=P.SSOL_FRONT)
    s.set_sun(sun_kind, (0, 0, -1), DNI, param=param)
    return s, dict(square=square, matte=matte, geom1=geom1)


def add_parabol_10(s, matte):
    poly = [(-5, -5), (-5, 5), (5, 5), (5, -5)]
    parabol = s.punched(P.Q_PARABOL, (10.0,), [(P.SSOL_AND, poly)])
    obj = s.object([(parabol, matte, matte)])
    return s.instance(obj, P.transform_from(None, (10, 0, 0)), receiver=P.SSOL_FRONT)
