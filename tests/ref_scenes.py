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


def rect_poly(hx, hy, y_min=None, y_max=None):
    """Carving polygon in the order of src/test_ssol_rect2D_geometry.h:51-56:
    (xmin, ymin), (xmin, ymax), (xmax, ymax), (xmax, ymin)."""
    y0 = -hy if y_min is None else y_min
    y1 = hy if y_max is None else y_max
    return [(-hx, y0), (-hx, y1), (hx, y1), (hx, y0)]


def _directional(s, direction):
    spec = s.spectrum([1, 2, 3], [1, 0.8, 1])
    s.set_sun("directional", direction, DNI, spectrum=spec)


def solver2(lib, punched_heliostats=False):
    """src/test_ssol_solver2.c:88-176 (and 2b.c with punched_heliostats):
    two 1x2 mirrors at x = -0.5 and x = +0.5 (meshes in 2.c, punched planes in
    2b.c), a flipped 2x2 punched-plane secondary at (2, 0, 2), a virtual
    target at (4, 0, 0) that is the 2x2 square in 2.c and the 1x2 rectangle
    in 2b.c; sun (1, 0, -1). Every instance but the target is a front
    receiver; only the heliostats are sampled."""
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    if punched_heliostats:
        hel = s.punched(P.Q_PLANE, (), [(P.SSOL_AND, rect_poly(0.5, 1))])
        tgt = s.rectangle(0.5, 1)
    else:
        hel = s.rectangle(0.5, 1)
        tgt = s.rectangle(1, 1)
    sec = s.punched(P.Q_PLANE, (), [(P.SSOL_AND, rect_poly(1, 1))])
    m_obj = s.object([(hel, m_mtl, m_mtl)])
    h1 = s.instance(m_obj, P.transform_from(None, (-0.5, 0, 0)), receiver=P.SSOL_FRONT)
    h2 = s.instance(m_obj, P.transform_from(None, (0.5, 0, 0)), receiver=P.SSOL_FRONT)
    secondary = s.instance(s.object([(sec, m_mtl, m_mtl)]),
                           P.transform_from(P.rotation_pitch_pi(), (2, 0, 2)),
                           receiver=P.SSOL_FRONT, sample=0)
    target = s.instance(s.object([(tgt, v_mtl, v_mtl)]), P.transform_from(None, (4, 0, 0)),
                        receiver=P.SSOL_FRONT, sample=0)
    _directional(s, (1, 0, -1))
    return s, dict(heliostat1=h1, heliostat2=h2, secondary=secondary, target=target)


def solver3(lib, heliostat_receiver=True):
    """src/test_ssol_solver3.c:76-136 (and test_ssol_by_receiver_integration.c
    with heliostat_receiver=False): a 20x20 punched-plane mirror at the
    origin, a flipped virtual 2x2 target at (0, 0, 2); sun (1, 0, -1)."""
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    plane = s.punched(P.Q_PLANE, (), [(P.SSOL_AND, rect_poly(10, 10))])
    heliostat = s.instance(s.object([(plane, m_mtl, m_mtl)]),
                           receiver=P.SSOL_FRONT if heliostat_receiver else 0)
    target = s.instance(s.object([(s.rectangle(1, 1), v_mtl, v_mtl)]),
                        P.transform_from(P.rotation_pitch_pi(), (0, 0, 2)),
                        receiver=P.SSOL_FRONT, sample=0)
    _directional(s, (1, 0, -1))
    return s, dict(heliostat=heliostat, target=target)


def solver4(lib):
    """src/test_ssol_solver4.c:74-144: a 20x20 punched paraboloid f = 10
    (100 slices) under a vertical sun; two flipped virtual 0.2x0.2 targets at
    the focus (z = 10) and 1e-4 above it."""
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    par = s.punched(P.Q_PARABOL, (10.0,), [(P.SSOL_AND, rect_poly(10, 10))], slices=100)
    heliostat = s.instance(s.object([(par, m_mtl, m_mtl)]))
    t_obj = s.object([(s.rectangle(0.1, 0.1), v_mtl, v_mtl)])
    t1 = s.instance(t_obj, P.transform_from(P.rotation_pitch_pi(), (0, 0, 10)),
                    receiver=P.SSOL_FRONT, sample=0)
    t2 = s.instance(t_obj, P.transform_from(P.rotation_pitch_pi(), (0, 0, 10 + 1e-4)),
                    receiver=P.SSOL_FRONT, sample=0)
    _directional(s, (0, 0, -1))
    return s, dict(heliostat=heliostat, target1=t1, target2=t2)


def solver5(lib):
    """src/test_ssol_solver5.c:74-136: a 20x20 punched parabolic cylinder
    f = 10 under a vertical sun; a flipped virtual 20x0.2 target along the
    focal line (z = 10)."""
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    cyl = s.punched(P.Q_PCYLINDER, (10.0,), [(P.SSOL_AND, rect_poly(10, 10))])
    heliostat = s.instance(s.object([(cyl, m_mtl, m_mtl)]))
    target = s.instance(s.object([(s.rectangle(10, 0.1), v_mtl, v_mtl)]),
                        P.transform_from(P.rotation_pitch_pi(), (0, 0, 10)),
                        receiver=P.SSOL_FRONT, sample=0)
    _directional(s, (0, 0, -1))
    return s, dict(heliostat=heliostat, target=target)


def solver6(lib):
    """src/test_ssol_solver6.c:131-176: two flipped 10x10 punched-plane
    mirrors at x = -25 and x = +25; above each at z = 10 a 10x10 square whose
    front is an absorbing matte (reflectivity 0) and back is virtual. Target 1
    (x = -25) is flipped and a front receiver: the sun crosses its virtual
    back and the mirror sends everything into its matte front. Target 2
    (x = +25) is not flipped and a back receiver: its matte front shadows
    mirror 2 entirely. Vertical sun."""
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    bck = s.matte(0.0)
    plane = s.punched(P.Q_PLANE, (), [(P.SSOL_AND, rect_poly(5, 5))])
    flip = P.rotation_pitch_pi()
    h1 = s.instance(s.object([(plane, m_mtl, m_mtl)]), P.transform_from(flip, (-25, 0, 0)))
    h2 = s.instance(s.object([(plane, m_mtl, m_mtl)]), P.transform_from(flip, (25, 0, 0)))
    sq = s.rectangle(5, 5)
    t1 = s.instance(s.object([(sq, bck, v_mtl)]), P.transform_from(flip, (-25, 0, 10)),
                    receiver=P.SSOL_FRONT, sample=0)
    t2 = s.instance(s.object([(sq, bck, v_mtl)]), P.transform_from(None, (25, 0, 10)),
                    receiver=P.SSOL_BACK, sample=0)
    _directional(s, (0, 0, -1))
    return s, dict(heliostat1=h1, heliostat2=h2, target1=t1, target2=t2)


def solver7(lib):
    """src/test_ssol_solver7.c:100-186: beam-down. A 4x4 punched paraboloid
    f = 10 sqrt2 H (H = 10) at x = 10 H, its axis turned toward the sun
    (1, 0, -1), focuses on the image focus of a 24x24 punched hyperboloid
    (real focal 9 H, image focal 1 H; mirror front, virtual back) placed at
    z = 9 H, which sends the beam to its real focus on a 2x2 target at the
    origin (matte reflectivity 0.1 front, virtual back, front receiver)."""
    H = 10.0
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    bck = s.matte(0.1)
    par = s.punched(P.Q_PARABOL, (10 * math.sqrt(2) * H,), [(P.SSOL_AND, rect_poly(2, 2))])
    c = math.cos(-0.25 * math.pi)
    sn = math.sin(-0.25 * math.pi)
    turn = ((c, 0, sn), (0, 1, 0), (-sn, 0, c))  # local +z -> (-1, 0, 1)/sqrt2
    heliostat = s.instance(s.object([(par, m_mtl, m_mtl)]), P.transform_from(turn, (10 * H, 0, 0)))
    hyp = s.punched(P.Q_HYPERBOL, (1 * H, 9 * H), [(P.SSOL_AND, rect_poly(12, 12))])
    secondary = s.instance(s.object([(hyp, m_mtl, v_mtl)]), P.transform_from(None, (0, 0, 9 * H)),
                           sample=0)
    target = s.instance(s.object([(s.rectangle(1, 1), bck, v_mtl)]), receiver=P.SSOL_FRONT,
                        sample=0)
    _directional(s, (1, 0, -1))
    return s, dict(heliostat=heliostat, secondary=secondary, target=target, total=16 * DNI)


def solver8(lib):
    """src/test_ssol_solver8.c:79-140: a punched parabolic cylinder f = 1
    carved to x in [-5, 5], y in [0, 4] under the sun (0, 1, -1); a flipped
    virtual 20x20 target at z = 4 collects sqrt2 x 40 DNI."""
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    cyl = s.punched(P.Q_PCYLINDER, (1.0,), [(P.SSOL_AND, rect_poly(5, None, 0, 4))])
    heliostat = s.instance(s.object([(cyl, m_mtl, m_mtl)]))
    target = s.instance(s.object([(s.rectangle(10, 10), v_mtl, v_mtl)]),
                        P.transform_from(P.rotation_pitch_pi(), (0, 0, 4)),
                        receiver=P.SSOL_FRONT, sample=0)
    _directional(s, (0, 1, -1))
    return s, dict(heliostat=heliostat, target=target, S=math.sqrt(2) * 40)


def cube_mesh(s, half):
    """src/test_ssol_cube_geometry.h:59-88: 8 corners, 12 triangles."""
    v = [(x, y, z) for x in (-half, half) for y in (-half, half) for z in (-half, half)]
    ids = [(0, 6, 4), (0, 2, 6), (0, 3, 2), (0, 1, 3), (2, 7, 6), (2, 3, 7),
           (4, 6, 7), (4, 7, 5), (0, 4, 5), (0, 5, 1), (1, 5, 7), (1, 7, 3)]
    return s.mesh(v, ids)


def solver9(lib):
    """src/test_ssol_solver9.c:78-133: a 10 m mirror cube centred at the
    origin, all faces sampled, under a vertical sun; a flipped virtual 6x10
    target at z = 6."""
    s = P.Scene(lib)
    m_mtl = s.mirror(1.0, 0.0)
    v_mtl = s.virtual()
    heliostat = s.instance(s.object([(cube_mesh(s, 5), m_mtl, m_mtl)]))
    target = s.instance(s.object([(s.rectangle(3, 5), v_mtl, v_mtl)]),
                        P.transform_from(P.rotation_pitch_pi(), (0, 0, 6)),
                        receiver=P.SSOL_FRONT, sample=0)
    _directional(s, (0, 0, -1))
    return s, dict(heliostat=heliostat, target=target, DNI_S=DNI * 100, DNI_TGT_S=DNI * 60)
