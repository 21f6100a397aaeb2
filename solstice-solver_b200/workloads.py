"""Synthetic solar-field workloads, described through the ssol C API.

No public benchmark scene ships with the reference, so these seeded
generators stand in for the solar fields the solver is used on. Every choice
that the workload descriptions leave open (frame, azimuth convention, field
sector, receiver tilt, back-face materials) is fixed here and documented in
the function docstrings.

Conventions: z up; azimuth measured from +y (north) clockwise toward +x
(east); the sun direction passed to ssol_sun_set_direction points from the
sun toward the scene.
"""
import math

import pyssol as P


def _unit(v):
    n = math.sqrt(sum(c * c for c in v))
    return tuple(c / n for c in v)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def to_sun(elevation_deg, azimuth_deg):
    el, az = math.radians(elevation_deg), math.radians(azimuth_deg)
    return (math.sin(az) * math.cos(el), math.cos(az) * math.cos(el), math.sin(el))


def frame_z_to(n, up=(0.0, 0.0, 1.0)):
    """Row-major rotation whose third column is n (local +z -> n)."""
    n = _unit(n)
    x = _cross(up, n)
    if sum(c * c for c in x) < 1e-12:
        x = (1.0, 0.0, 0.0)
    x = _unit(x)
    y = _cross(n, x)
    return ((x[0], y[0], n[0]), (x[1], y[1], n[1]), (x[2], y[2], n[2]))


def grid_mesh(scene, size_x, size_y, nx, ny):
    """Flat size_x x size_y rectangle split into nx x ny quads (2 triangles
    each, front face +z like the reference rectangle)."""
    verts = []
    for j in range(ny + 1):
        for i in range(nx + 1):
            verts.append((-0.5 * size_x + size_x * i / nx, -0.5 * size_y + size_y * j / ny, 0.0))
    ids = []
    for j in range(ny):
        for i in range(nx):
            a = j * (nx + 1) + i
            b, c, d = a + 1, a + nx + 2, a + nx + 1
            ids.append((a, c, b))
            ids.append((c, a, d))
    return scene.mesh(verts, ids)


# --------------------------------------------------------------- config 1
def single_mirror(lib, n_paths=1_000_000):
    """One 10x10 flat mirror and a 4x4 receiver 50 m along the reflected ray.

    Frame: to-sun s = (0, -cos45, sin45), to-receiver r = (0, cos45, sin45),
    so the mirror is horizontal at the origin. Sun: pillbox 4.65 mrad,
    DNI 1000, no atmosphere. Mirror: specular, reflectivity 0.9, both sides.
    Receiver: 4x4 at 50 r, front face toward the mirror, specular
    reflectivity 0.05 (absorptivity 0.95), front side receiver, not sampled.
    """
    s = P.Scene(lib)
    c = math.cos(math.pi / 4)
    sun_to = (0.0, -c, c)
    r = (0.0, c, c)
    mirror = s.rectangle(5, 5)
    m_mtl = s.mirror(0.9, 0.0)
    helio = s.instance(s.object([(mirror, m_mtl, m_mtl)]))
    rshape = s.rectangle(2, 2)
    r_mtl = s.mirror(0.05, 0.0)
    R = frame_z_to((-r[0], -r[1], -r[2]), up=(1.0, 0.0, 0.0))
    rcv = s.instance(s.object([(rshape, r_mtl, r_mtl)]),
                     P.transform_from(R, (50 * r[0], 50 * r[1], 50 * r[2])),
                     receiver=P.SSOL_FRONT, sample=0)
    s.set_sun("pillbox", tuple(-x for x in sun_to), 1000.0, param=4.65e-3)
    return s, {"heliostat": helio, "receiver": rcv, "receiver_shape": rshape,
               "n_paths": n_paths}


# --------------------------------------------------------------- config 2
def field_layout(n=1000, r_min=100.0, r_max=600.0, spacing=15.0, dr=14.0,
                 height=5.0):
    """Radial-staggered positions in a north sector, nearest first.

    Rows every `dr` metres from r_min; `spacing` metres between neighbours
    along a row; odd rows shifted by half a spacing. The sector half angle is
    the smallest (0.5 degree steps) that yields n positions within r_max.
    """
    def layout(half):
        pts = []
        k = 0
        rr = r_min
        while rr <= r_max + 1e-9:
            dphi = spacing / rr
            m = int(2 * half / dphi)
            off = 0.5 * dphi if k % 2 else 0.0
            for i in range(m + 1):
                phi = -half + off + i * dphi
                if phi > half:
                    break
                pts.append((rr * math.sin(phi), rr * math.cos(phi), height))
            k += 1
            rr += dr
        return pts

    half = math.radians(20)
    while True:
        pts = layout(half)
        if len(pts) >= n or half > math.radians(89):
            break
        half += math.radians(0.5)
    pts.sort(key=lambda p: (p[0] ** 2 + p[1] ** 2, p[0]))
    return pts[:n]


def heliostat_field(lib, n_helio=1000, elevation=30.0, azimuth=180.0, dni=900.0,
                    aim=(0.0, 0.0, 100.0), slope_error=2e-3, extinction=1e-4,
                    receiver_cells=64, per_primitive=True, reaim=None):
    """1000 flat 10x10 heliostats aimed at a 12x12 receiver on a 100 m tower.

    Heliostats: one object (2 triangles), instanced n_helio times on
    field_layout(); front: mirror reflectivity 0.9 with Beckmann slope error
    2 mrad; back: absorbing matte. Each normal bisects the to-sun direction
    and the direction to `aim`. Receiver: 12x12 plate centred on `aim`,
    facing the field centroid, specular reflectivity 0.05 (absorptivity
    0.95), split into receiver_cells^2 quads (2 triangles each) with
    per-primitive tallies on its front side. Sun: pillbox 4.65 mrad at
    (elevation, azimuth), DNI 900. Atmosphere: extinction 1e-4 /m.
    """
    s = P.Scene(lib)
    sun = to_sun(elevation, azimuth)
    pts = field_layout(n_helio)
    helio_shape = s.rectangle(5, 5)
    front = s.mirror(0.9, slope_error, P.BECKMANN)
    back = s.matte(0.0)
    hobj = s.object([(helio_shape, front, back)])
    helios, xfs = [], []
    for p in pts:
        a = _unit((aim[0] - p[0], aim[1] - p[1], aim[2] - p[2]))
        n = _unit((sun[0] + a[0], sun[1] + a[1], sun[2] + a[2]))
        xfs.append(P.transform_from(frame_z_to(n), p))
        helios.append(s.instance(hobj, xfs[-1]))
    cx = sum(p[0] for p in pts) / len(pts)
    cy = sum(p[1] for p in pts) / len(pts)
    cz = sum(p[2] for p in pts) / len(pts)
    rn = _unit((cx - aim[0], cy - aim[1], cz - aim[2]))
    rshape = grid_mesh(s, 12.0, 12.0, receiver_cells, receiver_cells)
    rmtl = s.mirror(0.05, 0.0)
    rcv = s.instance(s.object([(rshape, rmtl, rmtl)]), P.transform_from(frame_z_to(rn), aim),
                     receiver=P.SSOL_FRONT, per_primitive=1 if per_primitive else 0,
                     sample=0)
    s.set_sun("pillbox", tuple(-x for x in sun), dni, param=4.65e-3)
    if extinction:
        s.atmosphere(extinction)
    return s, {"heliostats": helios, "transforms": xfs, "receiver": rcv,
               "receiver_shape": rshape, "positions": pts, "sun": sun}


# --------------------------------------------------------------- config 3
def sun_grid(n_el=16, n_az=16, el_range=(5.0, 85.0), seed=0, dni_range=(300.0, 1000.0),
             budget_range=(1e5, 1e7)):
    """Sun positions of the batched workload: n_el elevations evenly spaced in
    el_range x n_az azimuths 0, 360/n_az, ...; per sun a DNI uniform in
    dni_range and a realisation budget log-uniform in budget_range, both
    drawn from a seeded generator."""
    import random
    rnd = random.Random(seed)
    suns = []
    for i in range(n_el):
        el = el_range[0] + (el_range[1] - el_range[0]) * i / max(1, n_el - 1)
        for j in range(n_az):
            az = 360.0 * j / n_az
            dni = rnd.uniform(*dni_range)
            lo, hi = math.log(budget_range[0]), math.log(budget_range[1])
            budget = int(math.exp(rnd.uniform(lo, hi)))
            suns.append({"elevation": el, "azimuth": az, "dni": dni, "budget": budget})
    return suns


def tracking_inputs(h, suns, aim=(0.0, 0.0, 100.0)):
    """Arguments of a tracking batch (pyssol.Batch.tracking) for the
    heliostats of a heliostat_field scene `h` and sun_grid entries: every
    heliostat aims at `aim`; per sun the direction from the sun toward the
    scene and the DNI. The device turns the heliostats with the rule
    heliostat_field follows, so item i is the field heliostat_field builds
    for sun i."""
    aims = [aim] * len(h["heliostats"])
    sp = [(tuple(-c for c in to_sun(sn["elevation"], sn["azimuth"])), sn["dni"]) for sn in suns]
    return h["heliostats"], aims, sp


def batched_fields(lib, suns, n_helio=1000, receiver_cells=64):
    """One heliostat_field scene per sun, heliostats re-aimed for that sun."""
    out = []
    for sun in suns:
        s, h = heliostat_field(lib, n_helio=n_helio, elevation=sun["elevation"],
                               azimuth=sun["azimuth"], dni=sun["dni"],
                               receiver_cells=receiver_cells)
        out.append((s, h))
    return out


# --------------------------------------------------------------- config 4
def surround_layout(n=5000, r_min=40.0, spacing=12.0, dr=10.0, height=4.0):
    """Radial-staggered surround field (full circle), nearest rows first:
    rows every `dr` metres from r_min, floor(2 pi r / spacing) positions per
    row, odd rows shifted by half a step, truncated to n positions."""
    pts = []
    k = 0
    rr = r_min
    while len(pts) < n:
        m = int(2 * math.pi * rr / spacing)
        off = 0.5 if k % 2 else 0.0
        for i in range(m):
            phi = 2 * math.pi * (i + off) / m
            pts.append((rr * math.sin(phi), rr * math.cos(phi), height))
        k += 1
        rr += dr
    return pts[:n]


def beam_down(lib, n_helio=5000, elevation=60.0, azimuth=180.0, dni=1000.0,
              sun_sigma=2.5e-3, secondary_height=120.0, image_focal=10.0,
              secondary_half=20.0, receiver_cells=30):
    """Beam-down tower: 5000 punched paraboloid heliostats, a hyperboloid
    secondary and a ground receiver under a glass window.

    Heliostats: 8x8 m punched paraboloids on surround_layout() (r <= 800 m;
    about 440 m for 5000), focal length = slant range from the heliostat
    centre to the secondary's vertex, each normal bisecting the to-sun
    direction and the direction to the hyperboloid's image focus; front:
    specular mirror reflectivity 0.9, back: absorbing matte.
    Secondary: punched hyperboloid, vertex at `secondary_height`, real focal
    length = secondary_height (real focus on the ground at the receiver),
    image focal length `image_focal` (image focus at 130 m), carved
    2 secondary_half = 40 m square;
    front (facing the ground): mirror reflectivity 0.95 with a pillbox
    microfacet slope distribution of 1.5 mrad; back: absorbing matte.
    Receiver: 6x6 m on the ground (front up), matte reflectivity 0.1
    (absorptivity 0.9), receiver_cells^2 quads with per-primitive tallies.
    Window: 6.5x6.5 m thin dielectric (n 1.5, absorption 20 /m, 5 mm) 0.5 m
    above the receiver, both sides. Sun: Gaussian sigma 2.5 mrad at
    (elevation, azimuth), DNI 1000, no atmosphere. Only the heliostats are
    sampled.
    """
    s = P.Scene(lib)
    sun = to_sun(elevation, azimuth)
    f2 = (0.0, 0.0, secondary_height + image_focal)
    vertex = (0.0, 0.0, secondary_height)
    pts = surround_layout(n_helio)
    front = s.mirror(0.9, 0.0)
    back = s.matte(0.0)
    carve = [(P.SSOL_AND, [(-4, -4), (-4, 4), (4, 4), (4, -4)])]
    helios = []
    for p in pts:
        a = _unit((f2[0] - p[0], f2[1] - p[1], f2[2] - p[2]))
        n = _unit((sun[0] + a[0], sun[1] + a[1], sun[2] + a[2]))
        focal = math.sqrt(sum((vertex[c] - p[c]) ** 2 for c in range(3)))
        shape = s.punched(P.Q_PARABOL, (focal,), carve)
        helios.append(s.instance(s.object([(shape, front, back)]),
                                 P.transform_from(frame_z_to(n), p)))
    q = secondary_half
    hyp = s.punched(P.Q_HYPERBOL, (image_focal, secondary_height),
                    [(P.SSOL_AND, [(-q, -q), (-q, q), (q, q), (q, -q)])])
    sec_mtl = s.mirror(0.95, 1.5e-3, P.PILLBOX)
    secondary = s.instance(s.object([(hyp, sec_mtl, back)]),
                           P.transform_from(None, vertex), sample=0)
    rshape = grid_mesh(s, 6.0, 6.0, receiver_cells, receiver_cells)
    rmtl = s.matte(0.1)
    receiver = s.instance(s.object([(rshape, rmtl, rmtl)]), receiver=P.SSOL_FRONT,
                          per_primitive=1, sample=0)
    air = s.medium(0.0, 1.0)
    glass = s.medium(20.0, 1.5)
    win_mtl = s.thin_dielectric(air, glass, 5e-3)
    window = s.instance(s.object([(s.rectangle(3.25, 3.25), win_mtl, win_mtl)]),
                        P.transform_from(None, (0.0, 0.0, 0.5)), sample=0)
    s.set_sun("gaussian", tuple(-x for x in sun), dni, param=sun_sigma)
    return s, {"heliostats": helios, "secondary": secondary, "receiver": receiver,
               "receiver_shape": rshape, "window": window, "positions": pts, "sun": sun}
