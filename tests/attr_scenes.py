"""Scenes with per-vertex attributes and spatially varying shaders (the
surface fragment of src/ssol_material.c:551-655), with closed forms.

All use a vertical directional sun, DNI 1000, and a virtual receiver that
collects everything reflected, so the receiver's incoming flux is DNI x the
integral of the mirror's reflectivity over its area."""
import math

import pyssol as P
import workloads as W

DNI = 1000.0


def ramp_mirror(lib, kind):
    """A 10x10 mirror (8x8 grid of quads) at the origin with a reflectivity
    shader that varies over it, and a flipped virtual 12x12 receiver at
    z = 5. kind:
      "P"  reflectivity 0.5 + 0.04 x   (x in [-5, 5])      -> mean 0.5
      "uv" reflectivity uv[0] with the default texcoords (the barycentric
           weight of a triangle's first vertex)            -> mean 1/3
      "tex" texcoords (x/10 + 1/2, y/10 + 1/2), reflectivity uv[0]^2
                                                          -> mean 1/3
    """
    s = P.Scene(lib)
    if kind == "P":
        refl = lambda wl, f: 0.5 + 0.04 * f.P[0]  # noqa: E731
        shape = W.grid_mesh(s, 10.0, 10.0, 8, 8)
        expected = 0.5
        exact = expected
    elif kind == "uv":
        refl = lambda wl, f: f.uv[0]  # noqa: E731
        shape = W.grid_mesh(s, 10.0, 10.0, 8, 8)
        expected = 1.0 / 3.0
        exact = expected
    else:
        refl = lambda wl, f: f.uv[0] * f.uv[0]  # noqa: E731
        n = 8
        verts, tex = [], []
        for j in range(n + 1):
            for i in range(n + 1):
                x, y = -5.0 + 10.0 * i / n, -5.0 + 10.0 * j / n
                verts.append((x, y, 0.0))
                tex.append((x / 10 + 0.5, y / 10 + 0.5))
        ids = []
        for j in range(n):
            for i in range(n):
                a = j * (n + 1) + i
                b, c, d = a + 1, a + n + 2, a + n + 1
                ids += [(a, c, b), (c, a, d)]
        shape = s.mesh(verts, ids, texcoords=tex)
        # per-vertex baking interpolates u^2 linearly inside each triangle;
        # the exact mean over the square is 1/3, the piecewise-linear one
        # 1/3 + (1/8)^2 / 6 per the trapezoid rule in u
        expected = 1.0 / 3.0 + (1.0 / 8) ** 2 / 6
        exact = 1.0 / 3.0
    m = s.mirror(refl, 0.0)
    mirror = s.instance(s.object([(shape, m, m)]))
    v = s.virtual()
    rcv = s.instance(s.object([(s.rectangle(6, 6), v, v)]),
                     P.transform_from(P.rotation_pitch_pi(), (0, 0, 5)),
                     receiver=P.SSOL_FRONT, sample=0)
    s.set_sun("directional", (0, 0, -1), DNI)
    return s, {"mirror": mirror, "receiver": rcv, "expected": DNI * 100 * expected,
               "exact": DNI * 100 * exact}


def tilted_normals(lib, alpha=0.1, dist=20.0, turn_z=False):
    """A flat 2x2 mirror whose vertex normals are all (sin a, 0, cos a): the
    vertical sun is reflected along (sin 2a, 0, cos 2a), onto a 4x4 receiver
    `dist` away on that line (with the geometric normal the light would go
    straight up and miss it). Incoming flux: DNI x 4 exactly.

    turn_z: the mirror's instance is turned by 90 degrees about z (the same
    square). Its third column is the identity's, so the vertex normals are
    kept in shape space (src/ssol_material.c:632-646) and the beam still
    goes along +x: the same DNI x 4."""
    s = P.Scene(lib)
    n = (math.sin(alpha), 0.0, math.cos(alpha))
    verts = [(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)]
    shape = s.mesh(verts, [(0, 2, 1), (2, 0, 3)], normals=[n] * 4)
    m = s.mirror(1.0, 0.0)
    if turn_z:
        s.instance(s.object([(shape, m, m)]),
                   (0.0, 1.0, 0.0, -1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0))
    else:
        s.instance(s.object([(shape, m, m)]))
    r = (math.sin(2 * alpha), 0.0, math.cos(2 * alpha))
    absorber = s.matte(0.0)
    rcv = s.instance(s.object([(s.rectangle(2, 2), absorber, absorber)]),
                     P.transform_from(W.frame_z_to(tuple(-c for c in r)),
                                      tuple(dist * c for c in r)),
                     receiver=P.SSOL_FRONT, sample=0)
    s.set_sun("directional", (0, 0, -1), DNI)
    return s, {"receiver": rcv, "expected": DNI * 4}
