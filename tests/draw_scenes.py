"""Scenes and closed forms for the preview renderers (ssol_draw_draft,
ssol_draw_pt; src/ssol_draw_draft.c, src/ssol_draw_pt.c).

- `camera_dirs`: the camera rays of every pixel for given sub-pixel
  offsets, restating camera_ray (src/ssol_camera.h:41-62) in float32 with
  numpy, for closed forms that depend on the ray direction only.
- `draft_offsets`: the draft's per-sample sub-pixel offsets (Philox block
  (i, 0, 0, 4), key 0, two 24-bit uniforms), the same for every pixel.
- `facing_plane`: a matte square under a camera looking straight down;
  draft pixel = mean over samples of -d_z; path-traced mean radiance
  rho / pi (sun straight above, unshadowed) + 0.1 rho E[cos] with E[cos] =
  2/3 for the cosine-sampled bounce that escapes to the sky.
- `mirror_sky`: a perfect mirror seen obliquely; every camera ray is
  reflected to the sky, no direct sun term (specular), so the path-traced
  pixel is exactly 0.1 R |d_z| averaged over its samples.
- `cornell_box`: the scene of the reference's draw test
  (src/test_ssol_draw.c:80-210): walls, short and tall blocks, one matte of
  reflectivity 1, the sun along (1, 1, -1), camera at (278, -1000, 273).
"""
import math

import numpy as np

import pyssol as P

M32 = 0xFFFFFFFF


def philox(c, k):
    """Philox4x32-10 block of counter c (4 words) and key k (2 words)."""
    c0, c1, c2, c3 = c
    k0, k1 = k
    for r in range(10):
        if r:
            k0 = (k0 + 0x9E3779B9) & M32
            k1 = (k1 + 0xBB67AE85) & M32
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & M32, p1 & M32, \
            ((p0 >> 32) ^ c3 ^ k1) & M32, p0 & M32
    return c0, c1, c2, c3


def u24(x):
    return np.float32((x >> 8) * (1.0 / 16777216.0))


def draft_offsets(spp):
    out = []
    for i in range(spp):
        b = philox((i & M32, i >> 32, 0, 4), (0, 0))
        out.append((u24(b[0]), u24(b[1])))
    return out


def camera_basis(position, target, up, fov, ratio):
    """Basis of ssol_camera_look_at after set_proj_ratio and set_fov, FP32."""
    f = np.float32
    p = np.array(position, dtype=f)
    z = np.array(target, dtype=f) - p
    z = z / f(np.sqrt(np.sum(z * z, dtype=f)))
    x = np.cross(z, np.array(up, dtype=f)).astype(f)
    x = x / f(np.sqrt(np.sum(x * x, dtype=f)))
    y = np.cross(z, x).astype(f)
    y = y / f(np.sqrt(np.sum(y * y, dtype=f)))
    # look_at takes the depth from the field of view stored in FP32
    depth = f(1.0 / math.tan(float(f(fov)) * 0.5))
    return x, y * f(1.0 / ratio), z * depth, p


def _unit_f32_then_f64(d):
    """f3_normalize in FP32 (camera_ray), then d3_normalize in FP64 (Li)"""
    f = np.float32
    l2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    d = (d / np.sqrt(l2.astype(f))[..., None]).astype(f).astype(np.float64)
    return d / np.linalg.norm(d, axis=-1, keepdims=True)


def camera_dirs(basis, width, height, offsets):
    """(len(offsets), height, width, 3) float64 unit camera directions."""
    ax, ay, az, _ = (b.astype(np.float32) for b in basis)
    f = np.float32
    xs = np.arange(width, dtype=f)
    ys = np.arange(height, dtype=f)
    out = []
    for ox, oy in offsets:
        sx = (xs + f(ox)) * f(f(1) / f(width))
        sy = (ys + f(oy)) * f(f(1) / f(height))
        fx = (sx * f(2) - f(1))[None, :, None]
        fy = (sy * f(2) - f(1))[:, None, None]
        d = (ax[None, None, :] * fx + ay[None, None, :] * fy) + az[None, None, :]
        out.append(_unit_f32_then_f64(d.astype(f)))
    return np.stack(out)


def _sun(s, direction=(0, 0, -1)):
    s.set_sun("directional", direction, 1000.0)


def facing_plane(lib, rho=0.5, width=48, height=32, fov=math.pi / 4):
    s = P.Scene(lib)
    m = s.matte(rho)
    s.instance(s.object([(s.rectangle(20, 20), m, m)]))
    _sun(s)
    ratio = width / height
    pos, tgt, up = (0.0, 0.0, 10.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0)
    cam = s.camera(pos, tgt, up, fov=fov, ratio=ratio)
    basis = camera_basis(pos, tgt, up, fov, ratio)
    return s, cam, {"basis": basis, "width": width, "height": height, "rho": rho,
                    "pt_mean": rho / math.pi + 0.1 * rho * 2.0 / 3.0}


def mirror_sky(lib, refl=0.8, width=40, height=40):
    s = P.Scene(lib)
    m = s.mirror(refl, 0.0)
    s.instance(s.object([(s.rectangle(50, 50), m, m)]))
    _sun(s, (0.3, 0.0, -1.0))
    pos, tgt, up = (0.0, -20.0, 10.0), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0)
    fov = math.pi / 6
    cam = s.camera(pos, tgt, up, fov=fov, ratio=1.0)
    basis = camera_basis(pos, tgt, up, fov, 1.0)
    return s, cam, {"basis": basis, "width": width, "height": height, "refl": refl}


def pixel_offsets_pt(width, height, spp, seed=0):
    """Sub-pixel positions of the path tracer's samples: Philox block
    (id, 0, 5) keyed by the seed, id = pixel x spp + sample."""
    out = np.zeros((spp, height, width, 2), dtype=np.float32)
    for py in range(height):
        for px in range(width):
            for s in range(spp):
                i = (py * width + px) * spp + s
                b = philox((i & M32, i >> 32, 0, 5), (seed & M32, seed >> 32))
                out[s, py, px] = (u24(b[0]), u24(b[1]))
    return out


def camera_dirs_per_pixel(basis, width, height, offs):
    """Directions for per-pixel offsets offs (spp, height, width, 2)."""
    ax, ay, az, _ = (b.astype(np.float32) for b in basis)
    f = np.float32
    xs = np.arange(width, dtype=f)[None, None, :]
    ys = np.arange(height, dtype=f)[None, :, None]
    sx = (xs + offs[..., 0]) * f(f(1) / f(width))
    sy = (ys + offs[..., 1]) * f(f(1) / f(height))
    fx = (sx * f(2) - f(1))[..., None]
    fy = (sy * f(2) - f(1))[..., None]
    d = (ax * fx + ay * fy) + az
    return _unit_f32_then_f64(d.astype(f))


CORNELL_WALLS = [(552, 0, 0), (0, 0, 0), (0, 559, 0), (552, 559, 0),
                 (552, 0, 548), (0, 0, 548), (0, 559, 548), (552, 559, 548)]
CORNELL_TALL = [(423, 247, 0), (265, 296, 0), (314, 456, 0), (472, 406, 0),
                (423, 247, 330), (265, 296, 330), (314, 456, 330), (472, 406, 330)]
CORNELL_SHORT = [(130, 65, 0), (82, 225, 0), (240, 272, 0), (290, 114, 0),
                 (130, 65, 165), (82, 225, 165), (240, 272, 165), (290, 114, 165)]
CORNELL_BLOCK_IDS = [4, 5, 6, 6, 7, 4, 1, 2, 6, 6, 5, 1, 0, 3, 7, 7, 4, 0,
                     2, 3, 7, 7, 6, 2, 0, 1, 5, 5, 4, 0]
CORNELL_WALL_IDS = [0, 1, 2, 2, 3, 0, 4, 5, 6, 6, 7, 4, 1, 2, 6, 6, 5, 1,
                    0, 3, 7, 7, 4, 0, 2, 3, 7, 7, 6, 2]


def _tris(ids):
    return [tuple(ids[i:i + 3]) for i in range(0, len(ids), 3)]


def cornell_box(lib, width=64, height=64, spectrum=True):
    """src/test_ssol_draw.c:80-210, 280-300 (camera at PROJ_RATIO = width /
    height, fov pi/4)."""
    s = P.Scene(lib)
    m = s.matte(1.0)
    for verts, ids in ((CORNELL_WALLS, CORNELL_WALL_IDS), (CORNELL_SHORT, CORNELL_BLOCK_IDS),
                       (CORNELL_TALL, CORNELL_BLOCK_IDS)):
        s.instance(s.object([(s.mesh(verts, _tris(ids)), m, m)]))
    d = (1.0, 1.0, -1.0)
    n = math.sqrt(3.0)
    d = tuple(c / n for c in d)
    if spectrum:
        s.set_sun("directional", d, 1000.0)
    cam = s.camera((278.0, -1000.0, 273.0), (278.0, 0.0, 273.0), (0.0, 0.0, 1.0),
                   fov=math.pi / 4.0, ratio=width / height)
    return s, cam


def sun_without_spectrum(s, direction=(0, 0, -1)):
    """Attach a directional sun with a DNI but no spectrum (raw calls)."""
    import ctypes as C
    h = s._new("ssol_sun_create_directional", "ssol_sun_ref_put", s.dev)
    s.lib.call("ssol_sun_set_direction", h, (C.c_double * 3)(*direction))
    s.lib.call("ssol_sun_set_dni", h, 1000.0)
    s.lib.call("ssol_scene_attach_sun", s.scn, h)
    s.sun = h
    return h
