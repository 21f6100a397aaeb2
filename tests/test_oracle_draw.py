"""Camera, image and renderer checks that need no GPU.

- Camera and image argument checks, layout, writes and sampling restate
  src/test_ssol_camera.c and src/test_ssol_image.c on both libraries (the
  B200 library's camera and image are host objects).
- The renderers' argument checks restate src/test_ssol_draw.c:310-390 on
  both libraries (every case fails before any device work).
- The oracle's renderers are checked against closed forms (draw_scenes)
  and for the writer's tile order (32 x 32 tiles, Morton order,
  src/ssol_draw.c:94-169)."""
import ctypes as C
import math

import numpy as np
import pytest

import draw_scenes as D
import pyssol as P


@pytest.fixture(params=["oracle", "product"])
def lib(request, oracle, product):
    return oracle if request.param == "oracle" else product


def test_camera_api(lib):
    s = P.Scene(lib)
    cam = C.c_void_p()
    assert lib.raw("ssol_camera_create", None, None) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_create", s.dev, None) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_create", None, C.byref(cam)) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_create", s.dev, C.byref(cam)) == P.RES_OK
    assert lib.raw("ssol_camera_ref_get", None) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_ref_get", cam) == P.RES_OK
    assert lib.raw("ssol_camera_ref_put", None) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_ref_put", cam) == P.RES_OK
    assert lib.raw("ssol_camera_set_proj_ratio", None, 0.0) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_set_proj_ratio", cam, 0.0) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_set_proj_ratio", None, 4 / 3) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_set_proj_ratio", cam, 4 / 3) == P.RES_OK
    assert lib.raw("ssol_camera_set_proj_ratio", cam, -4 / 3) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_set_fov", None, 0.0) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_set_fov", cam, 0.0) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_set_fov", None, math.pi / 4) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_set_fov", cam, math.pi / 4) == P.RES_OK
    assert lib.raw("ssol_camera_set_fov", cam, -math.pi / 4) == P.RES_BAD_ARG
    d3 = C.c_double * 3
    pos, tgt, up = d3(0, 0, 0), d3(0, 0, -1), d3(0, 1, 0)
    for a in (None, cam):
        for b in (None, pos):
            for c in (None, tgt):
                for d in (None, up):
                    expect = P.RES_OK if (a and b and c and d) else P.RES_BAD_ARG
                    assert lib.raw("ssol_camera_look_at", a, b, c, d) == expect
    assert lib.raw("ssol_camera_look_at", cam, pos, d3(0, 0, 0), up) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_look_at", cam, pos, tgt, d3(0, 0, 0)) == P.RES_BAD_ARG
    assert lib.raw("ssol_camera_ref_put", cam) == P.RES_OK
    s.close()


def _image(lib, s, w, h):
    img = C.c_void_p()
    lib.call("ssol_image_create", s.dev, C.byref(img))
    lib.call("ssol_image_setup", img, w, h, P.PIXEL_DOUBLE3)
    return img


def test_image_api(lib):
    """src/test_ssol_image.c:133-230"""
    s = P.Scene(lib)
    img = C.c_void_p()
    lib.call("ssol_image_create", s.dev, C.byref(img))
    assert lib.raw("ssol_image_ref_get", None) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_ref_get", img) == P.RES_OK
    assert lib.raw("ssol_image_ref_put", None) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_ref_put", img) == P.RES_OK
    assert lib.raw("ssol_image_setup", None, 128, 128, P.PIXEL_DOUBLE3) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_setup", img, 0, 128, P.PIXEL_DOUBLE3) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_setup", img, 32, 32, 99) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_setup", img, 128, 128, P.PIXEL_DOUBLE3) == P.RES_OK
    assert lib.raw("ssol_image_setup", img, 128, 128, P.PIXEL_DOUBLE3) == P.RES_OK
    assert lib.raw("ssol_image_setup", img, 16, 16, P.PIXEL_DOUBLE3) == P.RES_OK

    sz2 = C.c_size_t * 2
    block = (C.c_double * (8 * 8 * 3))(*([1.0] * 192))
    org, sz = sz2(0, 0), sz2(8, 8)
    for a in (None, img):
        for b in (None, org):
            for c in (None, sz):
                for d in (None, block):
                    expect = P.RES_OK if (a and b and c and d) else P.RES_BAD_ARG
                    assert lib.raw("ssol_image_write", a, b, c, P.PIXEL_DOUBLE3, d) == expect
    assert lib.raw("ssol_image_write", img, sz2(14, 0), sz, P.PIXEL_DOUBLE3, block) \
        == P.RES_BAD_ARG
    for (ox, oy), v in (((8, 0), 2.0), ((0, 8), 3.0), ((8, 8), 4.0)):
        b = (C.c_double * 192)(*([v] * 192))
        lib.call("ssol_image_write", img, sz2(ox, oy), sz, P.PIXEL_DOUBLE3, b)

    lay = P.ImageLayout()
    assert lib.raw("ssol_image_get_layout", None, None) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_get_layout", img, None) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_get_layout", None, C.byref(lay)) == P.RES_BAD_ARG
    lib.call("ssol_image_get_layout", img, C.byref(lay))
    assert lay.size > lay.offset
    assert lay.width == 16 and lay.height == 16
    assert lay.size - lay.offset >= 16 * 16
    assert lay.row_pitch >= 16
    assert lay.pixel_format == P.PIXEL_DOUBLE3
    mem = C.c_void_p()
    assert lib.raw("ssol_image_map", None, None) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_map", img, None) == P.RES_BAD_ARG
    assert lib.raw("ssol_image_map", None, C.byref(mem)) == P.RES_BAD_ARG
    lib.call("ssol_image_map", img, C.byref(mem))
    for y in range(16):
        row = C.cast(mem.value + lay.offset + y * lay.row_pitch, C.POINTER(C.c_double))
        for x in range(16):
            want = (1.0 if x < 8 else 2.0) if y < 8 else (3.0 if x < 8 else 4.0)
            assert row[x * 3] == want and row[x * 3 + 1] == want and row[x * 3 + 2] == want
    lib.call("ssol_image_unmap", img)
    lib.call("ssol_image_ref_put", img)
    s.close()


def test_image_sampling(lib):
    """check_sampling of src/test_ssol_image.c:24-107"""
    s = P.Scene(lib)
    img = _image(lib, s, 4, 2)
    lay = P.ImageLayout()
    lib.call("ssol_image_get_layout", img, C.byref(lay))
    mem = C.c_void_p()
    lib.call("ssol_image_map", img, C.byref(mem))
    colours = [[(1, 0, 0), (1, 0, 0), (1, 1, 0), (1, 1, 0)],
               [(1, 0, 1), (1, 0, 1), (0, 1, 1), (0, 1, 1)]]
    for y in range(2):
        for x in range(4):
            p = C.cast(mem.value + lay.offset + y * lay.row_pitch + x * 24,
                       C.POINTER(C.c_double))
            p[0], p[1], p[2] = colours[y][x]
    lib.call("ssol_image_unmap", img)
    pix = (C.c_double * 3)()

    def sample(filt, au, av, u, v):
        uv = (C.c_double * 2)(u, v)
        lib.call("ssol_image_sample", img, filt, au, av, uv, pix)
        return tuple(pix)

    NE, LI, CL, RE = P.FILTER_NEAREST, P.FILTER_LINEAR, P.ADDRESS_CLAMP, P.ADDRESS_REPEAT
    uv = (C.c_double * 2)(0, 0)
    for a in (None, img):
        for b in (None, uv):
            for c in (None, pix):
                expect = P.RES_OK if (a and b and c) else P.RES_BAD_ARG
                assert lib.raw("ssol_image_sample", a, NE, CL, CL, b, c) == expect
    assert sample(NE, CL, CL, 0, 0) == (1, 0, 0)
    assert sample(NE, CL, CL, 1 / 4, 0) == (1, 0, 0)
    assert sample(NE, CL, CL, 2 / 4, 0) == (1, 1, 0)
    assert sample(NE, CL, CL, 3 / 4, 0) == (1, 1, 0)
    assert sample(NE, CL, CL, -1 / 4, 0) == (1, 0, 0)
    assert sample(NE, RE, CL, -1 / 4, 0) == (1, 1, 0)
    assert sample(NE, CL, CL, 4 / 4, 0) == (1, 1, 0)
    assert sample(NE, RE, CL, 4 / 4, 0) == (1, 0, 0)
    assert sample(NE, CL, CL, 4 / 4, 1 / 2) == (0, 1, 1)
    assert sample(NE, RE, CL, 4 / 4, 2 / 2) == (1, 0, 1)
    assert sample(NE, RE, RE, 4 / 4, 2 / 2) == (1, 0, 0)
    assert sample(NE, CL, RE, 4 / 4, 2 / 2) == (1, 1, 0)
    assert sample(LI, CL, CL, 1 / 4 + 1 / 8, 1 / 4) == (0.75, 0.5, 0.5)
    lib.call("ssol_image_ref_put", img)
    s.close()


def test_draw_argument_checks(lib):
    """src/test_ssol_draw.c:310-390: every combination with a missing scene,
    camera, size, samples or writer fails, then a sun without spectrum"""
    s, cam = D.cornell_box(lib, spectrum=False)
    D.sun_without_spectrum(s, (0.577, 0.577, -0.577))

    def ok_writer(ctx, org, sz, fmt, pixels):
        return P.RES_OK
    wr = P.WRITE_PIXELS(ok_writer)
    null_wr = P.WRITE_PIXELS()
    up = (C.c_double * 3)(0, 0, 1)
    for kind in ("draft", "pt"):
        for spp in (0, 4):
            for w in (0, 256):
                for h in (0, 256):
                    for sc in (None, s.scn):
                        for cm in (None, cam):
                            for writer in (null_wr, wr):
                                if spp and w and h and sc and cm and writer:
                                    continue
                                if kind == "draft":
                                    r = lib.raw("ssol_draw_draft", sc, cm, w, h, spp,
                                                writer, None)
                                else:
                                    r = lib.raw("ssol_draw_pt", sc, cm, w, h, spp, up,
                                                writer, None)
                                assert r == P.RES_BAD_ARG
        # no sun spectrum
        if kind == "draft":
            assert lib.raw("ssol_draw_draft", s.scn, cam, 256, 256, 4, wr, None) \
                == P.RES_BAD_ARG
        else:
            assert lib.raw("ssol_draw_pt", s.scn, cam, 256, 256, 4, up, wr, None) \
                == P.RES_BAD_ARG
    s.close()


def test_draw_pt_needs_up(oracle):
    """src/test_ssol_draw.c:400-403"""
    s, cam = D.cornell_box(oracle)

    def ok_writer(ctx, org, sz, fmt, pixels):
        return P.RES_OK
    wr = P.WRITE_PIXELS(ok_writer)
    assert oracle.raw("ssol_draw_pt", s.scn, cam, 8, 8, 1, None, wr, None) == P.RES_BAD_ARG
    s.close()


def test_oracle_draft_facing_plane(oracle):
    s, cam, h = D.facing_plane(oracle)
    spp = 3
    _, img = s.draw("draft", cam, h["width"], h["height"], spp)
    d = D.camera_dirs(h["basis"], h["width"], h["height"], D.draft_offsets(spp))
    want = np.mean(-d[..., 2], axis=0)
    assert np.max(np.abs(img[..., 0] - want)) < 1e-12
    assert np.array_equal(img[..., 0], img[..., 1]) and np.array_equal(img[..., 0], img[..., 2])
    s.close()


def test_oracle_pt_mirror_sky(oracle):
    s, cam, h = D.mirror_sky(oracle)
    spp = 2
    _, img = s.draw("pt", cam, h["width"], h["height"], spp)
    offs = D.pixel_offsets_pt(h["width"], h["height"], spp)
    d = D.camera_dirs_per_pixel(h["basis"], h["width"], h["height"], offs)
    want = np.mean(0.1 * h["refl"] * np.abs(d[..., 2]), axis=0)
    assert np.max(np.abs(img[..., 0] - want)) < 1e-12
    s.close()


def test_oracle_pt_facing_plane(oracle):
    s, cam, h = D.facing_plane(oracle, width=32, height=32)
    spp = 16
    _, img = s.draw("pt", cam, 32, 32, spp)
    v = img[..., 0].ravel()
    # per pixel: mean of spp i.i.d. samples rho/pi + 0.1 rho cos, cos with
    # density 2 cos sin on the hemisphere (E = 2/3, Var = 1/2 - 4/9)
    se = 0.1 * h["rho"] * math.sqrt(0.5 - 4.0 / 9.0) / math.sqrt(spp * v.size)
    assert abs(v.mean() - h["pt_mean"]) < 4 * se
    s.close()


def test_oracle_tile_order(oracle):
    s, cam, _ = D.facing_plane(oracle, width=100, height=70)
    tiles = []
    s.draw("draft", cam, 100, 70, 1, tiles=tiles)
    ntx, nty = 4, 3
    n = 4 * 4
    want = []
    for code in range(n):
        x = sum(((code >> (2 * b)) & 1) << b for b in range(8))
        y = sum(((code >> (2 * b + 1)) & 1) << b for b in range(8))
        if x < ntx and y < nty:
            want.append((32 * x, 32 * y, min(32, 100 - 32 * x), min(32, 70 - 32 * y)))
    assert tiles == want
    s.close()


def test_oracle_draw_writer_error(oracle):
    s, cam, _ = D.facing_plane(oracle, width=64, height=64)
    calls = []

    def bad(ctx, org, sz, fmt, pixels):
        calls.append(1)
        return P.RES_IO_ERR
    wr = P.WRITE_PIXELS(bad)
    assert oracle.raw("ssol_draw_draft", s.scn, cam, 64, 64, 1, wr, None) == P.RES_IO_ERR
    assert len(calls) == 1
    s.close()


def test_oracle_draw_into_image(oracle):
    """ssol_image_write as the writer gives the same pixels as a Python one"""
    s, cam, h = D.facing_plane(oracle, width=40, height=24)
    _, ref = s.draw("draft", cam, 40, 24, 2)
    img = _image(oracle, s, 40, 24)
    wr = P.WRITE_PIXELS(("ssol_image_write", oracle.dll))
    oracle.call("ssol_draw_draft", s.scn, cam, 40, 24, 2, wr, img)
    mem = C.c_void_p()
    oracle.call("ssol_image_map", img, C.byref(mem))
    got = np.ctypeslib.as_array(C.cast(mem, C.POINTER(C.c_double)), shape=(24, 40, 3))
    assert np.array_equal(got, ref)
    oracle.call("ssol_image_ref_put", img)
    s.close()
