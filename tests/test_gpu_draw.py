"""The B200 renderers against the oracle and closed forms (draw_scenes).

Both libraries consume the same random numbers (draft offsets, per-sample
Philox streams of the path tracer), so pixels agree one by one except where
rounding sends a ray to another primitive (silhouettes, edges): the draft
and path-traced images are compared pixel by pixel with a bound on the
share of pixels that may differ. Closed forms are checked exactly (draft of
a plane, path-traced mirror reflecting to the sky) or statistically (matte
plane). The device entry points write a torch CUDA tensor; the host writer
gets the same image in 32 x 32 tiles in Morton order."""
import ctypes as C
import math

import numpy as np
import pytest

import draw_scenes as D
import pyssol as P

pytestmark = pytest.mark.gpu

PREC = [P.FP64, P.FP32]
PREC_IDS = ["fp64", "fp32"]


def device_image(s, kind, cam, w, h, spp, precision, up=(0, 0, 1), seed=0):
    import torch
    buf = torch.full((h, w, 3), -1.0, dtype=torch.float64, device="cuda")
    st = s.draw_device(kind, cam, w, h, spp, buf.data_ptr(), up=up, seed=seed,
                       options=P.options(precision=precision))
    torch.cuda.synchronize()
    return buf.cpu().numpy(), st


@pytest.mark.parametrize("precision", PREC, ids=PREC_IDS)
def test_gpu_draft_facing_plane(product, precision):
    s, cam, h = D.facing_plane(product)
    spp = 3
    img, st = device_image(s, "draft", cam, h["width"], h["height"], spp, precision)
    d = D.camera_dirs(h["basis"], h["width"], h["height"], D.draft_offsets(spp))
    want = np.mean(-d[..., 2], axis=0)
    tol = 1e-9 if precision == P.FP64 else 2e-6
    assert np.max(np.abs(img[..., 0] - want)) < tol
    assert st.paths == h["width"] * h["height"] * spp
    assert st.rays == st.paths
    s.close()


@pytest.mark.parametrize("precision", PREC, ids=PREC_IDS)
def test_gpu_pt_mirror_sky(product, precision):
    s, cam, h = D.mirror_sky(product)
    spp = 2
    img, st = device_image(s, "pt", cam, h["width"], h["height"], spp, precision)
    offs = D.pixel_offsets_pt(h["width"], h["height"], spp)
    d = D.camera_dirs_per_pixel(h["basis"], h["width"], h["height"], offs)
    want = np.mean(0.1 * h["refl"] * np.abs(d[..., 2]), axis=0)
    tol = 1e-9 if precision == P.FP64 else 2e-6
    assert np.max(np.abs(img[..., 0] - want)) < tol
    s.close()


@pytest.mark.parametrize("precision", PREC, ids=PREC_IDS)
def test_gpu_pt_facing_plane(product, oracle, precision):
    w = hh = 64
    spp = 16
    s, cam, h = D.facing_plane(product, width=w, height=hh)
    img, _ = device_image(s, "pt", cam, w, hh, spp, precision)
    v = img[..., 0].ravel()
    se = 0.1 * h["rho"] * math.sqrt(0.5 - 4.0 / 9.0) / math.sqrt(spp * v.size)
    assert abs(v.mean() - h["pt_mean"]) < 4 * se
    so, co, _ = D.facing_plane(oracle, width=w, height=hh)
    _, ref = so.draw("pt", co, w, hh, spp)
    assert np.max(np.abs(img - ref)) < (1e-9 if precision == P.FP64 else 1e-5)
    s.close()
    so.close()


def _compare(img, ref, tol, max_share):
    diff = np.abs(img - ref).max(axis=2)
    share = float(np.mean(diff > tol))
    assert share <= max_share, (share, float(diff.max()))
    return share


@pytest.mark.parametrize("precision", PREC, ids=PREC_IDS)
def test_gpu_draft_cornell(product, oracle, precision):
    w, h, spp = 96, 64, 4
    s, cam = D.cornell_box(product, w, h)
    _, img = s.draw("draft", cam, w, h, spp) if precision == P.FP32 else (
        None, device_image(s, "draft", cam, w, h, spp, precision)[0])
    so, co = D.cornell_box(oracle, w, h)
    _, ref = so.draw("draft", co, w, h, spp)
    assert ref.max() > 0.5 and ref.min() >= 0.0
    _compare(img, ref, 1e-5, 0.01)
    s.close()
    so.close()


@pytest.mark.parametrize("precision", PREC, ids=PREC_IDS)
def test_gpu_pt_cornell(product, oracle, precision):
    w, h, spp = 64, 64, 4
    s, cam = D.cornell_box(product, w, h)
    if precision == P.FP32:
        _, img = s.draw("pt", cam, w, h, spp, up=(0, 0, 1))
    else:
        img, _ = device_image(s, "pt", cam, w, h, spp, precision, up=(0, 0, 1))
    so, co = D.cornell_box(oracle, w, h)
    _, ref = so.draw("pt", co, w, h, spp, up=(0, 0, 1))
    assert ref.mean() > 0
    # paths that reach another primitive after a rounding difference differ
    # from there on; FP32 geometry moves more of them
    _compare(img, ref, 1e-6 * max(1.0, float(ref.max())),
             0.02 if precision == P.FP64 else 0.2)
    # and the images agree on average
    assert abs(img.mean() - ref.mean()) < 0.02 * ref.mean()
    s.close()
    so.close()


def test_gpu_draw_writer_tiles(product, oracle):
    """Host writer path: same tiles, same order, same pixels as the device
    entry point; a writer error stops the draw with that error"""
    w, h = 100, 70
    s, cam, _ = D.facing_plane(product, width=w, height=h)
    tiles = []
    _, img = s.draw("draft", cam, w, h, 2, tiles=tiles)
    so, co, _ = D.facing_plane(oracle, width=w, height=h)
    otiles = []
    so.draw("draft", co, w, h, 2, tiles=otiles)
    assert tiles == otiles
    dev, _ = device_image(s, "draft", cam, w, h, 2, P.FP32)
    assert np.array_equal(img, dev)

    def bad(ctx, org, sz, fmt, pixels):
        return P.RES_IO_ERR
    wr = P.WRITE_PIXELS(bad)
    assert product.raw("ssol_draw_draft", s.scn, cam, w, h, 1, wr, None) == P.RES_IO_ERR
    s.close()
    so.close()


def test_gpu_draw_into_image(product):
    s, cam, _ = D.facing_plane(product, width=40, height=24)
    _, ref = s.draw("draft", cam, 40, 24, 2)
    img = C.c_void_p()
    product.call("ssol_image_create", s.dev, C.byref(img))
    product.call("ssol_image_setup", img, 40, 24, P.PIXEL_DOUBLE3)
    wr = P.WRITE_PIXELS(("ssol_image_write", product.dll))
    product.call("ssol_draw_draft", s.scn, cam, 40, 24, 2, wr, img)
    mem = C.c_void_p()
    product.call("ssol_image_map", img, C.byref(mem))
    got = np.ctypeslib.as_array(C.cast(mem, C.POINTER(C.c_double)), shape=(24, 40, 3))
    assert np.array_equal(got, ref)
    product.call("ssol_image_ref_put", img)
    s.close()


@pytest.mark.parametrize("precision", PREC, ids=PREC_IDS)
def test_gpu_draft_vertex_normals(product, oracle, precision):
    """A flat square with vertex normals tilted by 0.3 rad: the draft shows
    cos(Ns, -dir), not cos(Ng, -dir)"""
    def scene(lib):
        s = P.Scene(lib)
        a = 0.3
        n = (math.sin(a), 0.0, math.cos(a))
        verts = [(-20, -20, 0), (20, -20, 0), (20, 20, 0), (-20, 20, 0)]
        m = s.matte(0.5)
        s.instance(s.object([(s.mesh(verts, [(0, 2, 1), (2, 0, 3)], normals=[n] * 4), m, m)]))
        s.set_sun("directional", (0, 0, -1), 1000.0)
        cam = s.camera((0, 0, 10), (0, 0, 0), (0, 1, 0), fov=math.pi / 4, ratio=1.0)
        return s, cam, n
    s, cam, n = scene(product)
    img, _ = device_image(s, "draft", cam, 32, 32, 1, precision)
    basis = D.camera_basis((0, 0, 10), (0, 0, 0), (0, 1, 0), math.pi / 4, 1.0)
    d = D.camera_dirs(basis, 32, 32, D.draft_offsets(1))[0]
    # vertex data are FP32 (struct ssol_vertex_data), normalised in FP64
    nf = np.array(n, dtype=np.float32).astype(np.float64)
    nf /= np.linalg.norm(nf)
    want = np.maximum(-(d[..., 0] * nf[0] + d[..., 2] * nf[2]), 0.0)
    assert np.max(np.abs(img[..., 0] - want)) < (1e-9 if precision == P.FP64 else 2e-6)
    so, co, _ = scene(oracle)
    _, ref = so.draw("draft", co, 32, 32, 1)
    assert np.max(np.abs(img - ref)) < (1e-9 if precision == P.FP64 else 2e-6)
    s.close()
    so.close()


@pytest.mark.parametrize("precision", PREC, ids=PREC_IDS)
def test_gpu_draw_paraboloid(product, oracle, precision):
    """Punched paraboloid mirrors and a matte target: quadric hits, their
    normals and the mirror's rough microfacet BRDF in the path tracer"""
    def scene(lib):
        s = P.Scene(lib)
        m = s.mirror(0.9, 0.002)
        mt = s.matte(0.6)
        para = s.punched(P.Q_PARABOL, (10.0,),
                         [(P.SSOL_AND, [(-3, -3), (3, -3), (3, 3), (-3, 3)])])
        s.instance(s.object([(para, m, m)]))
        s.instance(s.object([(s.rectangle(1.5, 1.5), mt, mt)]),
                   P.transform_from(None, (0, 0, 10)))
        s.set_sun("directional", (0.1, 0.0, -1.0), 1000.0)
        cam = s.camera((0.0, -25.0, 14.0), (0.0, 0.0, 3.0), (0.0, 0.0, 1.0),
                       fov=math.pi / 5, ratio=1.0)
        return s, cam
    s, cam = scene(product)
    so, co = scene(oracle)
    img, st = device_image(s, "draft", cam, 64, 64, 2, precision)
    _, ref = so.draw("draft", co, 64, 64, 2)
    assert st.quadric_tests > 0
    _compare(img, ref, 1e-5, 0.02)
    img, _ = device_image(s, "pt", cam, 64, 64, 8, precision, up=(0, 0, 1))
    _, ref = so.draw("pt", co, 64, 64, 8, up=(0, 0, 1))
    _compare(img, ref, 1e-6, 0.03 if precision == P.FP64 else 0.25)
    assert abs(img.mean() - ref.mean()) < 0.03 * ref.mean()
    s.close()
    so.close()
