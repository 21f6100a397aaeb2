"""The host binned-SAH builder (solstice-solver_b200/csrc/bvh.cpp), checked
on the CPU: tests/bvh_host/check_bvh.cpp is compiled with the builder's own
source and run on primitive boxes of several layouts. For each layout, leaf
sizes 1 and 4 and 1, 4 and 16 threads, every primitive must sit in exactly
one leaf, every slot's box must hold what lies below it, the depth must stay
within the traversal stack's 30 levels, and the threads must change neither
the tree's depth, its node count nor its SAH cost (the splits do not depend
on them). The device-side traversal of these trees is what the GPU parity
tests check."""
import math
import os
import random
import shutil
import subprocess

import pytest

import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "solstice-solver_b200", "csrc")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("bvh") / "check_bvh")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + CSRC, "-I" + CUDA_INC,
                    os.path.join(ROOT, "tests", "bvh_host", "check_bvh.cpp"),
                    os.path.join(CSRC, "bvh.cpp"), "-o", out, "-lpthread"],
                   check=True, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return out


def _run(checker, boxes):
    text = "".join("%.17g %.17g %.17g %.17g %.17g %.17g\n" % tuple(b) for b in boxes)
    p = subprocess.run([checker], input=text, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True, timeout=300)
    assert p.returncode == 0, p.stdout
    assert p.stdout.count("ok") == 2, p.stdout
    return p.stdout


def _tri_box(pts):
    return [min(p[c] for p in pts) for c in range(3)] + [max(p[c] for p in pts) for c in range(3)]


def _field_boxes(n_helio=1000, cells=64, el=30.0, az=180.0, aim=(0.0, 0.0, 100.0)):
    """Triangle boxes of workloads.heliostat_field: 10x10 heliostats turned
    toward the aim point and a cells x cells receiver on the tower."""
    sun = W.to_sun(el, az)
    boxes = []

    def place(frame, origin, local):
        return [tuple(sum(frame[r][k] * q[k] for k in range(3)) + origin[r] for r in range(3))
                for q in local]

    for p in W.field_layout(n_helio):
        a = W._unit((aim[0] - p[0], aim[1] - p[1], aim[2] - p[2]))
        nrm = W._unit((sun[0] + a[0], sun[1] + a[1], sun[2] + a[2]))
        v = place(W.frame_z_to(nrm), p, [(-5, -5, 0), (5, -5, 0), (5, 5, 0), (-5, 5, 0)])
        boxes += [_tri_box([v[0], v[1], v[2]]), _tri_box([v[0], v[2], v[3]])]
    rn = W._unit((0.0 - aim[0], 350.0 - aim[1], 5.0 - aim[2]))
    frame = W.frame_z_to(rn)
    for j in range(cells):
        for i in range(cells):
            x0, x1 = -6 + 12 * i / cells, -6 + 12 * (i + 1) / cells
            y0, y1 = -6 + 12 * j / cells, -6 + 12 * (j + 1) / cells
            q = place(frame, aim, [(x0, y0, 0), (x1, y0, 0), (x1, y1, 0), (x0, y1, 0)])
            boxes += [_tri_box([q[0], q[2], q[1]]), _tri_box([q[2], q[0], q[3]])]
    return boxes


def test_field_layout(checker):
    """The 1000-heliostat field: 10,192 triangles, the parallel top levels."""
    boxes = _field_boxes()
    assert len(boxes) == 10192
    _run(checker, boxes)


def test_random_and_coincident_boxes(checker):
    """Seeded random boxes, then the same with a quarter of them stacked on
    one box (centroid ties, the median-split fallback)."""
    rnd = random.Random(5)
    boxes = []
    for _ in range(6000):
        c = [rnd.uniform(-100, 100) for _ in range(3)]
        h = [rnd.uniform(0.01, 2.0) for _ in range(3)]
        boxes.append([c[k] - h[k] for k in range(3)] + [c[k] + h[k] for k in range(3)])
    _run(checker, boxes)
    stacked = boxes[:4500] + [[1.0, 2.0, 3.0, 1.5, 2.5, 3.5]] * 1500
    _run(checker, stacked)


def test_small_and_chain_layouts(checker):
    """One to three primitives, and the chain of single-bit Morton codes
    (one triangle per axis and bit, five at the origin, one far corner)."""
    for n in (1, 2, 3):
        _run(checker, [[i, 0, 0, i + 0.5, 0.5, 0.5] for i in range(n)])
    centres = [(0.1 * k, 0.0, 0.0) for k in range(5)]
    for lvl in range(10):
        v = 2.0 ** lvl + 0.5
        centres += [(v, 0.0, 0.0), (0.0, v, 0.0), (0.0, 0.0, v)]
    centres.append((1024.0, 1024.0, 1024.0))
    a = 0.04
    _run(checker, [[x - a, y - a, z, x + a, y + a, z] for (x, y, z) in centres])


def test_depth_bound_on_a_geometric_chain(checker):
    """Boxes at positions halving toward the origin (2000 of them, sizes
    shrinking with them): the SAH split peels one off per level, so the
    depth cap and its median fallback must hold the tree to 30 levels."""
    boxes = []
    for i in range(2000):
        x = math.ldexp(1.0, -(i % 60)) * (1 + (i // 60) * 1e-3)
        s = x * 1e-3
        boxes.append([x - s, -s, -s, x + s, s, s])
    _run(checker, boxes)
