"""A C program as the caller: tests/c_caller/solve_mirror.c includes only
ssol.h and ssp.h, builds the single-mirror scene through the C API, solves
and prints the estimates. It is compiled and linked with gcc against both
shared libraries (the oracle and the B200 library, which export the same
symbols), and its printed estimates are compared with the same scene built
through the ctypes binding in Python (workloads.single_mirror).

The reference's own test programs (src/test_ssol_solver1.c and the rest) are C
callers of exactly this kind; this is the check that such a program links and
runs against the B200 library unchanged.
"""
import os
import shutil
import subprocess

import pytest

import pyssol as P
import workloads as W
from conftest import ROOT, _ensure_oracle, _ensure_product

SRC = os.path.join(ROOT, "tests", "c_caller", "solve_mirror.c")
GLOBALS = ("cos_factor", "absorbed_by_receivers", "shadowed", "missing")
RECEIVER = ("incoming_flux", "absorbed_flux")

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="no gcc")


def _compile(lib_path, out):
    lib_dir = os.path.dirname(lib_path)
    name = os.path.basename(lib_path)[3:-3]  # libX.so -> X
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-O2",
           "-I", os.path.join(ROOT, "include"), "-o", out, SRC,
           "-L", lib_dir, "-l" + name, "-Wl,-rpath," + lib_dir, "-lm"]
    subprocess.run(cmd, check=True, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return out


def _run(exe, n, seed):
    p = subprocess.run([exe, str(n), str(seed)], check=True, capture_output=True,
                       text=True, timeout=300)
    out = {}
    for line in p.stdout.splitlines():
        name, e, se = line.split()
        out[name] = (float(e), float(se))
    assert set(out) == set(GLOBALS + RECEIVER)
    return out


def _python(lib, n, seed):
    s, info = W.single_mirror(lib)
    est = s.solve(n, seed=seed)
    g = est.globals()
    r = est.receiver(info["receiver"])
    out = {k: (g[k][0], g[k][2]) for k in GLOBALS}
    out.update({k: (r[k][0], r[k][2]) for k in RECEIVER})
    return out


def test_c_caller_links_against_both_libraries(tmp_path):
    """Compiles with -Werror against the headers and links against the
    oracle and against the B200 library (no GPU needed to link)."""
    _compile(_ensure_oracle(), str(tmp_path / "solve_mirror_oracle"))
    _compile(_ensure_product(), str(tmp_path / "solve_mirror_b200"))


def test_c_caller_matches_python_binding_on_oracle(tmp_path, oracle):
    """Same scene, same seed, same library: the C program and the ctypes
    binding print identical numbers (the oracle is sequential, so bit-exact)."""
    exe = _compile(_ensure_oracle(), str(tmp_path / "solve_mirror_oracle"))
    n, seed = 50_000, 5
    c_out = _run(exe, n, seed)
    py_out = _python(oracle, n, seed)
    assert c_out == py_out
    assert c_out["incoming_flux"][0] > 0


@pytest.mark.gpu
def test_c_caller_on_b200(tmp_path, product, oracle):
    """The C program linked against the B200 library: the same numbers as the
    Python binding on the same library and seed (the same Philox stream;
    only the order of the FP64 atomic adds may differ, hence 1e-9), and
    within 4 standard errors (plus 1e-5 relative for the FP32 geometry) of
    the oracle on its own seed."""
    exe = _compile(_ensure_product(), str(tmp_path / "solve_mirror_b200"))
    n, seed = 2_000_000, 7
    c_out = _run(exe, n, seed)
    py_out = _python(product, n, seed)
    for k in GLOBALS + RECEIVER:
        e_c, se_c = c_out[k]
        e_p, se_p = py_out[k]
        assert e_c == pytest.approx(e_p, rel=1e-9, abs=1e-12), k
        # the SE of a quantity that is the same on every path (cos_factor
        # here) is rounding noise of sum(w^2)/N - (sum(w)/N)^2
        assert se_c == pytest.approx(se_p, rel=1e-6, abs=1e-7 * abs(e_p) + 1e-12), k
    ref = _python(oracle, 200_000, 11)
    for k in GLOBALS + RECEIVER:
        e_c, se_c = c_out[k]
        e_o, se_o = ref[k]
        # FP32 geometry: 1e-5 relative on top of the statistical bound
        tol = 4 * (se_c ** 2 + se_o ** 2) ** 0.5 + 1e-5 * abs(e_o)
        assert abs(e_c - e_o) <= tol, (k, e_c, e_o, tol)
    assert c_out["incoming_flux"][0] > 0


def test_struct_layouts_match_the_binding(tmp_path):
    """The ctypes mirrors of ssol_b200_options and ssol_b200_stats have the C
    structs' sizes and field offsets, and the binding's defaults and builder
    values are the header's (no GPU: nothing is called)."""
    import ctypes as C
    exe = str(tmp_path / "struct_sizes")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "c_caller", "struct_sizes.c")],
                   check=True, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    c = {k: int(v) for k, v in (line.split() for line in out.splitlines())}
    o, st = P.B200Options, P.B200Stats
    assert c["options.size"] == C.sizeof(o)
    assert c["options.bvh_builder"] == o.bvh_builder.offset
    assert c["options.count_work"] == o.count_work.offset
    assert c["stats.size"] == C.sizeof(st)
    assert c["stats.bvh_device"] == st.bvh_device.offset
    d = P.options()
    assert (c["default.precision"], c["default.block_size"], c["default.waves"],
            c["default.bvh_builder"], c["default.count_work"]) == \
        (d.precision, d.block_size, d.waves, d.bvh_builder, d.count_work)
    assert (c["builder.auto"], c["builder.sah"], c["builder.lbvh"]) == \
        (P.BVH_AUTO, P.BVH_SAH, P.BVH_LBVH)
