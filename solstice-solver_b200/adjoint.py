"""Aim gradients of a heliostat field through ssol_solve_adjoint.

- `solve_adjoint`: one call of the C entry point (objective values, flux map,
  per-heliostat gradients of the absorbed power and of the spillage).
- `AimField`: aim offsets theta (n x 2: rotations about each heliostat's
  local x and y axes through its centre) applied to the instance transforms
  of a scene built through pyssol.
- `AimObjective`: a torch.autograd.Function whose forward is the solve and
  whose backward returns the adjoint gradient, so that the field can be
  optimised with torch.
- `finite_difference_check`: central differences with common random numbers
  (the same Philox keys for +h and -h) against the adjoint, which reports the
  bias from the shadowing and blocking terms the adjoint does not
  differentiate (its receiver-edge term is smoothed over a band).
"""
import ctypes as C
import math

import pyssol as P


class AdjointMap(C.Structure):
    _fields_ = [("receiver", C.c_void_p), ("lower", C.c_double * 2),
                ("upper", C.c_double * 2), ("nx", C.c_uint), ("ny", C.c_uint),
                ("target", C.c_double), ("edge_band", C.c_double)]


class AdjointResult(C.Structure):
    _fields_ = [("absorbed", C.c_double), ("absorbed_se", C.c_double),
                ("spillage", C.c_double), ("hits", C.c_ulonglong),
                ("kernel_ms", C.c_double), ("rays", C.c_ulonglong),
                ("node_visits", C.c_ulonglong), ("triangle_tests", C.c_ulonglong),
                ("quadric_tests", C.c_ulonglong)]


_SIG = [P.VP, P.VP, C.c_size_t, P.PVP, C.c_size_t, C.POINTER(AdjointMap),
        C.POINTER(P.B200Options), C.POINTER(AdjointResult), C.POINTER(C.c_double),
        C.POINTER(C.c_double), C.POINTER(C.c_double)]


def solve_adjoint(scene, heliostats, receiver, lower, upper, nx, ny, target, n,
                  seed=0, options=None, want_map=False, gradients=True):
    """Returns a dict: absorbed, absorbed_se, spillage, hits, kernel_ms,
    d_absorbed and d_spillage (lists of 2 per heliostat: theta_x, theta_y),
    map (nx * ny flux densities, row by row) when want_map."""
    lib = scene.lib
    fn = lib.dll.ssol_solve_adjoint
    fn.argtypes = _SIG
    fn.restype = C.c_int
    helios = list(heliostats) if gradients else []
    nh = len(helios)
    arr = (C.c_void_p * max(1, nh))(*[h.value for h in helios])
    m = AdjointMap()
    m.receiver = receiver.value
    m.lower[0], m.lower[1] = lower
    m.upper[0], m.upper[1] = upper
    m.nx, m.ny = nx, ny
    m.target = target
    res = AdjointResult()
    ga = (C.c_double * max(1, 2 * nh))()
    gs = (C.c_double * max(1, 2 * nh))()
    fmap = (C.c_double * (nx * ny))() if want_map else None
    rng = scene.rng(seed=seed)
    err = fn(scene.scn, rng, int(n), C.cast(arr, P.PVP), nh, C.byref(m),
             C.byref(options) if options is not None else None, C.byref(res),
             ga if nh else None, gs if nh else None, fmap)
    if err != P.RES_OK:
        raise P.SsolError("ssol_solve_adjoint", err)
    out = {"absorbed": res.absorbed, "absorbed_se": res.absorbed_se,
           "spillage": res.spillage, "hits": res.hits, "kernel_ms": res.kernel_ms,
           "counters": {k: getattr(res, k) for k in ("rays", "node_visits",
                                                      "triangle_tests", "quadric_tests")},
           "d_absorbed": list(ga[:2 * nh]), "d_spillage": list(gs[:2 * nh])}
    if want_map:
        out["map"] = list(fmap)
    return out


def _rot(axis, angle):
    """Row-major rotation of `angle` about the unit `axis` (Rodrigues)."""
    x, y, z = axis
    c, s = math.cos(angle), math.sin(angle)
    t = 1 - c
    return ((c + x * x * t, x * y * t - z * s, x * z * t + y * s),
            (y * x * t + z * s, c + y * y * t, y * z * t - x * s),
            (z * x * t - y * s, z * y * t + x * s, c + z * z * t))


def _mul(a, b):
    return tuple(tuple(sum(a[i][k] * b[k][j] for k in range(3)) for j in range(3))
                 for i in range(3))


def _unit(v):
    n = math.sqrt(sum(c * c for c in v))
    return tuple(c / n for c in v)


class AimField:
    """Aim offsets of `heliostats` on a pyssol scene. `transforms` are the
    heliostats' base 3x4 column-major transforms (as given to
    ssol_instance_set_transform); offsets turn each heliostat by
    R = Rot(e_x, theta_x) Rot(e_y, theta_y) about its translation, e_x and
    e_y its base local axes, matching the parameters of ssol_solve_adjoint at
    theta = 0."""

    def __init__(self, scene, heliostats, transforms, receiver, lower, upper, nx, ny,
                 target, n, seed=0, options=None):
        self.scene = scene
        self.helios = list(heliostats)
        self.base = [tuple(t) for t in transforms]
        self.args = (receiver, lower, upper, nx, ny, target, n)
        self.seed = seed
        self.options = options

    def offset_transform(self, i, theta_x, theta_y):
        """The 3x4 column-major transform of heliostat i at offsets (theta_x, theta_y)."""
        t = self.base[i]
        R0 = ((t[0], t[3], t[6]), (t[1], t[4], t[7]), (t[2], t[5], t[8]))
        ex = _unit((t[0], t[1], t[2]))
        ey = _unit((t[3], t[4], t[5]))
        R = _mul(_mul(_rot(ex, theta_x), _rot(ey, theta_y)), R0)
        return P.transform_from(R, (t[9], t[10], t[11]))

    def set_offset(self, i, theta_x, theta_y):
        xf = self.offset_transform(i, theta_x, theta_y)
        self.scene.lib.call("ssol_instance_set_transform", self.helios[i], P._transform(xf))

    def reset(self, i):
        self.scene.lib.call("ssol_instance_set_transform", self.helios[i],
                            P._transform(self.base[i]))

    def apply(self, theta):
        for i, (tx, ty) in enumerate(theta):
            if tx or ty:
                self.set_offset(i, tx, ty)
            else:
                self.reset(i)

    def evaluate(self, gradients=True, want_map=False):
        receiver, lower, upper, nx, ny, target, n = self.args
        return solve_adjoint(self.scene, self.helios, receiver, lower, upper, nx, ny,
                             target, n, seed=self.seed, options=self.options,
                             want_map=want_map, gradients=gradients)


def aim_objective():
    """torch.autograd.Function over theta (n x 2, float64): forward applies
    the offsets and returns [absorbed, spillage]; backward chains the adjoint
    gradients (taken about the applied configuration)."""
    import torch

    class AimObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, field):
            field.apply(theta.detach().cpu().tolist())
            r = field.evaluate(gradients=True)
            ga = torch.tensor(r["d_absorbed"], dtype=torch.float64).view(-1, 2)
            gs = torch.tensor(r["d_spillage"], dtype=torch.float64).view(-1, 2)
            ctx.save_for_backward(ga, gs)
            return torch.tensor([r["absorbed"], r["spillage"]], dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            ga, gs = ctx.saved_tensors
            return grad_out[0] * ga + grad_out[1] * gs, None

    return AimObjective


def finite_difference_check(field, params, h=1e-4):
    """Central differences (common random numbers) of both objectives for the
    (heliostat, axis) pairs in `params`, against the adjoint at theta = 0.
    Returns one dict per parameter with the adjoint and FD values."""
    for i in range(len(field.helios)):
        field.reset(i)
    base = field.evaluate(gradients=True)
    rows = []
    for i, k in params:
        vals = []
        for sgn in (1, -1):
            field.set_offset(i, sgn * h if k == 0 else 0.0, sgn * h if k == 1 else 0.0)
            vals.append(field.evaluate(gradients=False))
            field.reset(i)
        rows.append({
            "heliostat": i, "axis": k,
            "adjoint_absorbed": base["d_absorbed"][2 * i + k],
            "fd_absorbed": (vals[0]["absorbed"] - vals[1]["absorbed"]) / (2 * h),
            "adjoint_spillage": base["d_spillage"][2 * i + k],
            "fd_spillage": (vals[0]["spillage"] - vals[1]["spillage"]) / (2 * h),
        })
    return base, rows
