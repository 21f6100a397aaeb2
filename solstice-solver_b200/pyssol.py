"""ctypes binding of the ssol C API (include/ssol.h, ssp.h, ssol_b200.h).

The same binding drives any library that exports the ssol_* symbols: the
B200 library (libssol_b200.so) or a CPU implementation of the same API. It
mirrors the reference's call sequence (src/ssol.h): create a device, build
shapes / materials / objects / instances, attach them with a sun (and an
atmosphere) to a scene, call ``ssol_solve`` and read the estimator.

``Scene`` is a thin convenience layer used by the tests and the benchmark: it
keeps every ctypes callback alive for as long as the scene lives.
"""
import ctypes as C
import math
import os

RES_OK, RES_BAD_ARG, RES_MEM_ERR, RES_IO_ERR, RES_UNKNOWN_ERR, RES_BAD_OP = 0, 1, 2, 3, 4, 5

SSOL_FRONT, SSOL_BACK = 1, 2
(MAT_DIELECTRIC, MAT_MATTE, MAT_MIRROR, MAT_THIN_DIELECTRIC, MAT_VIRTUAL) = range(5)
BECKMANN, PILLBOX = 0, 1
SSOL_AND, SSOL_SUB = 0, 1
(Q_PLANE, Q_PARABOL, Q_PARABOL2F, Q_HYPERBOL, Q_PCYLINDER, Q_HEMISPHERE) = range(6)
SSOL_POSITION, SSOL_NORMAL, SSOL_TEXCOORD = 0, 1, 2
SSOL_DATA_REAL, SSOL_DATA_SPECTRUM = 0, 1
SSP_RNG_THREEFRY = 4
FP32, FP64 = 0, 1
SIZE_MAX = (1 << 64) - 1

HERE = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB = os.path.join(HERE, "libssol_b200.so")


class SsolError(RuntimeError):
    def __init__(self, func, res):
        super().__init__("%s returned %d" % (func, res))
        self.res = res


# ---------------------------------------------------------------- structures
class McResult(C.Structure):
    _fields_ = [("E", C.c_double), ("V", C.c_double), ("SE", C.c_double)]


class McGlobal(C.Structure):
    _fields_ = [(n, McResult) for n in (
        "cos_factor", "absorbed_by_receivers", "shadowed", "missing",
        "extinguished_by_atmosphere", "other_absorbed")]


RCV_FIELDS = ("incoming_flux", "incoming_if_no_atm_loss", "incoming_if_no_field_loss",
              "incoming_lost_in_field", "incoming_lost_in_atmosphere", "absorbed_flux",
              "absorbed_if_no_atm_loss", "absorbed_if_no_field_loss",
              "absorbed_lost_in_field", "absorbed_lost_in_atmosphere")
GLOBAL_FIELDS = ("cos_factor", "absorbed_by_receivers", "shadowed", "missing",
                 "extinguished_by_atmosphere", "other_absorbed")


class PathTracker(C.Structure):
    """struct ssol_path_tracker (src/ssol.h:359-364); negative => default"""
    _fields_ = [("sun_ray_length", C.c_double), ("infinite_ray_length", C.c_double)]


class PathVertex(C.Structure):
    _fields_ = [("pos", C.c_double * 3), ("weight", C.c_double)]


class SsolPath(C.Structure):
    _fields_ = [("path__", C.c_void_p)]


PATH_TYPES = {0: "missing", 1: "shadow", 2: "success", 3: "error"}


class McReceiver(C.Structure):
    _fields_ = [(n, McResult) for n in RCV_FIELDS] + [
        ("N__", C.c_size_t), ("mc__", C.c_void_p), ("instance__", C.c_void_p)]


class McPrimitive(C.Structure):
    _fields_ = [(n, McResult) for n in RCV_FIELDS]


class McShape(C.Structure):
    _fields_ = [("N__", C.c_size_t), ("mc__", C.c_void_p), ("shape__", C.c_void_p)]


class McSampled(C.Structure):
    _fields_ = [("cos_factor", McResult), ("shadowed", McResult), ("nb_samples", C.c_size_t)]


GET_IDS = C.CFUNCTYPE(None, C.c_uint, C.POINTER(C.c_uint), C.c_void_p)
GET_FLOATS = C.CFUNCTYPE(None, C.c_uint, C.POINTER(C.c_float), C.c_void_p)
GET_WLEN = C.CFUNCTYPE(None, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_double),
                       C.c_void_p)
GET_CARVE = C.CFUNCTYPE(None, C.c_size_t, C.POINTER(C.c_double), C.c_void_p)


class VertexData(C.Structure):
    _fields_ = [("usage", C.c_int), ("get", GET_FLOATS)]


class SurfaceFragment(C.Structure):
    _fields_ = [("dir", C.c_double * 3), ("P", C.c_double * 3), ("Ng", C.c_double * 3),
                ("Ns", C.c_double * 3), ("uv", C.c_double * 2), ("dPdu", C.c_double * 3),
                ("dPdv", C.c_double * 3)]


SHADER = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_double, C.POINTER(SurfaceFragment),
                     C.POINTER(C.c_double))


class MirrorShader(C.Structure):
    _fields_ = [("normal", SHADER), ("reflectivity", SHADER), ("roughness", SHADER)]


class MatteShader(C.Structure):
    _fields_ = [("normal", SHADER), ("reflectivity", SHADER)]


class NormalShader(C.Structure):
    _fields_ = [("normal", SHADER)]


class DataValue(C.Union):
    _fields_ = [("real", C.c_double), ("spectrum", C.c_void_p)]


class Data(C.Structure):
    _fields_ = [("type", C.c_int), ("value", DataValue)]


class Medium(C.Structure):
    _fields_ = [("extinction", Data), ("refractive_index", Data)]


class QuadricData(C.Union):
    _fields_ = [("d", C.c_double * 2)]


class Quadric(C.Structure):
    _fields_ = [("type", C.c_int), ("data", QuadricData), ("transform", C.c_double * 12),
                ("slices_count_hint", C.c_size_t)]


class Carving(C.Structure):
    _fields_ = [("get", GET_CARVE), ("nb_vertices", C.c_size_t), ("operation", C.c_int),
                ("context", C.c_void_p)]


class PunchedSurface(C.Structure):
    _fields_ = [("quadric", C.POINTER(Quadric)), ("carvings", C.POINTER(Carving)),
                ("nb_carvings", C.c_size_t)]


class B200Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("block_size", C.c_int), ("grid_blocks", C.c_int),
                ("waves", C.c_int), ("bvh_leaf_size", C.c_int),
                ("max_segments", C.c_ulonglong), ("min_blocks_per_sm", C.c_int),
                ("bvh_builder", C.c_int), ("count_work", C.c_int)]


BVH_AUTO, BVH_SAH, BVH_LBVH = 0, 1, 2


class SunPosition(C.Structure):
    _fields_ = [("direction", C.c_double * 3), ("dni", C.c_double)]


class B200Stats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double)] + [(n, C.c_ulonglong) for n in (
        "rays", "node_visits", "triangle_tests", "quadric_tests", "bounces", "paths",
        "killed", "scene_bytes", "tally_bytes", "bvh_nodes", "bvh_depth", "bvh_device")]


class ImageLayout(C.Structure):
    _fields_ = [("row_pitch", C.c_size_t), ("offset", C.c_size_t), ("size", C.c_size_t),
                ("width", C.c_size_t), ("height", C.c_size_t), ("pixel_format", C.c_int)]


PIXEL_DOUBLE3 = 0
FILTER_LINEAR, FILTER_NEAREST = 0, 1
ADDRESS_CLAMP, ADDRESS_REPEAT = 0, 1
WRITE_PIXELS = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_size_t),
                           C.POINTER(C.c_size_t), C.c_int, C.c_void_p)

VP = C.c_void_p
PVP = C.POINTER(C.c_void_p)
_SIGS = {
    "ssol_device_create": [VP, VP, C.c_uint, C.c_int, PVP],
    "ssol_device_ref_put": [VP],
    "ssol_scene_create": [VP, PVP], "ssol_scene_ref_put": [VP],
    "ssol_scene_attach_instance": [VP, VP], "ssol_scene_detach_instance": [VP, VP],
    "ssol_scene_attach_sun": [VP, VP], "ssol_scene_detach_sun": [VP, VP],
    "ssol_scene_attach_atmosphere": [VP, VP], "ssol_scene_detach_atmosphere": [VP, VP],
    "ssol_scene_clear": [VP],
    "ssol_shape_create_mesh": [VP, PVP], "ssol_shape_create_punched_surface": [VP, PVP],
    "ssol_shape_ref_put": [VP],
    "ssol_mesh_setup": [VP, C.c_uint, GET_IDS, C.c_uint, C.POINTER(VertexData), C.c_uint, VP],
    "ssol_punched_surface_setup": [VP, C.POINTER(PunchedSurface)],
    "ssol_shape_get_triangles_count": [VP, C.POINTER(C.c_uint)],
    "ssol_shape_get_vertices_count": [VP, C.POINTER(C.c_uint)],
    "ssol_shape_get_triangle_indices": [VP, C.c_uint, C.c_uint * 3],
    "ssol_shape_get_vertex_attrib": [VP, C.c_uint, C.c_int, C.c_double * 3],
    "ssol_material_create_mirror": [VP, PVP], "ssol_material_create_matte": [VP, PVP],
    "ssol_material_create_virtual": [VP, PVP], "ssol_material_create_dielectric": [VP, PVP],
    "ssol_material_create_thin_dielectric": [VP, PVP], "ssol_material_ref_put": [VP],
    "ssol_mirror_setup": [VP, C.POINTER(MirrorShader), C.c_int],
    "ssol_matte_setup": [VP, C.POINTER(MatteShader)],
    "ssol_dielectric_setup": [VP, C.POINTER(NormalShader), C.POINTER(Medium), C.POINTER(Medium)],
    "ssol_thin_dielectric_setup": [VP, C.POINTER(NormalShader), C.POINTER(Medium),
                                   C.POINTER(Medium), C.c_double],
    "ssol_object_create": [VP, PVP], "ssol_object_ref_put": [VP],
    "ssol_object_add_shaded_shape": [VP, VP, VP, VP],
    "ssol_object_get_area": [VP, C.POINTER(C.c_double)],
    "ssol_object_instantiate": [VP, PVP], "ssol_instance_ref_put": [VP],
    "ssol_instance_set_transform": [VP, C.c_double * 12],
    "ssol_instance_set_receiver": [VP, C.c_int, C.c_int],
    "ssol_instance_sample": [VP, C.c_int],
    "ssol_instance_get_area": [VP, C.POINTER(C.c_double)],
    "ssol_spectrum_create": [VP, PVP], "ssol_spectrum_ref_put": [VP],
    "ssol_spectrum_setup": [VP, GET_WLEN, C.c_size_t, VP],
    "ssol_sun_create_directional": [VP, PVP], "ssol_sun_create_pillbox": [VP, PVP],
    "ssol_sun_create_gaussian": [VP, PVP], "ssol_sun_create_buie": [VP, PVP],
    "ssol_sun_ref_put": [VP],
    "ssol_sun_set_direction": [VP, C.c_double * 3], "ssol_sun_set_dni": [VP, C.c_double],
    "ssol_sun_set_spectrum": [VP, VP],
    "ssol_sun_pillbox_set_half_angle": [VP, C.c_double],
    "ssol_sun_gaussian_set_std_dev": [VP, C.c_double],
    "ssol_sun_set_buie_param": [VP, C.c_double],
    "ssol_atmosphere_create": [VP, PVP], "ssol_atmosphere_ref_put": [VP],
    "ssol_atmosphere_set_extinction": [VP, C.POINTER(Data)],
    "ssol_solve": [VP, VP, C.c_size_t, C.c_size_t, VP, PVP],
    "ssol_estimator_get_tracked_paths_count": [VP, C.POINTER(C.c_size_t)],
    "ssol_estimator_get_tracked_path": [VP, C.c_size_t, C.POINTER(SsolPath)],
    "ssol_path_get_vertices_count": [C.POINTER(SsolPath), C.POINTER(C.c_size_t)],
    "ssol_path_get_vertex": [C.POINTER(SsolPath), C.c_size_t, C.POINTER(PathVertex)],
    "ssol_path_get_type": [C.POINTER(SsolPath), C.POINTER(C.c_int)],
    "ssol_estimator_ref_put": [VP],
    "ssol_estimator_get_mc_global": [VP, C.POINTER(McGlobal)],
    "ssol_estimator_get_mc_receiver": [VP, VP, C.c_int, C.POINTER(McReceiver)],
    "ssol_estimator_get_mc_sampled_x_receiver": [VP, VP, VP, C.c_int, C.POINTER(McReceiver)],
    "ssol_estimator_get_mc_sampled": [VP, VP, C.POINTER(McSampled)],
    "ssol_estimator_get_realisation_count": [VP, C.POINTER(C.c_size_t)],
    "ssol_estimator_get_failed_count": [VP, C.POINTER(C.c_size_t)],
    "ssol_estimator_get_sampled_area": [VP, C.POINTER(C.c_double)],
    "ssol_estimator_get_sampled_count": [VP, C.POINTER(C.c_size_t)],
    "ssol_estimator_get_rng_state": [VP, PVP],
    "ssol_mc_receiver_get_mc_shape": [C.POINTER(McReceiver), VP, C.POINTER(McShape)],
    "ssol_mc_shape_get_mc_primitive": [C.POINTER(McShape), C.c_uint, C.POINTER(McPrimitive)],
    "ssol_camera_create": [VP, PVP], "ssol_camera_ref_get": [VP],
    "ssol_camera_ref_put": [VP],
    "ssol_camera_set_proj_ratio": [VP, C.c_double], "ssol_camera_set_fov": [VP, C.c_double],
    "ssol_camera_look_at": [VP, C.POINTER(C.c_double), C.POINTER(C.c_double),
                            C.POINTER(C.c_double)],
    "ssol_image_create": [VP, PVP], "ssol_image_ref_get": [VP], "ssol_image_ref_put": [VP],
    "ssol_image_setup": [VP, C.c_size_t, C.c_size_t, C.c_int],
    "ssol_image_get_layout": [VP, C.POINTER(ImageLayout)],
    "ssol_image_map": [VP, C.POINTER(C.c_void_p)], "ssol_image_unmap": [VP],
    "ssol_image_sample": [VP, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), VP],
    "ssol_image_write": [VP, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.c_int, VP],
    "ssol_draw_draft": [VP, VP, C.c_size_t, C.c_size_t, C.c_size_t, WRITE_PIXELS, VP],
    "ssol_draw_pt": [VP, VP, C.c_size_t, C.c_size_t, C.c_size_t, C.POINTER(C.c_double),
                     WRITE_PIXELS, VP],
    "ssp_rng_create": [VP, C.c_int, PVP], "ssp_rng_ref_put": [VP],
    "ssp_rng_set": [VP, C.c_uint64], "ssp_rng_discard": [VP, C.c_uint64],
}
_OPTIONAL = {
    "ssol_solve_ex": [VP, VP, C.c_size_t, C.c_size_t, VP, C.POINTER(B200Options), PVP],
    "ssol_estimator_get_b200_stats": [VP, C.POINTER(B200Stats)],
    "ssol_b200_plan_create": [VP, C.POINTER(B200Options), PVP],
    "ssol_b200_plan_ref_put": [VP],
    "ssol_b200_plan_reset": [VP, VP],
    "ssol_b200_plan_abort": [VP],
    "ssol_b200_plan_get_tallies": [VP, PVP, C.POINTER(C.c_size_t), PVP,
                                   C.POINTER(C.c_size_t)],
    "ssol_b200_tallies_size": [VP, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)],
    "ssol_b200_estimator_create_from_tallies": [VP, VP, C.c_uint64, C.c_size_t,
                                                C.POINTER(C.c_double), C.c_size_t,
                                                C.POINTER(C.c_uint64), C.c_size_t, PVP],
    "ssol_b200_plan_launch": [VP, VP, C.c_uint64, C.c_uint64, VP],
    "ssol_b200_plan_finish": [VP, VP, C.c_uint64, C.c_size_t, VP, PVP],
    "ssol_b200_batch_create": [PVP, C.c_size_t, C.POINTER(B200Options), PVP],
    "ssol_b200_batch_ref_put": [VP],
    "ssol_b200_batch_reset": [VP, VP],
    "ssol_b200_batch_launch": [VP, VP, C.POINTER(C.c_uint64), VP],
    "ssol_b200_batch_finish": [VP, VP, C.c_size_t, VP, PVP],
    "ssol_b200_batch_launch_noalloc": [VP, VP, C.POINTER(C.c_uint64), VP],
    "ssol_b200_batch_get_mc_global": [VP, VP, C.POINTER(McGlobal)],
    "ssol_b200_batch_create_tracking": [VP, PVP, C.c_size_t, C.POINTER(C.c_double),
                                        C.POINTER(SunPosition), C.c_size_t,
                                        C.POINTER(B200Options), PVP],
    "ssol_b200_autotune": [VP, VP, C.c_uint64, C.POINTER(B200Options),
                           C.POINTER(C.c_double)],
    "ssol_b200_draw_draft_device": [VP, VP, C.c_size_t, C.c_size_t, C.c_size_t,
                                    C.POINTER(B200Options), VP, C.POINTER(B200Stats)],
    "ssol_b200_draw_pt_device": [VP, VP, C.c_size_t, C.c_size_t, C.c_size_t,
                                 C.POINTER(C.c_double), C.c_uint64, C.POINTER(B200Options),
                                 VP, C.POINTER(B200Stats)],
}


class Lib:
    """One loaded implementation of the ssol C API."""

    def __init__(self, path):
        self.path = path
        self.dll = C.CDLL(path, mode=getattr(os, "RTLD_LOCAL", 0) | os.RTLD_NOW)
        for name, args in _SIGS.items():
            f = getattr(self.dll, name)
            f.argtypes = args
            f.restype = C.c_int
        self.has_b200 = hasattr(self.dll, "ssol_b200_plan_create")
        if self.has_b200:
            for name, args in _OPTIONAL.items():
                f = getattr(self.dll, name, None)
                if f is None:  # an older build of the library
                    continue
                f.argtypes = args
                f.restype = C.c_int
        self.dll.ssol_param_buffer_create.argtypes = [VP, C.c_size_t, PVP]
        self.dll.ssol_param_buffer_create.restype = C.c_int
        self.dll.ssol_param_buffer_ref_put.argtypes = [VP]
        self.dll.ssol_param_buffer_ref_put.restype = C.c_int
        self.dll.ssol_param_buffer_allocate.argtypes = [VP, C.c_size_t, C.c_size_t, VP]
        self.dll.ssol_param_buffer_allocate.restype = VP
        self.dll.ssol_material_set_param_buffer.argtypes = [VP, VP]
        self.dll.ssol_material_set_param_buffer.restype = C.c_int
        # native shaders for constant properties (B200 library only)
        self.native_shaders = hasattr(self.dll, "ssol_b200_shader_param0")
        self.dll.ssp_rng_get.argtypes = [VP]
        self.dll.ssp_rng_get.restype = C.c_uint64
        self.dll.ssp_rng_canonical.argtypes = [VP]
        self.dll.ssp_rng_canonical.restype = C.c_double

    def call(self, name, *args):
        res = getattr(self.dll, name)(*args)
        if res != RES_OK:
            raise SsolError(name, res)
        return res

    def raw(self, name, *args):
        return getattr(self.dll, name)(*args)


# ------------------------------------------------------------- result helpers
def mc(r):
    return (r.E, r.V, r.SE)


class Estimator:
    def __init__(self, scene, handle, res):
        self.scene = scene
        self.lib = scene.lib
        self.h = handle
        self.res = res

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.raw("ssol_estimator_ref_put", self.h)
            self.h = None

    def globals(self):
        g = McGlobal()
        self.lib.call("ssol_estimator_get_mc_global", self.h, C.byref(g))
        return {n: mc(getattr(g, n)) for n in GLOBAL_FIELDS}

    def receiver(self, inst, side=SSOL_FRONT):
        r = McReceiver()
        self.lib.call("ssol_estimator_get_mc_receiver", self.h, inst, side, C.byref(r))
        return {n: mc(getattr(r, n)) for n in RCV_FIELDS}

    def receiver_raw(self, inst, side=SSOL_FRONT):
        r = McReceiver()
        self.lib.call("ssol_estimator_get_mc_receiver", self.h, inst, side, C.byref(r))
        return r

    def sampled_x_receiver(self, samp, inst, side=SSOL_FRONT):
        r = McReceiver()
        self.lib.call("ssol_estimator_get_mc_sampled_x_receiver", self.h, samp, inst, side,
                      C.byref(r))
        return {n: mc(getattr(r, n)) for n in RCV_FIELDS}

    def sampled(self, inst):
        s = McSampled()
        self.lib.call("ssol_estimator_get_mc_sampled", self.h, inst, C.byref(s))
        return {"cos_factor": mc(s.cos_factor), "shadowed": mc(s.shadowed),
                "nb_samples": s.nb_samples}

    def primitives(self, inst, shape, side=SSOL_FRONT):
        """Per-primitive results (per unit area) of `shape` in receiver `inst`."""
        r = self.receiver_raw(inst, side)
        ms = McShape()
        self.lib.call("ssol_mc_receiver_get_mc_shape", C.byref(r), shape, C.byref(ms))
        n = C.c_uint()
        self.lib.call("ssol_shape_get_triangles_count", shape, C.byref(n))
        out = []
        for i in range(n.value):
            p = McPrimitive()
            self.lib.call("ssol_mc_shape_get_mc_primitive", C.byref(ms), i, C.byref(p))
            out.append({k: mc(getattr(p, k)) for k in RCV_FIELDS})
        return out

    def paths(self):
        """Tracked paths: [(type, [((x, y, z), weight), ...]), ...]"""
        n = C.c_size_t()
        self.lib.call("ssol_estimator_get_tracked_paths_count", self.h, C.byref(n))
        out = []
        for i in range(n.value):
            p = SsolPath()
            self.lib.call("ssol_estimator_get_tracked_path", self.h, i, C.byref(p))
            nv, t = C.c_size_t(), C.c_int()
            self.lib.call("ssol_path_get_vertices_count", C.byref(p), C.byref(nv))
            self.lib.call("ssol_path_get_type", C.byref(p), C.byref(t))
            verts = []
            for k in range(nv.value):
                v = PathVertex()
                self.lib.call("ssol_path_get_vertex", C.byref(p), k, C.byref(v))
                verts.append((tuple(v.pos), v.weight))
            out.append((PATH_TYPES.get(t.value, t.value), verts))
        return out

    def count(self, what):
        v = C.c_size_t()
        self.lib.call("ssol_estimator_get_%s" % what, self.h, C.byref(v))
        return v.value

    def sampled_area(self):
        v = C.c_double()
        self.lib.call("ssol_estimator_get_sampled_area", self.h, C.byref(v))
        return v.value

    def stats(self):
        s = B200Stats()
        self.lib.call("ssol_estimator_get_b200_stats", self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in B200Stats._fields_}


def _transform(t):
    a = (C.c_double * 12)()
    for i, v in enumerate(t):
        a[i] = v
    return a


IDENTITY = (1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0)


def transform_from(R=None, T=(0, 0, 0)):
    """3x4 column-major transform from a row-major 3x3 rotation R and T."""
    if R is None:
        R = ((1, 0, 0), (0, 1, 0), (0, 0, 1))
    return (R[0][0], R[1][0], R[2][0], R[0][1], R[1][1], R[2][1],
            R[0][2], R[1][2], R[2][2], T[0], T[1], T[2])


def rotation_pitch_pi():
    """180 degree rotation about y: flips the faces of a z = 0 plane."""
    return ((-1, 0, 0), (0, 1, 0), (0, 0, -1))


class Scene:
    """A device + scene on one library, with helpers to describe content."""

    def __init__(self, lib, nthreads=0xffffffff):
        self.lib = lib
        self._keep = []
        self._handles = []
        self.dev = C.c_void_p()
        lib.call("ssol_device_create", None, None, nthreads, 0, C.byref(self.dev))
        self.scn = C.c_void_p()
        lib.call("ssol_scene_create", self.dev, C.byref(self.scn))
        self.sun = None

    def close(self):
        lib = self.lib
        if self.scn:
            lib.raw("ssol_scene_ref_put", self.scn)
            self.scn = None
        for put, h in reversed(self._handles):
            lib.raw(put, h)
        self._handles = []
        if self.dev:
            lib.raw("ssol_device_ref_put", self.dev)
            self.dev = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _new(self, create, put, *args):
        h = C.c_void_p()
        self.lib.call(create, *args, C.byref(h))
        self._handles.append((put, h))
        return h

    # ---- spectra and data
    def spectrum(self, wavelengths, values):
        h = self._new("ssol_spectrum_create", "ssol_spectrum_ref_put", self.dev)
        wl = list(wavelengths)
        va = list(values)

        def get(i, w, d, ctx):
            w[0] = wl[i]
            d[0] = va[i]
        cb = GET_WLEN(get)
        self._keep.append(cb)
        self.lib.call("ssol_spectrum_setup", h, cb, len(wl), None)
        return h

    def data(self, value):
        d = Data()
        if isinstance(value, C.c_void_p):
            d.type = SSOL_DATA_SPECTRUM
            d.value.spectrum = value
        else:
            d.type = SSOL_DATA_REAL
            d.value.real = float(value)
        return d

    def medium(self, extinction=0.0, refractive_index=1.0):
        m = Medium()
        m.extinction = self.data(extinction)
        m.refractive_index = self.data(refractive_index)
        return m

    # ---- shapes
    def mesh(self, vertices, indices, normals=None, texcoords=None):
        """Mesh with optional per-vertex normals and texcoords."""
        h = self._new("ssol_shape_create_mesh", "ssol_shape_ref_put", self.dev)
        verts = [tuple(map(float, v)) for v in vertices]
        ids = [tuple(map(int, t)) for t in indices]

        def get_ids(i, out, ctx):
            t = ids[i]
            out[0], out[1], out[2] = t

        def floats(values, n):
            vals = [tuple(map(float, v)) for v in values]

            def get(i, out, ctx):
                for k in range(n):
                    out[k] = vals[i][k]
            return GET_FLOATS(get)
        cb_ids = GET_IDS(get_ids)
        cbs = [(SSOL_POSITION, floats(verts, 3))]
        if normals is not None:
            cbs.append((SSOL_NORMAL, floats(normals, 3)))
        if texcoords is not None:
            cbs.append((SSOL_TEXCOORD, floats(texcoords, 2)))
        self._keep += [cb_ids] + [c for _, c in cbs]
        attr = (VertexData * len(cbs))()
        for k, (usage, cb) in enumerate(cbs):
            attr[k].usage = usage
            attr[k].get = cb
        self.lib.call("ssol_mesh_setup", h, len(ids), cb_ids, len(verts), attr, len(cbs),
                      None)
        return h

    def rectangle(self, hx, hy):
        """The reference tests' rectangle: 4 vertices, triangles {0,2,1, 2,0,3}
        (src/test_ssol_rect_geometry.h:54-66); front face +z."""
        v = [(-hx, -hy, 0), (hx, -hy, 0), (hx, hy, 0), (-hx, hy, 0)]
        return self.mesh(v, [(0, 2, 1), (2, 0, 3)])

    def punched(self, qtype, params=(), carvings=(), transform=IDENTITY, slices=None):
        """Punched quadric; carvings = [(op, [(x, y), ...]), ...]."""
        h = self._new("ssol_shape_create_punched_surface", "ssol_shape_ref_put", self.dev)
        q = Quadric()
        q.type = qtype
        for i, p in enumerate(params):
            q.data.d[i] = p
        for i, v in enumerate(transform):
            q.transform[i] = v
        q.slices_count_hint = SIZE_MAX if slices is None else slices
        carr = (Carving * max(1, len(carvings)))()
        for k, (op, poly) in enumerate(carvings):
            pts = [tuple(map(float, p)) for p in poly]

            def get(i, out, ctx, pts=pts):
                out[0], out[1] = pts[i]
            cb = GET_CARVE(get)
            self._keep.append(cb)
            carr[k].get = cb
            carr[k].nb_vertices = len(pts)
            carr[k].operation = op
            carr[k].context = None
        ps = PunchedSurface()
        ps.quadric = C.pointer(q)
        ps.carvings = carr
        ps.nb_carvings = len(carvings)
        self._keep += [q, carr, ps]
        self.lib.call("ssol_punched_surface_setup", h, C.byref(ps))
        return h

    def triangles_count(self, shape):
        n = C.c_uint()
        self.lib.call("ssol_shape_get_triangles_count", shape, C.byref(n))
        return n.value

    # ---- materials
    def _const(self, value):
        """Shader callback: a constant, or a Python function f(wl, frag)
        of the wavelength and the surface fragment (P, Ng, Ns, uv, ...)"""
        if callable(value):
            fn = value

            def f(dev, buf, wl, frag, out):
                out[0] = float(fn(wl, frag[0]))
        else:
            def f(dev, buf, wl, frag, out):
                out[0] = value
        cb = SHADER(f)
        self._keep.append(cb)
        return cb

    def _normal(self):
        def f(dev, buf, wl, frag, out):
            out[0], out[1], out[2] = frag[0].Ns[0], frag[0].Ns[1], frag[0].Ns[2]
        cb = SHADER(f)
        self._keep.append(cb)
        return cb

    def _native(self, material, values):
        """Native shaders reading `values` from the material's parameter
        buffer (ssol_b200_shader_param0/1, ssol_b200_shader_Ns), or None when
        the library has none or a value is a Python function. Python
        callbacks would take the interpreter's lock on every call when the
        library snapshots scenes from its worker threads."""
        if not self.lib.native_shaders or any(callable(v) for v in values):
            return None
        buf = self._new("ssol_param_buffer_create", "ssol_param_buffer_ref_put", self.dev,
                        8 * len(values))
        mem = self.lib.dll.ssol_param_buffer_allocate(buf, 8 * len(values), 8, None)
        arr = C.cast(mem, C.POINTER(C.c_double))
        for i, v in enumerate(values):
            arr[i] = float(v)
        self.lib.call("ssol_material_set_param_buffer", material, buf)
        dll = self.lib.dll
        return ([SHADER(("ssol_b200_shader_param%d" % i, dll)) for i in range(len(values))],
                SHADER(("ssol_b200_shader_Ns", dll)))

    def mirror(self, reflectivity=1.0, roughness=0.0, distrib=BECKMANN):
        h = self._new("ssol_material_create_mirror", "ssol_material_ref_put", self.dev)
        nat = self._native(h, (reflectivity, roughness))
        if nat is not None:
            (r, g), n = nat
            s = MirrorShader(n, r, g)
            self._keep += [n, r, g]
        else:
            s = MirrorShader(self._normal(), self._const(reflectivity), self._const(roughness))
        self.lib.call("ssol_mirror_setup", h, C.byref(s), distrib)
        return h

    def matte(self, reflectivity=0.0):
        h = self._new("ssol_material_create_matte", "ssol_material_ref_put", self.dev)
        nat = self._native(h, (reflectivity,))
        if nat is not None:
            (r,), n = nat
            s = MatteShader(n, r)
            self._keep += [n, r]
        else:
            s = MatteShader(self._normal(), self._const(reflectivity))
        self.lib.call("ssol_matte_setup", h, C.byref(s))
        return h

    def virtual(self):
        return self._new("ssol_material_create_virtual", "ssol_material_ref_put", self.dev)

    def dielectric(self, outside, inside):
        h = self._new("ssol_material_create_dielectric", "ssol_material_ref_put", self.dev)
        s = NormalShader(self._normal())
        self.lib.call("ssol_dielectric_setup", h, C.byref(s), C.byref(outside),
                      C.byref(inside))
        return h

    def thin_dielectric(self, outside, slab, thickness):
        h = self._new("ssol_material_create_thin_dielectric", "ssol_material_ref_put",
                      self.dev)
        s = NormalShader(self._normal())
        self.lib.call("ssol_thin_dielectric_setup", h, C.byref(s), C.byref(outside),
                      C.byref(slab), float(thickness))
        return h

    # ---- objects, instances
    def object(self, shaded):
        """shaded: list of (shape, front, back)."""
        h = self._new("ssol_object_create", "ssol_object_ref_put", self.dev)
        for shape, front, back in shaded:
            self.lib.call("ssol_object_add_shaded_shape", h, shape, front, back)
        return h

    def instance(self, obj, transform=IDENTITY, receiver=0, per_primitive=0, sample=1,
                 attach=True):
        h = self._new("ssol_object_instantiate", "ssol_instance_ref_put", obj)
        self.lib.call("ssol_instance_set_transform", h, _transform(transform))
        self.lib.call("ssol_instance_set_receiver", h, receiver, per_primitive)
        self.lib.call("ssol_instance_sample", h, sample)
        if attach:
            self.lib.call("ssol_scene_attach_instance", self.scn, h)
        return h

    # ---- sun, atmosphere
    def set_sun(self, kind="directional", direction=(0, 0, -1), dni=1000.0,
                param=None, spectrum=None):
        create = {"directional": "ssol_sun_create_directional",
                  "pillbox": "ssol_sun_create_pillbox",
                  "gaussian": "ssol_sun_create_gaussian",
                  "buie": "ssol_sun_create_buie"}[kind]
        h = self._new(create, "ssol_sun_ref_put", self.dev)
        d = (C.c_double * 3)(*direction)
        self.lib.call("ssol_sun_set_direction", h, d)
        self.lib.call("ssol_sun_set_dni", h, float(dni))
        if kind == "pillbox":
            self.lib.call("ssol_sun_pillbox_set_half_angle", h, float(param))
        elif kind == "gaussian":
            self.lib.call("ssol_sun_gaussian_set_std_dev", h, float(param))
        elif kind == "buie":
            self.lib.call("ssol_sun_set_buie_param", h, float(param))
        if spectrum is None:
            spectrum = self.spectrum([1, 2, 3], [1, 0.8, 1])
        self.lib.call("ssol_sun_set_spectrum", h, spectrum)
        if self.sun is not None:
            self.lib.call("ssol_scene_detach_sun", self.scn, self.sun)
        self.lib.call("ssol_scene_attach_sun", self.scn, h)
        self.sun = h
        return h

    def atmosphere(self, extinction):
        h = self._new("ssol_atmosphere_create", "ssol_atmosphere_ref_put", self.dev)
        d = self.data(extinction)
        self.lib.call("ssol_atmosphere_set_extinction", h, C.byref(d))
        self.lib.call("ssol_scene_attach_atmosphere", self.scn, h)
        return h

    # ---- camera and renderers
    def camera(self, position=(0, 0, 0), target=(0, 0, -1), up=(0, 1, 0), fov=None,
               ratio=None):
        """A pinhole camera (ssol_camera_*): fov is the horizontal field of
        view in radians, ratio width / height; both set before look_at, as
        the reference's draw test does."""
        h = self._new("ssol_camera_create", "ssol_camera_ref_put", self.dev)
        if ratio is not None:
            self.lib.call("ssol_camera_set_proj_ratio", h, float(ratio))
        if fov is not None:
            self.lib.call("ssol_camera_set_fov", h, float(fov))
        d3 = C.c_double * 3
        self.lib.call("ssol_camera_look_at", h, d3(*position), d3(*target), d3(*up))
        return h

    def draw(self, kind, cam, width, height, spp, up=(0, 0, 1), tiles=None, check=True):
        """ssol_draw_draft (kind "draft") or ssol_draw_pt (kind "pt") through a
        writer that fills a (height, width, 3) float64 array; `tiles`, when a
        list, receives (x, y, w, h) per writer call. Returns (res, image)."""
        import numpy as np
        img = np.zeros((height, width, 3))

        def write(ctx, org, sz, fmt, pixels):
            ox, oy, sx, sy = org[0], org[1], sz[0], sz[1]
            if fmt != PIXEL_DOUBLE3 or ox + sx > width or oy + sy > height:
                return RES_BAD_ARG
            buf = np.ctypeslib.as_array(C.cast(pixels, C.POINTER(C.c_double)),
                                        shape=(sy, sx, 3))
            img[oy:oy + sy, ox:ox + sx] = buf
            if tiles is not None:
                tiles.append((ox, oy, sx, sy))
            return RES_OK

        cb = WRITE_PIXELS(write)
        if kind == "draft":
            res = self.lib.raw("ssol_draw_draft", self.scn, cam, width, height, spp, cb, None)
        else:
            res = self.lib.raw("ssol_draw_pt", self.scn, cam, width, height, spp,
                               (C.c_double * 3)(*up), cb, None)
        if check and res != RES_OK:
            raise SsolError("ssol_draw_" + kind, res)
        return res, img

    def draw_device(self, kind, cam, width, height, spp, device_pixels, up=(0, 0, 1),
                    seed=0, options=None):
        """ssol_b200_draw_*_device into `device_pixels` (a device address of
        width x height x 3 doubles). Returns the B200Stats."""
        st = B200Stats()
        opt = C.byref(options) if options is not None else None
        if kind == "draft":
            self.lib.call("ssol_b200_draw_draft_device", self.scn, cam, width, height, spp,
                          opt, C.c_void_p(device_pixels), C.byref(st))
        else:
            self.lib.call("ssol_b200_draw_pt_device", self.scn, cam, width, height, spp,
                          (C.c_double * 3)(*up), seed, opt, C.c_void_p(device_pixels),
                          C.byref(st))
        return st

    # ---- solve
    def rng(self, seed=0, position=0):
        h = self._new("ssp_rng_create", "ssp_rng_ref_put", None, SSP_RNG_THREEFRY)
        self.lib.call("ssp_rng_set", h, seed)
        if position:
            self.lib.call("ssp_rng_discard", h, position)
        return h

    def solve(self, n, seed=0, max_failed=0, rng=None, options=None, check=True,
              tracker=None):
        """tracker: None, or (sun_ray_length, infinite_ray_length)"""
        if rng is None:
            rng = self.rng(seed)
        est = C.c_void_p()
        tr = None
        if tracker is not None:
            tr = PathTracker(float(tracker[0]), float(tracker[1]))
            tr = C.byref(tr)
        if options is not None:
            res = self.lib.raw("ssol_solve_ex", self.scn, rng, n, max_failed, tr,
                               C.byref(options), C.byref(est))
        else:
            res = self.lib.raw("ssol_solve", self.scn, rng, n, max_failed, tr,
                               C.byref(est))
        if check and res not in (RES_OK,):
            if est:
                self.lib.raw("ssol_estimator_ref_put", est)
            raise SsolError("ssol_solve", res)
        return Estimator(self, est, res) if est else None


class Batch:
    """Several scenes traced by one persistent launch (ssol_b200_batch_*)."""

    def __init__(self, lib, scenes, opts=None):
        self.lib = lib
        self.scenes = list(scenes)
        arr = (C.c_void_p * len(scenes))(*[s.scn.value for s in scenes])
        self.h = C.c_void_p()
        lib.call("ssol_b200_batch_create", C.cast(arr, PVP), len(scenes),
                 C.byref(opts) if opts is not None else None, C.byref(self.h))

    @classmethod
    def tracking(cls, scene, heliostats, aims, suns, opts=None):
        """One item per sun of `scene` with `heliostats` (instance handles)
        turned toward it and aimed at `aims` (one (x, y, z) each)
        (ssol_b200_batch_create_tracking); suns: [(direction, dni), ...]."""
        self = cls.__new__(cls)
        self.lib = scene.lib
        self.scenes = [scene] * len(suns)
        hel = (C.c_void_p * max(1, len(heliostats)))(*[x.value for x in heliostats])
        flat = [float(c) for a in aims for c in a]
        aa = (C.c_double * max(1, len(flat)))(*flat)
        sp = (SunPosition * len(suns))()
        for i, (d, dni) in enumerate(suns):
            sp[i].direction[:] = [float(c) for c in d]
            sp[i].dni = float(dni)
        self.h = C.c_void_p()
        self.lib.call("ssol_b200_batch_create_tracking", scene.scn, C.cast(hel, PVP),
                      len(heliostats), aa, sp, len(suns),
                      C.byref(opts) if opts is not None else None, C.byref(self.h))
        return self

    def reset(self, stream=None):
        self.lib.call("ssol_b200_batch_reset", self.h, stream)

    def launch(self, rng, budgets, stream=None):
        b = (C.c_uint64 * len(budgets))(*[int(x) for x in budgets])
        self.lib.call("ssol_b200_batch_launch", self.h, rng, b, stream)

    def launch_noalloc(self, rng, budgets, stream=None):
        b = (C.c_uint64 * len(budgets))(*[int(x) for x in budgets])
        self.lib.call("ssol_b200_batch_launch_noalloc", self.h, rng, b, stream)

    def globals(self, stream=None):
        """Per item, the global estimates (ssol_b200_batch_get_mc_global)."""
        n = len(self.scenes)
        arr = (McGlobal * n)()
        self.lib.call("ssol_b200_batch_get_mc_global", self.h, stream, arr)
        return [{k: mc(getattr(g, k)) for k in GLOBAL_FIELDS} for g in arr]

    def finish(self, rng, max_failed=0, stream=None):
        n = len(self.scenes)
        arr = (C.c_void_p * n)()
        res = self.lib.raw("ssol_b200_batch_finish", self.h, rng, max_failed, stream,
                           C.cast(arr, PVP))
        if res not in (RES_OK, RES_BAD_OP):
            raise SsolError("ssol_b200_batch_finish", res)
        return [Estimator(s, C.c_void_p(arr[i]), res) for i, s in enumerate(self.scenes)]

    def close(self):
        if self.h:
            self.lib.raw("ssol_b200_batch_ref_put", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceArray:
    """A device buffer of the library seen through __cuda_array_interface__,
    so that torch.as_tensor(DeviceArray(...), device="cuda") shares it."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3}


def plan_tallies(lib, plan):
    """(sums, counts) of a plan (ssol_b200_plan_get_tallies) as DeviceArray
    views: FP64 sums and 64-bit counts (viewed as int64, which adds alike)."""
    sp, cp = C.c_void_p(), C.c_void_p()
    ns, nc = C.c_size_t(), C.c_size_t()
    lib.call("ssol_b200_plan_get_tallies", plan, C.byref(sp), C.byref(ns), C.byref(cp),
             C.byref(nc))
    return DeviceArray(sp.value, ns.value, "<f8"), DeviceArray(cp.value, nc.value, "<i8")


def tallies_size(scene):
    ns, nc = C.c_size_t(), C.c_size_t()
    scene.lib.call("ssol_b200_tallies_size", scene.scn, C.byref(ns), C.byref(nc))
    return ns.value, nc.value


def estimator_from_tallies(scene, rng, n, sums, counts, max_failed=0):
    """Estimator of `n` realisations of `scene` from host tallies (sequences
    of floats and of non-negative ints)."""
    sa = (C.c_double * len(sums))(*[float(x) for x in sums])
    ca = (C.c_uint64 * len(counts))(*[int(x) & 0xffffffffffffffff for x in counts])
    est = C.c_void_p()
    res = scene.lib.raw("ssol_b200_estimator_create_from_tallies", scene.scn, rng, int(n),
                        max_failed, sa, len(sums), ca, len(counts), C.byref(est))
    if res not in (RES_OK, RES_BAD_OP):
        raise SsolError("ssol_b200_estimator_create_from_tallies", res)
    return Estimator(scene, est, res)


def options(precision=FP32, block_size=256, grid_blocks=0, waves=1, leaf=0,
            max_segments=0, min_blocks=0, bvh=BVH_AUTO, count=0):
    o = B200Options()
    o.precision = precision
    o.block_size = block_size
    o.grid_blocks = grid_blocks
    o.waves = waves
    o.bvh_leaf_size = leaf
    o.max_segments = max_segments
    o.min_blocks_per_sm = min_blocks
    o.bvh_builder = bvh
    o.count_work = count
    return o


def autotune(scene, trial_paths=4_000_000, opts=None, seed=0):
    """Fastest launch shape and BVH leaf size for `scene` (ssol_b200_autotune);
    returns (options, best_ms)."""
    o = opts if opts is not None else options()
    best = C.c_double()
    rng = scene.rng(seed=seed)
    scene.lib.call("ssol_b200_autotune", scene.scn, rng, int(trial_paths), C.byref(o),
                   C.byref(best))
    return o, best.value


def load_product(path=PRODUCT_LIB):
    """The B200 library; raises if it is not built (no silent fallback)."""
    if not os.path.exists(path):
        raise FileNotFoundError("libssol_b200.so is not built: run __graft_entry__.build()")
    return Lib(path)


def combined_ok(a, b, k=3.0, floor=0.0):
    """|Ea - Eb| <= k * sqrt(SEa^2 + SEb^2) (+ floor) for (E, V, SE) tuples."""
    return abs(a[0] - b[0]) <= k * math.sqrt(a[2] ** 2 + b[2] ** 2) + floor
