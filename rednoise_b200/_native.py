"""ctypes declarations for librednoise_b200.so (include/rednoise/*.h).

The library is built in-tree (``rednoise_b200/librednoise_b200.so``) by
``make -C rednoise_b200/csrc``. Loading fails loudly if it is missing: there is
no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# RN_B200_LIBRARY selects another build of the library (for instance the
# bounds-checked librednoise_b200_debug.so); the default is the in-tree release build.
LIB_PATH = os.environ.get("RN_B200_LIBRARY") or os.path.join(_HERE, "librednoise_b200.so")

RN_OK = 0
RN_ERR_INVALID_ARGUMENT = 1
RN_ERR_CUDA = 2
RN_ERR_OUT_OF_MEMORY = 3
RN_ERR_UNSUPPORTED = 4
RN_ERR_DEVICE_TIMEOUT = 5
RN_ERR_CAPACITY = 6
RN_ERR_INTERNAL = 7
RN_PT_DEVICE_POINTERS = 1
RN_PT_ORDER_NEAREST = 2
RN_PT_WIDTH2 = 4
RN_PT_WAVEFRONT_STATIC = 8
RN_PT_RAY_SORT = 16
RN_PT_NO_RAY_SORT = 32
RN_PT_LBVH = 64
RN_PT_SHADING_FLAT, RN_PT_SHADING_GOURAUD, RN_PT_SHADING_PHONG = 0, 1, 2
RN_PT_STATIC_MAX_PIXELS = 512 * 512
RN_PT_RNG_REFERENCE, RN_PT_RNG_COUNTER = 0, 1

STATUS_NAMES = {
    0: "RN_OK",
    1: "RN_ERR_INVALID_ARGUMENT",
    2: "RN_ERR_CUDA",
    3: "RN_ERR_OUT_OF_MEMORY",
    4: "RN_ERR_UNSUPPORTED",
    5: "RN_ERR_DEVICE_TIMEOUT",
    6: "RN_ERR_CAPACITY",
    7: "RN_ERR_INTERNAL",
}

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int)
vp = ctypes.c_void_p


class RnError(RuntimeError):
    """A non-RN_OK status from the native library."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("num_triangles", ctypes.c_int),
        ("vertices", vp),
        ("ref_rgb", vp),
        ("ref_material", vp),
        ("ref_roughness", vp),
        ("ref_normal", vp),
        ("albedo", vp),
        ("emission", vp),
        ("material", vp),
        ("material_param", vp),
        ("ref_vertex_normals", vp),
    ]


class SceneInfo(ctypes.Structure):
    _fields_ = [
        ("num_triangles", ctypes.c_int),
        ("internal_nodes", ctypes.c_int),
        ("depth", ctypes.c_int),
        ("device_bytes", ctypes.c_longlong),
        ("build_ms", ctypes.c_double),
    ]


class Light(ctypes.Structure):
    """rn_light: the reference Light's fields (src/Light.h:13-29)."""

    _fields_ = [
        ("type", ctypes.c_int),
        ("position", ctypes.c_float * 3),
        ("direction", ctypes.c_float * 3),
        ("colour", ctypes.c_float * 3),
        ("intensity", ctypes.c_float),
        ("radius", ctypes.c_float),
        ("cone_cos", ctypes.c_float),
        ("atten_constant", ctypes.c_float),
        ("atten_linear", ctypes.c_float),
        ("atten_quadratic", ctypes.c_float),
        ("u_axis", ctypes.c_float * 3),
        ("v_axis", ctypes.c_float * 3),
    ]

    @classmethod
    def default(cls, **kw) -> "Light":
        """A Light with the reference defaults (point light at (0, 0.95, 0))."""
        lt = cls()
        lt.type = 0
        lt.position[:] = (0.0, 0.95, 0.0)
        lt.direction[:] = (0.0, -1.0, 0.0)
        lt.colour[:] = (1.0, 1.0, 1.0)
        lt.intensity = 40.0
        lt.radius = 0.0
        lt.cone_cos = 0.9
        lt.atten_constant = 0.0
        lt.atten_linear = 0.0
        lt.atten_quadratic = 12.566370
        lt.u_axis[:] = (0.3, 0.0, 0.0)
        lt.v_axis[:] = (0.0, 0.0, 0.3)
        for k, v in kw.items():
            if isinstance(getattr(lt, k), ctypes.Array):
                getattr(lt, k)[:] = tuple(v)
            else:
                setattr(lt, k, v)
        return lt


class RefParams(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
        ("position", ctypes.c_float * 3),
        ("target", ctypes.c_float * 3),
        ("focal_length", ctypes.c_float),
        ("scale", ctypes.c_float),
        ("orthographic", ctypes.c_int),
        ("ortho_scale", ctypes.c_float),
        ("samples", ctypes.c_int),
        ("max_depth", ctypes.c_int),
        ("num_lights", ctypes.c_int),
        ("lights", ctypes.POINTER(Light)),
        ("aperture", ctypes.c_float),
        ("focus_distance", ctypes.c_float),
        ("camera_motion", ctypes.c_float * 3),
        ("aperture_blades", ctypes.c_int),
    ]


class Camera(ctypes.Structure):
    """rn_pt_camera: pinhole camera with a vertical field of view."""

    _fields_ = [
        ("position", ctypes.c_float * 3),
        ("target", ctypes.c_float * 3),
        ("up", ctypes.c_float * 3),
        ("vfov_deg", ctypes.c_float),
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
    ]

    @classmethod
    def make(cls, position, target, up=(0.0, 1.0, 0.0), vfov_deg=40.0, width=64, height=64) -> "Camera":
        c = cls()
        c.position[:] = tuple(float(x) for x in position)
        c.target[:] = tuple(float(x) for x in target)
        c.up[:] = tuple(float(x) for x in up)
        c.vfov_deg = vfov_deg
        c.width = int(width)
        c.height = int(height)
        return c


RN_PT_AUTO, RN_PT_MEGAKERNEL, RN_PT_WAVEFRONT = 0, 1, 2


class Settings(ctypes.Structure):
    """rn_pt_settings."""

    _fields_ = [
        ("spp", ctypes.c_int),
        ("max_depth", ctypes.c_int),
        ("rr_depth", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
        ("sample_offset", ctypes.c_uint),
        ("env", ctypes.c_float * 3),
    ]

    @classmethod
    def make(cls, spp=16, max_depth=5, rr_depth=None, integrator=RN_PT_AUTO, seed=0, sample_offset=0,
             env=(0.0, 0.0, 0.0)) -> "Settings":
        s = cls()
        s.spp = int(spp)
        s.max_depth = int(max_depth)
        s.rr_depth = int(max_depth if rr_depth is None else rr_depth)
        s.integrator = int(integrator)
        s.seed = int(seed)
        s.sample_offset = int(sample_offset)
        s.env[:] = tuple(float(x) for x in env)
        return s


class StageTimes(ctypes.Structure):
    """rn_pt_stage_times."""

    _fields_ = [(k, ctypes.c_double) for k in ("camera_ms", "ray_sort_ms", "extend_ms", "shade_ms", "shadow_sort_ms",
                                               "shadow_ms", "accumulate_ms", "total_ms")] + [
        (k, ctypes.c_int) for k in ("launches", "waves", "samples_per_wave", "dynamic_fetch", "ray_sort")]


class Tuning(ctypes.Structure):
    """rn_pt_tuning."""

    _fields_ = [
        ("integrator", ctypes.c_int),
        ("samples_per_wave", ctypes.c_int),
        ("megakernel_sps", ctypes.c_double),
        ("wavefront_sps", ctypes.c_double),
        ("dynamic_fetch", ctypes.c_int),
        ("ray_sort", ctypes.c_int),
    ]


class Job(ctypes.Structure):
    """rn_pt_job: scene + camera + settings."""

    _fields_ = [("scene", vp), ("camera", Camera), ("settings", Settings)]


# name -> (restype, argtypes)
SIGNATURES = {
    # drop-in ABI (include/rednoise/rednoise.h)
    "rn_scene_load_obj": (vp, [ctypes.c_char_p, ctypes.c_float]),
    "rn_scene_free": (None, [vp]),
    "rn_scene_triangle_count": (ctypes.c_int, [vp]),
    "rn_render": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, vp]),
    "rn_save_png": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, vp]),
    "rn_version": (ctypes.c_char_p, []),
    # additive ABI (include/rednoise/rednoise_pt.h)
    "rn_pt_scene_create": (ctypes.c_int, [ctypes.POINTER(SceneDesc), ctypes.POINTER(vp)]),
    "rn_pt_scene_prepare": (ctypes.c_int, [vp]),
    "rn_pt_scene_get_info": (ctypes.c_int, [vp, ctypes.POINTER(SceneInfo)]),
    "rn_pt_scene_dump_bvh": (ctypes.c_int, [vp, vp, c_int_p, vp, vp]),
    "rn_pt_scene_get_triangles": (ctypes.c_int, [vp, vp, vp, vp, vp]),
    "rn_pt_trace_closest": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, ctypes.c_uint, vp, vp, vp, vp, vp]),
    "rn_pt_trace_any": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_uint, vp, vp]),
    "rn_pt_ref_params_init": (None, [ctypes.POINTER(RefParams), ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_int]),
    "rn_pt_render_reference": (ctypes.c_int, [vp, ctypes.POINTER(RefParams), ctypes.c_uint, vp, vp, vp]),
    "rn_pt_render_raytraced": (ctypes.c_int, [vp, ctypes.POINTER(RefParams), ctypes.c_int, ctypes.c_float, vp,
                                              ctypes.c_uint, vp, vp]),
    "rn_pt_scene_get_vertex_normals": (ctypes.c_int, [vp, vp]),
    "rn_pt_scene_build_lbvh": (ctypes.c_int, [vp, vp, ctypes.POINTER(ctypes.c_double)]),
    "rn_pt_tonemap": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_uint,
                                     vp]),
    "rn_pt_bloom": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_uint,
                                   vp]),
    "rn_pt_fxaa": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint, vp]),
    "rn_pt_accum_add": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint, vp]),
    "rn_pt_accum_resolve": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint, vp]),
    "rn_pt_render_photon_mapped": (ctypes.c_int, [vp, ctypes.POINTER(RefParams), ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_uint, vp, vp, vp]),
    "rn_pt_inject_allocation_failure": (ctypes.c_int, [ctypes.c_longlong]),
    "rn_pt_render_bidirectional": (ctypes.c_int, [vp, ctypes.POINTER(RefParams), ctypes.c_int, ctypes.c_float,
                                                  ctypes.c_int, ctypes.c_ulonglong, ctypes.c_uint, vp, vp, vp]),
    "rn_pt_render_metropolis": (ctypes.c_int, [vp, ctypes.POINTER(RefParams), ctypes.c_longlong, ctypes.c_float,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_uint, vp, vp,
                                               vp, vp]),
    "rn_pt_render": (ctypes.c_int, [vp, ctypes.POINTER(Camera), ctypes.POINTER(Settings), ctypes.c_uint, vp, vp]),
    "rn_pt_render_accumulate": (ctypes.c_int, [vp, ctypes.POINTER(Camera), ctypes.POINTER(Settings), ctypes.c_uint,
                                               vp, vp]),
    "rn_pt_render_static": (ctypes.c_int, [vp, ctypes.POINTER(Camera), ctypes.POINTER(Settings), ctypes.c_uint, vp,
                                           vp]),
    "rn_pt_count_traversal": (ctypes.c_int, [vp, ctypes.POINTER(Camera), ctypes.POINTER(Settings), vp]),
    "rn_pt_profile_wavefront": (ctypes.c_int, [vp, ctypes.POINTER(Camera), ctypes.POINTER(Settings), ctypes.c_uint,
                                               vp, vp, ctypes.POINTER(StageTimes)]),
    "rn_pt_probe_read": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                        ctypes.POINTER(ctypes.c_float)]),
    "rn_pt_autotune": (ctypes.c_int, [vp, ctypes.POINTER(Camera), ctypes.POINTER(Settings), ctypes.c_uint,
                                      ctypes.POINTER(Tuning)]),
    "rn_pt_scene_set_materials": (ctypes.c_int, [vp, vp, vp, ctypes.c_uint, vp]),
    "rn_pt_backward": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(Camera), ctypes.POINTER(Settings),
                                      ctypes.POINTER(vp), ctypes.c_uint, vp, vp, vp]),
    "rn_pt_batch_create": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                          ctypes.POINTER(vp)]),
    "rn_pt_batch_render": (ctypes.c_int, [vp, ctypes.c_uint, ctypes.c_uint, vp, ctypes.POINTER(vp)]),
    "rn_pt_batch_integrator": (ctypes.c_int, [vp]),
    "rn_pt_batch_free": (None, [vp]),
    "rn_pt_last_error": (ctypes.c_char_p, []),
}

_LIB = None


def load() -> ctypes.CDLL:
    """Load the in-tree native library once and declare every signature."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.isfile(LIB_PATH):
        raise OSError(
            f"{LIB_PATH} is missing: build it with `make -C rednoise_b200/csrc` "
            "(or __graft_entry__.build()). There is no CPU fallback."
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(status: int, what: str = "") -> None:
    """Raise RnError for a non-RN_OK status, with the library's message."""
    if status != RN_OK:
        msg = load().rn_pt_last_error()
        msg = msg.decode("utf-8", "replace") if msg else ""
        raise RnError(status, f"{what}: {msg}" if what else msg)
