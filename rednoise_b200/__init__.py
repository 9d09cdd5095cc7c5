"""rednoise_b200: the RedNoise Monte-Carlo path tracer on B200 (sm_100a).

The module mirrors the reference Python binding
(bindings/python/rednoise/__init__.py: ``RenderMode``, ``Scene.load_obj``,
``Scene.render``, ``Image``, ``version``) over the same C ABI, served here by
CUDA kernels. ``Scene.render(mode="pathtraced")`` runs the reference path-tracer
semantics on the GPU. Additive APIs (array scenes, batched ray queries,
reference-mode renders with lights and depth of field) live on the same classes.
"""
from __future__ import annotations

import ctypes
import os
from enum import IntEnum
from typing import Optional, Sequence, Tuple, Union

import numpy as np

from . import _native
from ._native import Camera, Light, RnError, Settings

__all__ = ["RenderMode", "Scene", "Image", "Light", "Camera", "Settings", "RnError", "version"]
__version__ = "0.1.2"


class RenderMode(IntEnum):
    """Which renderer to run, mirroring the C ``rn_render_mode`` enum."""

    WIREFRAME = 0
    RASTERISED = 1
    RAYTRACED = 2
    PATHTRACED = 3

    @classmethod
    def coerce(cls, value: Union["RenderMode", int, str]) -> "RenderMode":
        """Coerce an int, a case-insensitive name or a member into a member."""
        if isinstance(value, cls):
            return value
        if isinstance(value, bool):
            raise TypeError("render mode must not be a bool")
        if isinstance(value, int):
            return cls(value)
        if isinstance(value, str):
            key = value.strip().upper().replace("-", "").replace("_", "").replace(" ", "")
            for member in cls:
                if member.name.replace("_", "") == key:
                    return member
            valid = ", ".join(m.name.lower() for m in cls)
            raise ValueError(f"unknown render mode {value!r}; expected one of: {valid}")
        raise TypeError(f"render mode must be RenderMode, int or str, not {type(value).__name__}")


def _sort_flag(ray_sort: Optional[bool]) -> int:
    if ray_sort is None:
        return 0
    return _native.RN_PT_RAY_SORT if ray_sort else _native.RN_PT_NO_RAY_SORT


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _f32(a, shape_last: Optional[int] = None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float32)
    if shape_last is not None and out.size % shape_last:
        raise ValueError(f"array size {out.size} is not a multiple of {shape_last}")
    return out


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


class Image:
    """An RGBA8 image (row-major ``width * height`` RGBA quadruplets)."""

    __slots__ = ("_rgba", "_width", "_height")

    def __init__(self, rgba: bytes, width: int, height: int):
        expected = width * height * 4
        if len(rgba) != expected:
            raise ValueError(f"rgba buffer has {len(rgba)} bytes, expected {expected} for a {width}x{height} image")
        self._rgba = bytes(rgba)
        self._width = int(width)
        self._height = int(height)

    @property
    def rgba(self) -> bytes:
        return self._rgba

    @property
    def width(self) -> int:
        return self._width

    @property
    def height(self) -> int:
        return self._height

    @property
    def size(self) -> Tuple[int, int]:
        return (self._width, self._height)

    def to_numpy(self) -> np.ndarray:
        """The pixels as a (height, width, 4) uint8 array."""
        return np.frombuffer(self._rgba, dtype=np.uint8).reshape(self._height, self._width, 4)

    def save(self, path: Union[str, os.PathLike]) -> None:
        """Write the image as a PNG through the native ``rn_save_png``."""
        path = os.fspath(path)
        ext = os.path.splitext(path)[1].lower()
        if ext and ext != ".png":
            raise ValueError(f"native saving only supports .png; got {ext!r}")
        ok = _native.load().rn_save_png(os.fsencode(path), self._width, self._height, self._rgba)
        if ok != 1:
            raise RuntimeError(f"rn_save_png failed to write {path!r}")

    def __repr__(self) -> str:
        return f"<rednoise_b200.Image {self._width}x{self._height} RGBA8>"


class Scene:
    """A scene backed by a native ``rn_scene`` handle (triangles + device BVH)."""

    __slots__ = ("_handle",)

    def __init__(self, handle: int):
        if not handle:
            raise ValueError("Scene requires a non-NULL native handle")
        self._handle = handle

    # ---- construction --------------------------------------------------------
    @classmethod
    def load_obj(cls, path: Union[str, os.PathLike], scale: float = 0.35) -> "Scene":
        """Load a Wavefront OBJ (and its .mtl), scaling vertices by ``scale``."""
        path = os.fspath(path)
        if not os.path.isfile(path):
            raise FileNotFoundError(f"OBJ file not found: {path!r}")
        handle = _native.load().rn_scene_load_obj(os.fsencode(path), ctypes.c_float(scale))
        if not handle:
            raise RuntimeError(f"rn_scene_load_obj failed to load {path!r}")
        return cls(handle)

    @classmethod
    def from_arrays(
        cls,
        vertices,
        *,
        ref_rgb=None,
        ref_material=None,
        ref_roughness=None,
        ref_normal=None,
        albedo=None,
        emission=None,
        material=None,
        material_param=None,
        ref_vertex_normals=None,
    ) -> "Scene":
        """Create a scene from arrays (``vertices``: (n, 9) or (n, 3, 3) floats)."""
        v = _f32(vertices, 9).reshape(-1, 9)
        n = v.shape[0]
        keep = [v]
        desc = _native.SceneDesc()
        desc.num_triangles = n
        desc.vertices = _ptr(v)

        def opt(arr, conv, width, field):
            if arr is None:
                return
            a = conv(arr).reshape(-1)
            if a.size != n * width:
                raise ValueError(f"{field}: expected {n * width} values, got {a.size}")
            keep.append(a)
            setattr(desc, field, _ptr(a))

        opt(ref_rgb, _i32, 3, "ref_rgb")
        opt(ref_material, _i32, 1, "ref_material")
        opt(ref_roughness, _f32, 1, "ref_roughness")
        opt(ref_normal, _f32, 3, "ref_normal")
        opt(albedo, _f32, 3, "albedo")
        opt(emission, _f32, 3, "emission")
        opt(material, _i32, 1, "material")
        opt(material_param, _f32, 1, "material_param")
        opt(ref_vertex_normals, _f32, 9, "ref_vertex_normals")
        out = ctypes.c_void_p()
        _native.check(_native.load().rn_pt_scene_create(ctypes.byref(desc), ctypes.byref(out)), "rn_pt_scene_create")
        return cls(out.value)

    # ---- reference API ------------------------------------------------------
    @property
    def triangle_count(self) -> int:
        self._check_open()
        return int(_native.load().rn_scene_triangle_count(self._handle))

    def render(
        self,
        mode: Union[RenderMode, int, str] = "pathtraced",
        width: int = 640,
        height: int = 480,
        cam_z: float = 4.0,
        samples: int = 64,
    ) -> Image:
        """Render through ``rn_render`` and return an :class:`Image`.

        ``"pathtraced"`` and ``"raytraced"`` are served; both run on the GPU with
        the reference's camera, default light, depth 4 and 8-bit output.
        """
        self._check_open()
        render_mode = RenderMode.coerce(mode)
        width, height = int(width), int(height)
        if width <= 0 or height <= 0:
            raise ValueError(f"width and height must be positive, got {width}x{height}")
        buf = ctypes.create_string_buffer(width * height * 4)
        lib = _native.load()
        ok = lib.rn_render(self._handle, int(render_mode), width, height, ctypes.c_float(cam_z), int(samples), buf)
        if ok != 1:
            msg = lib.rn_pt_last_error() or b""
            raise RuntimeError(f"rn_render failed (mode={render_mode.name}, {width}x{height}): {msg.decode()}")
        return Image(buf.raw, width, height)

    # ---- additive API ----------------------------------------------------------
    def prepare(self) -> None:
        """Build the reference BVH and upload the scene now."""
        self._check_open()
        _native.check(_native.load().rn_pt_scene_prepare(self._handle), "rn_pt_scene_prepare")

    def info(self) -> dict:
        self._check_open()
        inf = _native.SceneInfo()
        _native.check(_native.load().rn_pt_scene_get_info(self._handle, ctypes.byref(inf)), "rn_pt_scene_get_info")
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    def triangles(self) -> dict:
        """The scene's triangles: vertices (n, 9), ref_rgb (n, 3), ref_material (n,), normal (n, 3)."""
        self._check_open()
        n = self.triangle_count
        v = np.zeros((n, 9), np.float32)
        rgb = np.zeros((n, 3), np.int32)
        mat = np.zeros(n, np.int32)
        nrm = np.zeros((n, 3), np.float32)
        _native.check(_native.load().rn_pt_scene_get_triangles(self._handle, _ptr(v), _ptr(rgb), _ptr(mat),
                                                               _ptr(nrm)), "get_triangles")
        return {"vertices": v, "ref_rgb": rgb, "ref_material": mat, "normal": nrm}

    def bvh(self) -> dict:
        """The host-built BVH: ``order`` and per-node ``bounds`` / ``links``."""
        self._check_open()
        lib = _native.load()
        cnt = ctypes.c_int(0)
        _native.check(lib.rn_pt_scene_dump_bvh(self._handle, None, ctypes.byref(cnt), None, None), "dump_bvh")
        n = self.triangle_count
        order = np.zeros(n, np.int32)
        bounds = np.zeros((cnt.value, 6), np.float32)
        links = np.zeros((cnt.value, 4), np.int32)
        _native.check(lib.rn_pt_scene_dump_bvh(self._handle, _ptr(order), ctypes.byref(cnt), _ptr(bounds),
                                               _ptr(links)), "dump_bvh")
        return {"order": order, "bounds": bounds, "links": links}

    def trace_closest(self, origins, directions, ignore=None, nearest_first: bool = False, width2: bool = False,
                      lbvh: bool = False):
        """Closest hit per ray: (tri, t, u, v) numpy arrays (tri = -1 on a miss).
        ``width2`` traverses the 2-wide reference tree instead of its 4-wide collapse."""
        self._check_open()
        o = _f32(origins, 3).reshape(-1, 3)
        d = _f32(directions, 3).reshape(-1, 3)
        if o.shape != d.shape:
            raise ValueError("origins and directions must have the same shape")
        n = o.shape[0]
        ig = None if ignore is None else _i32(ignore).reshape(-1)
        tri = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        u = np.empty(n, np.float32)
        v = np.empty(n, np.float32)
        flags = (_native.RN_PT_ORDER_NEAREST if nearest_first else 0) | (_native.RN_PT_WIDTH2 if width2 else 0) | (
            _native.RN_PT_LBVH if lbvh else 0)
        _native.check(_native.load().rn_pt_trace_closest(self._handle, n, _ptr(o), _ptr(d), _ptr(ig), flags, None,
                                                         _ptr(tri), _ptr(t), _ptr(u), _ptr(v)), "trace_closest")
        return tri, t, u, v

    def trace_any(self, origins, directions, tmax, ignore=None, width2: bool = False, lbvh: bool = False) -> np.ndarray:
        """Occlusion per ray (1 if anything is hit strictly before ``tmax``)."""
        self._check_open()
        o = _f32(origins, 3).reshape(-1, 3)
        d = _f32(directions, 3).reshape(-1, 3)
        n = o.shape[0]
        tm = _f32(tmax).reshape(-1)
        if tm.size != n:
            raise ValueError("tmax must have one value per ray")
        ig = None if ignore is None else _i32(ignore).reshape(-1)
        occ = np.empty(n, np.int32)
        flags = (_native.RN_PT_WIDTH2 if width2 else 0) | (_native.RN_PT_LBVH if lbvh else 0)
        _native.check(_native.load().rn_pt_trace_any(self._handle, n, _ptr(o), _ptr(d), _ptr(tm), _ptr(ig), flags,
                                                     None, _ptr(occ)), "trace_any")
        return occ

    def render_reference(
        self,
        width: int,
        height: int,
        samples: int,
        *,
        position: Sequence[float] = (0.0, 0.0, 4.0),
        target: Sequence[float] = (0.0, 0.0, 0.0),
        focal_length: float = 2.0,
        scale: float = 150.0,
        lights: Optional[Sequence[Light]] = None,
        max_depth: int = 4,
        aperture: float = 0.0,
        focus_distance: float = 4.0,
        camera_motion: Sequence[float] = (0.0, 0.0, 0.0),
        aperture_blades: int = 0,
        orthographic: bool = False,
        ortho_scale: float = 1.0,
        want_mean: bool = False,
    ):
        """renderPathTraced semantics with every argument exposed.

        Returns the Canvas as (height, width) uint32 0xAARRGGBB, plus the float
        per-pixel sample mean (height, width, 3) when ``want_mean``.
        """
        self._check_open()
        p = _native.RefParams()
        _native.load().rn_pt_ref_params_init(ctypes.byref(p), int(width), int(height), ctypes.c_float(4.0),
                                             int(samples))
        p.position[:] = tuple(float(x) for x in position)
        p.target[:] = tuple(float(x) for x in target)
        p.focal_length = focal_length
        p.scale = scale
        p.max_depth = max_depth
        p.aperture = aperture
        p.focus_distance = focus_distance
        p.camera_motion[:] = tuple(float(x) for x in camera_motion)
        p.aperture_blades = aperture_blades
        p.orthographic = 1 if orthographic else 0
        p.ortho_scale = ortho_scale
        arr = None
        if lights:
            arr = (Light * len(lights))(*lights)
            p.num_lights = len(lights)
            p.lights = ctypes.cast(arr, ctypes.POINTER(Light))
        canvas = np.empty((height, width), np.uint32)
        mean = np.empty((height, width, 3), np.float32) if want_mean else None
        _native.check(_native.load().rn_pt_render_reference(self._handle, ctypes.byref(p), 0, None, _ptr(canvas),
                                                            _ptr(mean)), "render_reference")
        return (canvas, mean) if want_mean else canvas

    def _camera_params(self, width, height, position, target, focal_length, scale) -> "_native.RefParams":
        p = _native.RefParams()
        _native.load().rn_pt_ref_params_init(ctypes.byref(p), int(width), int(height), ctypes.c_float(4.0), 1)
        p.position[:] = tuple(float(x) for x in position)
        p.target[:] = tuple(float(x) for x in target)
        p.focal_length = focal_length
        p.scale = scale
        return p

    def render_bidirectional(
        self,
        width: int,
        height: int,
        samples: int = 64,
        exposure: float = 40.0,
        *,
        rng: str = "reference",
        seed: int = 0,
        position: Sequence[float] = (0.0, 0.0, 4.0),
        target: Sequence[float] = (0.0, 0.0, 0.0),
        focal_length: float = 2.0,
        scale: float = 150.0,
        want_rgb: bool = False,
    ):
        """renderBidirectional semantics (src/BDPT.cpp:65-144): the Canvas as
        (height, width) uint32 0xAARRGGBB. rng "reference" draws from the
        reference's per-row std::mt19937 streams (the reference's canvas); "counter"
        from Philox streams under seed. want_rgb adds the (height, width, 3) float
        image before tone mapping."""
        self._check_open()
        if rng not in ("reference", "counter"):
            raise ValueError("rng must be 'reference' or 'counter'")
        p = self._camera_params(width, height, position, target, focal_length, scale)
        canvas = np.empty((height, width), np.uint32)
        rgb = np.empty((height, width, 3), np.float32) if want_rgb else None
        mode = _native.RN_PT_RNG_REFERENCE if rng == "reference" else _native.RN_PT_RNG_COUNTER
        _native.check(_native.load().rn_pt_render_bidirectional(self._handle, ctypes.byref(p), int(samples),
                                                                ctypes.c_float(exposure), mode, int(seed), 0, None,
                                                                _ptr(canvas), _ptr(rgb)), "render_bidirectional")
        return (canvas, rgb) if want_rgb else canvas

    def render_metropolis(
        self,
        width: int,
        height: int,
        mutations: int = 4000000,
        exposure: float = 16.0,
        *,
        chains: int = 0,
        bootstrap: int = 100000,
        seed: int = 0,
        position: Sequence[float] = (0.0, 0.0, 4.0),
        target: Sequence[float] = (0.0, 0.0, 0.0),
        focal_length: float = 2.0,
        scale: float = 150.0,
        want_rgb: bool = False,
    ):
        """renderMetropolis semantics (src/Metropolis.cpp:85-192) with the steps
        split over parallel chains: the Canvas as (height, width) uint32. want_rgb
        adds the normalised (height, width, 3) radiance estimate and the bootstrap
        mean luminance b."""
        self._check_open()
        p = self._camera_params(width, height, position, target, focal_length, scale)
        canvas = np.empty((height, width), np.uint32)
        rgb = np.empty((height, width, 3), np.float32) if want_rgb else None
        b = ctypes.c_double(0.0)
        _native.check(_native.load().rn_pt_render_metropolis(self._handle, ctypes.byref(p), int(mutations),
                                                             ctypes.c_float(exposure), int(chains), int(bootstrap),
                                                             int(seed), 0, None, _ptr(canvas), _ptr(rgb),
                                                             ctypes.byref(b)), "render_metropolis")
        return (canvas, rgb, b.value) if want_rgb else canvas

    def render_raytraced(
        self,
        width: int,
        height: int,
        *,
        position: Sequence[float] = (0.0, 0.0, 4.0),
        target: Sequence[float] = (0.0, 0.0, 0.0),
        focal_length: float = 2.0,
        scale: float = 150.0,
        lights: Optional[Sequence[Light]] = None,
        max_depth: int = 4,
        shading: int = _native.RN_PT_SHADING_PHONG,
        fog_density: float = 0.0,
        fog_colour: Optional[Sequence[float]] = None,
        orthographic: bool = False,
        ortho_scale: float = 1.0,
    ) -> np.ndarray:
        """renderRaytraced semantics (Whitted ray tracing): the Canvas as
        (height, width) uint32 0xAARRGGBB."""
        self._check_open()
        p = _native.RefParams()
        _native.load().rn_pt_ref_params_init(ctypes.byref(p), int(width), int(height), ctypes.c_float(4.0), 1)
        p.position[:] = tuple(float(x) for x in position)
        p.target[:] = tuple(float(x) for x in target)
        p.focal_length = focal_length
        p.scale = scale
        p.max_depth = max_depth
        p.orthographic = 1 if orthographic else 0
        p.ortho_scale = ortho_scale
        arr = None
        if lights:
            arr = (Light * len(lights))(*lights)
            p.num_lights = len(lights)
            p.lights = ctypes.cast(arr, ctypes.POINTER(Light))
        fog = None if fog_colour is None else np.asarray(fog_colour, np.float32)
        canvas = np.empty((height, width), np.uint32)
        _native.check(_native.load().rn_pt_render_raytraced(self._handle, ctypes.byref(p), int(shading),
                                                            ctypes.c_float(fog_density), _ptr(fog), 0, None,
                                                            _ptr(canvas)), "render_raytraced")
        return canvas

    def render_photon_mapped(
        self,
        width: int,
        height: int,
        num_photons: int = 200000,
        *,
        gather_rays: int = 0,
        position: Sequence[float] = (0.0, 0.0, 4.0),
        target: Sequence[float] = (0.0, 0.0, 0.0),
        focal_length: float = 2.0,
        scale: float = 150.0,
        lights: Optional[Sequence[Light]] = None,
        return_count: bool = False,
    ):
        """renderPhotonMapped semantics: the Canvas as (height, width) uint32
        0xAARRGGBB (and the number of stored photons with ``return_count``)."""
        self._check_open()
        p = _native.RefParams()
        _native.load().rn_pt_ref_params_init(ctypes.byref(p), int(width), int(height), ctypes.c_float(4.0), 1)
        p.position[:] = tuple(float(x) for x in position)
        p.target[:] = tuple(float(x) for x in target)
        p.focal_length = focal_length
        p.scale = scale
        arr = None
        if lights:
            arr = (Light * len(lights))(*lights)
            p.num_lights = len(lights)
            p.lights = ctypes.cast(arr, ctypes.POINTER(Light))
        canvas = np.empty((height, width), np.uint32)
        count = ctypes.c_uint(0)
        _native.check(_native.load().rn_pt_render_photon_mapped(self._handle, ctypes.byref(p), int(num_photons),
                                                                int(gather_rays), 0, None, _ptr(canvas),
                                                                ctypes.byref(count)), "render_photon_mapped")
        return (canvas, int(count.value)) if return_count else canvas

    def build_lbvh(self) -> float:
        """Build the GPU linear BVH (used by calls given ``lbvh=True``); returns its build time in ms."""
        self._check_open()
        ms = ctypes.c_double(0.0)
        _native.check(_native.load().rn_pt_scene_build_lbvh(self._handle, None, ctypes.byref(ms)),
                      "rn_pt_scene_build_lbvh")
        return ms.value

    def vertex_normals(self) -> np.ndarray:
        """Per-corner vertex normals, (n, 9) float32 (the OBJ loader's smoothing)."""
        self._check_open()
        out = np.zeros((self.triangle_count, 9), np.float32)
        _native.check(_native.load().rn_pt_scene_get_vertex_normals(self._handle, _ptr(out)), "vertex_normals")
        return out

    def render_physical(self, camera: "Camera", settings: "Settings", nearest_first: bool = False,
                        out: Optional[np.ndarray] = None, wavefront_static: bool = False,
                        ray_sort: Optional[bool] = None, lbvh: bool = False) -> np.ndarray:
        """Physical-mode render: per-pixel mean radiance as (height, width, 3) float32.
        ``ray_sort`` forces the wavefront's ray binning on or off (None: the tuned choice)."""
        self._check_open()
        rgb = out if out is not None else np.empty((camera.height, camera.width, 3), np.float32)
        flags = (_native.RN_PT_ORDER_NEAREST if nearest_first else 0) | (
            _native.RN_PT_WAVEFRONT_STATIC if wavefront_static else 0) | _sort_flag(ray_sort) | (
            _native.RN_PT_LBVH if lbvh else 0)
        _native.check(_native.load().rn_pt_render(self._handle, ctypes.byref(camera), ctypes.byref(settings), flags,
                                                  None, _ptr(rgb)), "rn_pt_render")
        return rgb

    def accumulate(self, camera: "Camera", settings: "Settings", accum: np.ndarray,
                   nearest_first: bool = False) -> np.ndarray:
        """Add the per-pixel sum of the settings' samples to ``accum`` (float32, in place)."""
        self._check_open()
        if accum.dtype != np.float32 or not accum.flags.c_contiguous or accum.size != camera.width * camera.height * 3:
            raise ValueError("accum must be a contiguous float32 array of width*height*3 values")
        flags = _native.RN_PT_ORDER_NEAREST if nearest_first else 0
        _native.check(_native.load().rn_pt_render_accumulate(self._handle, ctypes.byref(camera),
                                                             ctypes.byref(settings), flags, None, _ptr(accum)),
                      "rn_pt_render_accumulate")
        return accum

    def profile_wavefront(self, camera: "Camera", settings: "Settings", ray_sort: Optional[bool] = None,
                          wavefront_static: bool = False) -> Tuple[np.ndarray, dict]:
        """One wavefront frame launched stage by stage with CUDA events between the
        stages (the configuration an RN_PT_AUTO render would use): (mean image as
        (height, width, 3) float32, per-stage device milliseconds and counts)."""
        self._check_open()
        rgb = np.empty((camera.height, camera.width, 3), np.float32)
        t = _native.StageTimes()
        flags = _sort_flag(ray_sort) | (_native.RN_PT_WAVEFRONT_STATIC if wavefront_static else 0)
        _native.check(_native.load().rn_pt_profile_wavefront(self._handle, ctypes.byref(camera),
                                                             ctypes.byref(settings), flags, None, _ptr(rgb),
                                                             ctypes.byref(t)), "rn_pt_profile_wavefront")
        return rgb, {k: getattr(t, k) for k, _ in t._fields_}

    def autotune(self, camera: "Camera", settings: "Settings", nearest_first: bool = False) -> dict:
        """Measure megakernel vs wavefront (and wavefront queue capacities) for this
        camera / settings; RN_PT_AUTO renders then use the fastest."""
        self._check_open()
        t = _native.Tuning()
        flags = _native.RN_PT_ORDER_NEAREST if nearest_first else 0
        _native.check(_native.load().rn_pt_autotune(self._handle, ctypes.byref(camera), ctypes.byref(settings), flags,
                                                    ctypes.byref(t)), "rn_pt_autotune")
        return {k: getattr(t, k) for k, _ in t._fields_}

    def set_materials(self, albedo=None, emission=None) -> None:
        """Overwrite per-triangle albedo and / or emitted radiance (host arrays, n x 3)."""
        self._check_open()
        a = None if albedo is None else _f32(albedo).reshape(-1)
        e = None if emission is None else _f32(emission).reshape(-1)
        n3 = 3 * self.triangle_count
        for x in (a, e):
            if x is not None and x.size != n3:
                raise ValueError(f"expected {n3} values")
        _native.check(_native.load().rn_pt_scene_set_materials(self._handle, _ptr(a), _ptr(e), 0, None),
                      "rn_pt_scene_set_materials")

    def backward(self, views, d_images):
        """Path-replay adjoint over views [(camera, settings)] given dL/d(mean image) per
        view (host arrays, h x w x 3). Returns (d_albedo, d_emission), each n x 3 float32."""
        self._check_open()
        nv = len(views)
        cams = (_native.Camera * nv)(*[v[0] for v in views])
        sets = (_native.Settings * nv)(*[v[1] for v in views])
        imgs = [_f32(g).reshape(-1) for g in d_images]
        for (c, _), g in zip(views, imgs):
            if g.size != c.width * c.height * 3:
                raise ValueError("image gradient size does not match its camera")
        ptrs = (ctypes.c_void_p * nv)(*[g.ctypes.data for g in imgs])
        n = self.triangle_count
        ga = np.zeros((n, 3), np.float32)
        ge = np.zeros((n, 3), np.float32)
        _native.check(_native.load().rn_pt_backward(self._handle, nv, cams, sets, ptrs, 0, None, _ptr(ga), _ptr(ge)),
                      "rn_pt_backward")
        return ga, ge

    def count_traversal(self, camera: "Camera", settings: "Settings") -> dict:
        """Reference-traversal test counts over one render's rays (profiling counters)."""
        self._check_open()
        out = np.zeros(7, np.int64)
        _native.check(_native.load().rn_pt_count_traversal(self._handle, ctypes.byref(camera),
                                                           ctypes.byref(settings), _ptr(out)),
                      "rn_pt_count_traversal")
        keys = ("samples", "closest", "any", "closest_boxes", "closest_tris", "any_boxes", "any_tris")
        return {k: int(v) for k, v in zip(keys, out)}

    # ---- lifetime ----------------------------------------------------------------
    @property
    def handle(self) -> int:
        return self._handle

    def close(self) -> None:
        """Release the native scene. Safe to call multiple times."""
        handle = self._handle
        if handle:
            self._handle = 0
            if _native._LIB is not None:
                _native._LIB.rn_scene_free(handle)

    def _check_open(self) -> None:
        if not self._handle:
            raise RuntimeError("operation on a closed Scene")

    def __enter__(self) -> "Scene":
        return self

    def __exit__(self, exc_type, exc_val, exc_tb) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __repr__(self) -> str:
        if not self._handle:
            return "<rednoise_b200.Scene closed>"
        return f"<rednoise_b200.Scene handle=0x{self._handle:x}>"


class Batch:
    """Many (scene, camera, settings) jobs rendered per launch (rn_pt_batch_*).

    With ``integrator=RN_PT_WAVEFRONT`` all jobs share one wave schedule whose
    frame is captured once as a CUDA graph and replayed on every ``render``.
    """

    def __init__(self, jobs, integrator: int = _native.RN_PT_AUTO, nearest_first: bool = False,
                 ray_sort: Optional[bool] = None):
        self._scenes = [j[0] for j in jobs]  # keep the scenes alive
        arr = (_native.Job * len(jobs))()
        for i, (scene, camera, settings) in enumerate(jobs):
            arr[i].scene = scene.handle
            arr[i].camera = camera
            arr[i].settings = settings
        self._shapes = [(c.height, c.width, 3) for _, c, _ in jobs]
        out = ctypes.c_void_p()
        flags = (_native.RN_PT_ORDER_NEAREST if nearest_first else 0) | _sort_flag(ray_sort)
        _native.check(_native.load().rn_pt_batch_create(arr, len(jobs), integrator, flags, ctypes.byref(out)),
                      "rn_pt_batch_create")
        self._handle = out.value

    @property
    def integrator(self) -> int:
        return int(_native.load().rn_pt_batch_integrator(self._handle))

    def render(self, sample_offset: int = 0, outs=None):
        """Render every job; returns a list of (h, w, 3) float32 mean images."""
        outs = outs if outs is not None else [np.empty(s, np.float32) for s in self._shapes]
        ptrs = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        _native.check(_native.load().rn_pt_batch_render(self._handle, int(sample_offset), 0, None, ptrs),
                      "rn_pt_batch_render")
        return outs

    def render_device(self, outs, stream_handle: int = 0, sample_offset: int = 0) -> None:
        """Asynchronous render into device buffers (sequence of data pointers)."""
        ptrs = (ctypes.c_void_p * len(outs))(*outs)
        _native.check(_native.load().rn_pt_batch_render(self._handle, int(sample_offset),
                                                        _native.RN_PT_DEVICE_POINTERS,
                                                        ctypes.c_void_p(stream_handle) if stream_handle else None,
                                                        ptrs), "rn_pt_batch_render")

    def close(self) -> None:
        if self._handle and _native._LIB is not None:
            _native._LIB.rn_pt_batch_free(self._handle)
        self._handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def version() -> str:
    """The native library version string ("0.1.2", as the reference reports)."""
    raw = _native.load().rn_version()
    return raw.decode("utf-8", "replace") if raw else ""
