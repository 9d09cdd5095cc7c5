"""TEST INFRASTRUCTURE ONLY -- the CPU oracle of rednoise_b200.

Two checkers, loaded through ctypes:
  * ``ref()``  -- oracle/_ref/librn_ref.so: the reference renderer's own sources
    (BVH.cpp, Geometry.cpp, Renderer.cpp, ObjLoader.cpp, ...) compiled here by
    oracle/Makefile, plus the flat test shim oracle/ref_shim.cpp;
  * ``orc()``  -- oracle/_build/librn_oracle.so: the independent CPU restatement
    oracle/rn_oracle.cpp, pinned against ``ref()`` by tests/test_oracle.py.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py may use
this package; the product library never links or calls it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_PATH = os.path.join(HERE, "_ref", "librn_ref.so")
ORC_PATH = os.path.join(HERE, "_build", "librn_oracle.so")

vp = ctypes.c_void_p
ci = ctypes.c_int
cf = ctypes.c_float

_REF = None
_ORC = None


def P(a):
    """ctypes pointer of a contiguous numpy array (None passes NULL)."""
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def ref_available() -> bool:
    return os.path.isfile(REF_PATH)


def reference_dir():
    """The reference source tree: $RN_REFERENCE_DIR, else the directory oracle/Makefile
    built _ref/librn_ref.so from (recorded in _ref/source_dir.txt); None when neither
    names an existing directory (the GPU box has no reference tree)."""
    d = os.environ.get("RN_REFERENCE_DIR")
    if not d:
        rec = os.path.join(HERE, "_ref", "source_dir.txt")
        if os.path.isfile(rec):
            with open(rec) as f:
                d = f.read().strip()
    return d if d and os.path.isdir(d) else None


def ref() -> ctypes.CDLL:
    global _REF
    if _REF is None:
        lib = ctypes.CDLL(REF_PATH)
        sig = {
            "refsh_model_new": (vp, [ci, vp, vp, vp, vp, vp]),
            "refsh_model_from_obj": (vp, [ctypes.c_char_p, cf]),
            "refsh_model_count": (ci, [vp]),
            "refsh_model_get": (None, [vp, vp, vp, vp, vp, vp, vp]),
            "refsh_model_free": (None, [vp]),
            "refsh_bvh_new": (vp, [vp]),
            "refsh_bvh_free": (None, [vp]),
            "refsh_bvh_node_count": (ci, [vp]),
            "refsh_bvh_root": (ci, [vp]),
            "refsh_bvh_dump": (None, [vp, vp, vp, vp]),
            "refsh_bvh_intersect": (None, [vp, ci, vp, vp, vp, vp, vp, vp, vp]),
            "refsh_bvh_occluded": (None, [vp, ci, vp, vp, vp, vp, vp]),
            "refsh_brute_intersect": (None, [vp, ci, vp, vp, vp, vp]),
            "refsh_intersect_triangle": (ci, [vp, vp, vp, vp, vp, vp]),
            "refsh_render_pathtraced": (None, [vp, ci, ci, cf, vp, vp, ci, ci, vp, cf, cf, vp, ci, vp]),
            "refsh_render_raytraced": (None, [vp, ci, ci, cf, vp, vp, ci, ci, vp, cf, vp, vp]),
            "refsh_model_set_vertex_normals": (None, [vp, vp]),
            "refsh_render_photon_mapped": (None, [vp, ci, ci, cf, vp, vp, ci, ci, ci, vp, vp]),
            "refsh_tonemap": (None, [vp, ci, ci, cf, cf]),
            "refsh_bloom": (None, [vp, ci, ci, cf, cf]),
            "refsh_fxaa": (None, [vp, ci, ci]),
            "refsh_accum": (None, [ci, vp, ci, ci, vp]),
            "refsh_render_bidirectional": (None, [vp, ci, ci, cf, vp, vp, ci, cf, vp]),
            "refsh_render_metropolis": (None, [vp, ci, ci, cf, vp, vp, ci, cf, vp]),
            "rn_scene_load_obj": (vp, [ctypes.c_char_p, cf]),
            "rn_scene_free": (None, [vp]),
            "rn_render": (ci, [vp, ci, ci, ci, cf, ci, vp]),
        }
        for k, (r, a) in sig.items():
            getattr(lib, k).restype = r
            getattr(lib, k).argtypes = a
        _REF = lib
    return _REF


def orc() -> ctypes.CDLL:
    global _ORC
    if _ORC is None:
        lib = ctypes.CDLL(ORC_PATH)
        sig = {
            "orc_bvh_new": (vp, [ci, vp]),
            "orc_bvh_free": (None, [vp]),
            "orc_bvh_node_count": (ci, [vp]),
            "orc_bvh_dump": (None, [vp, vp, vp, vp]),
            "orc_intersect": (None, [vp, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
            "orc_occluded": (None, [vp, ci, vp, vp, vp, vp, vp, vp, vp]),
            "orc_render_reference": (None, [vp, vp, vp, vp, vp, ci, ci, ci, ci, cf, vp, vp, ci, ci, ci, vp, vp,
                                            vp]),
            "orc_pt_scene_new": (vp, [ci, vp, vp, vp, vp, vp]),
            "orc_pt_scene_free": (None, [vp]),
            "orc_pt_render": (None, [vp, vp, ci, ci, ci, ci, ci, ctypes.c_ulonglong, ctypes.c_uint, vp, ci, vp, ci,
                                     vp]),
            "orc_pt_count": (None, [vp, vp, ci, ci, ci, ci, ci, ctypes.c_ulonglong, ctypes.c_uint, vp, ci, vp, vp]),
            "orc_pt_backward": (None, [vp, vp, ci, ci, ci, ci, ci, ctypes.c_ulonglong, ctypes.c_uint, vp, vp, ci,
                                       vp, vp]),
            "orc_bsdf_eval": (None, [ci, vp, ctypes.c_double, vp, vp, ci, vp, vp, vp, vp]),
            "orc_bsdf_sample": (None, [ci, vp, ctypes.c_double, vp, vp, ci, vp, vp, vp, vp, vp]),
            "orc_sincos_turn": (None, [ci, vp, vp, vp]),
            "orc_bdpt_render": (None, [vp, vp, vp, ci, ci, ci, ci, cf, vp, vp, ci, cf, ci, ctypes.c_ulonglong, ci,
                                       vp, vp]),
            "orc_mlt_render": (None, [vp, vp, vp, ci, ci, cf, vp, vp, ctypes.c_longlong, ci, ci, ctypes.c_ulonglong,
                                      cf, ci, vp, vp, vp]),
        }
        for k, (r, a) in sig.items():
            getattr(lib, k).restype = r
            getattr(lib, k).argtypes = a
        _ORC = lib
    return _ORC


# ---- convenience wrappers ---------------------------------------------------------

def ref_postfx(kind: str, canvas, *args) -> np.ndarray:
    """The reference's toneMap / applyBloom / applyFXAA on a copy of canvas ((h, w) uint32)."""
    c = np.ascontiguousarray(canvas, np.uint32).copy()
    h, w = c.shape
    fn = {"tonemap": ref().refsh_tonemap, "bloom": ref().refsh_bloom, "fxaa": ref().refsh_fxaa}[kind]
    fn(P(c), w, h, *args)
    return c


def ref_accum(frames) -> np.ndarray:
    """The reference AccumBuffer: add every frame ((k, h, w) uint32), then resolve."""
    f = np.ascontiguousarray(frames, np.uint32)
    k, h, w = f.shape
    out = np.zeros((h, w), np.uint32)
    ref().refsh_accum(k, P(f), w, h, P(out))
    return out


class RefModel:
    """A reference triangle list (vector<ModelTriangle>) and, lazily, its BVH."""

    def __init__(self, handle):
        self.h = handle
        self._bvh = None

    @classmethod
    def from_obj(cls, path: str, scale: float) -> "RefModel":
        return cls(ref().refsh_model_from_obj(os.fsencode(path), scale))

    @classmethod
    def from_arrays(cls, v9, rgb=None, material=None, roughness=None, normal=None) -> "RefModel":
        v = np.ascontiguousarray(v9, np.float32).reshape(-1, 9)
        keep = [v]
        args = []
        for a, dt in ((rgb, np.int32), (material, np.int32), (roughness, np.float32), (normal, np.float32)):
            if a is None:
                args.append(None)
            else:
                arr = np.ascontiguousarray(a, dt)
                keep.append(arr)
                args.append(P(arr))
        return cls(ref().refsh_model_new(v.shape[0], P(v), *args))

    @property
    def count(self) -> int:
        return ref().refsh_model_count(self.h)

    def arrays(self) -> dict:
        n = self.count
        v = np.zeros((n, 9), np.float32)
        rgb = np.zeros((n, 3), np.int32)
        mat = np.zeros(n, np.int32)
        nrm = np.zeros((n, 3), np.float32)
        rough = np.zeros(n, np.float32)
        ref().refsh_model_get(self.h, P(v), P(rgb), P(mat), P(nrm), P(rough), None)
        return {"v": v, "rgb": rgb, "material": mat, "normal": nrm, "roughness": rough}

    def vertex_normals(self) -> np.ndarray:
        """ModelTriangle::vertexNormals of every triangle, (n, 9) float32."""
        vn = np.zeros((self.count, 9), np.float32)
        ref().refsh_model_get(self.h, None, None, None, None, None, P(vn))
        return vn

    def set_vertex_normals(self, vn9) -> None:
        vn = np.ascontiguousarray(vn9, np.float32).reshape(-1, 9)
        assert vn.shape[0] == self.count
        ref().refsh_model_set_vertex_normals(self.h, P(vn))

    def render_raytraced(self, w, h, focal=2.0, pos=(0, 0, 4), target=(0, 0, 0), shading=2, lights=None,
                         fog_density=0.0, fog_colour=None) -> np.ndarray:
        """The reference renderRaytraced (src/Renderer.cpp:909-948): 0xAARRGGBB canvas."""
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        lt = None if lights is None or len(lights) == 0 else np.ascontiguousarray(lights, np.float32).reshape(-1, 24)
        fog = None if fog_colour is None else np.asarray(fog_colour, np.float32)
        out = np.zeros((h, w), np.uint32)
        ref().refsh_render_raytraced(self.h, w, h, focal, P(pos), P(target), int(shading),
                                     0 if lt is None else lt.shape[0], P(lt), float(fog_density), P(fog), P(out))
        return out

    def render_photon_mapped(self, w, h, num_photons=200000, gather_rays=0, focal=2.0, pos=(0, 0, 4),
                             target=(0, 0, 0), lights=None) -> np.ndarray:
        """The reference renderPhotonMapped (src/Renderer.cpp:1300-1349): 0xAARRGGBB canvas."""
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        lt = None if lights is None or len(lights) == 0 else np.ascontiguousarray(lights, np.float32).reshape(-1, 24)
        out = np.zeros((h, w), np.uint32)
        ref().refsh_render_photon_mapped(self.h, w, h, focal, P(pos), P(target), int(num_photons), int(gather_rays),
                                         0 if lt is None else lt.shape[0], P(lt), P(out))
        return out

    def render_bidirectional(self, w, h, samples=64, exposure=40.0, focal=2.0, pos=(0, 0, 4),
                             target=(0, 0, 0)) -> np.ndarray:
        """The reference renderBidirectional (src/BDPT.cpp:65-144): 0xAARRGGBB canvas."""
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        out = np.zeros((h, w), np.uint32)
        ref().refsh_render_bidirectional(self.h, w, h, focal, P(pos), P(target), int(samples), float(exposure), P(out))
        return out

    def render_metropolis(self, w, h, mutations=4000000, exposure=16.0, focal=2.0, pos=(0, 0, 4),
                          target=(0, 0, 0)) -> np.ndarray:
        """The reference renderMetropolis (src/Metropolis.cpp:85-192): 0xAARRGGBB canvas."""
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        out = np.zeros((h, w), np.uint32)
        ref().refsh_render_metropolis(self.h, w, h, focal, P(pos), P(target), int(mutations), float(exposure), P(out))
        return out

    def bvh(self):
        if self._bvh is None:
            self._bvh = ref().refsh_bvh_new(self.h)
        return self._bvh

    def dump_bvh(self) -> dict:
        b = self.bvh()
        nn = ref().refsh_bvh_node_count(b)
        order = np.zeros(self.count, np.int32)
        bounds = np.zeros((nn, 6), np.float32)
        links = np.zeros((nn, 4), np.int32)
        ref().refsh_bvh_dump(b, P(order), P(bounds), P(links))
        return {"order": order, "bounds": bounds, "links": links, "root": ref().refsh_bvh_root(b)}

    def intersect(self, o, d, ignore=None):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = o.shape[0]
        ig = None if ignore is None else np.ascontiguousarray(ignore, np.int32)
        idx = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        ref().refsh_bvh_intersect(self.bvh(), n, P(o), P(d), P(ig), P(idx), P(t), P(u), P(v))
        return idx, t, u, v

    def occluded(self, o, d, tmax, ignore=None):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        tm = np.ascontiguousarray(tmax, np.float32)
        n = o.shape[0]
        ig = None if ignore is None else np.ascontiguousarray(ignore, np.int32)
        occ = np.zeros(n, np.int32)
        ref().refsh_bvh_occluded(self.bvh(), n, P(o), P(d), P(tm), P(ig), P(occ))
        return occ

    def brute(self, o, d):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = o.shape[0]
        idx = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        ref().refsh_brute_intersect(self.h, n, P(o), P(d), P(idx), P(t))
        return idx, t

    def render(self, w, h, samples, focal=2.0, pos=(0, 0, 4), target=(0, 0, 0), lights=None, aperture=0.0,
               focus=4.0, motion=(0, 0, 0), blades=0) -> np.ndarray:
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        motion = np.asarray(motion, np.float32)
        lt = None if lights is None or len(lights) == 0 else np.ascontiguousarray(lights, np.float32).reshape(-1, 24)
        out = np.zeros((h, w), np.uint32)
        ref().refsh_render_pathtraced(self.h, w, h, focal, P(pos), P(target), samples,
                                      0 if lt is None else lt.shape[0], P(lt), aperture, focus, P(motion), blades,
                                      P(out))
        return out

    def close(self):
        if self._bvh is not None:
            ref().refsh_bvh_free(self._bvh)
            self._bvh = None
        if self.h:
            ref().refsh_model_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bsdf_eval(mat, albedo, param, ng, wo, wi):
    """The physical estimator's BSDF in double precision for directions wi ((k, 3)):
    (f cos (k, 3), pdf (k,), ok (k,))."""
    a, n, o = (np.ascontiguousarray(x, np.float64) for x in (albedo, ng, wo))
    wi = np.ascontiguousarray(wi, np.float64).reshape(-1, 3)
    k = wi.shape[0]
    fc = np.zeros((k, 3))
    pdf = np.zeros(k)
    ok = np.zeros(k, np.int32)
    orc().orc_bsdf_eval(int(mat), P(a), float(param), P(n), P(o), k, P(wi), P(fc), P(pdf), P(ok))
    return fc, pdf, ok.astype(bool)


def bsdf_sample(mat, albedo, param, ng, wo, u):
    """Continuation samples from uniforms u ((count, 3)): (wi, weight, pdf, ok)."""
    a, n, o = (np.ascontiguousarray(x, np.float64) for x in (albedo, ng, wo))
    u = np.ascontiguousarray(u, np.float64).reshape(-1, 3)
    k = u.shape[0]
    wi = np.zeros((k, 3))
    w = np.zeros((k, 3))
    pdf = np.zeros(k)
    ok = np.zeros(k, np.int32)
    orc().orc_bsdf_sample(int(mat), P(a), float(param), P(n), P(o), k, P(u), P(wi), P(w), P(pdf), P(ok))
    return wi, w, pdf, ok.astype(bool)


def sincos_turn(u):
    """The FP32 estimator's (sin(2 pi u), cos(2 pi u)) for float32 u in [0, 1)."""
    u = np.ascontiguousarray(u, np.float32).reshape(-1)
    s = np.zeros_like(u)
    c = np.zeros_like(u)
    orc().orc_sincos_turn(u.size, P(u), P(s), P(c))
    return s, c


class OrcBvh:
    """The oracle restatement's BVH over a (n, 9) vertex array."""

    def __init__(self, v9):
        self.v = np.ascontiguousarray(v9, np.float32).reshape(-1, 9)
        self.h = orc().orc_bvh_new(self.v.shape[0], P(self.v))

    def dump(self) -> dict:
        nn = orc().orc_bvh_node_count(self.h)
        order = np.zeros(self.v.shape[0], np.int32)
        bounds = np.zeros((nn, 6), np.float32)
        links = np.zeros((nn, 4), np.int32)
        orc().orc_bvh_dump(self.h, P(order), P(bounds), P(links))
        return {"order": order, "bounds": bounds, "links": links}

    def intersect(self, o, d, ignore=None, counts=False):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = o.shape[0]
        ig = None if ignore is None else np.ascontiguousarray(ignore, np.int32)
        idx = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        bx = np.zeros(n, np.int32) if counts else None
        tr = np.zeros(n, np.int32) if counts else None
        orc().orc_intersect(self.h, n, P(o), P(d), P(ig), P(idx), P(t), P(u), P(v), P(bx), P(tr))
        return (idx, t, u, v, bx, tr) if counts else (idx, t, u, v)

    def occluded(self, o, d, tmax, ignore=None, counts=False):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        tm = np.ascontiguousarray(tmax, np.float32)
        n = o.shape[0]
        ig = None if ignore is None else np.ascontiguousarray(ignore, np.int32)
        occ = np.zeros(n, np.int32)
        bx = np.zeros(n, np.int32) if counts else None
        tr = np.zeros(n, np.int32) if counts else None
        orc().orc_occluded(self.h, n, P(o), P(d), P(tm), P(ig), P(occ), P(bx), P(tr))
        return (occ, bx, tr) if counts else occ

    def render_reference(self, normal, material, rgb, roughness, w, h, samples, y0=0, y1=None, focal=2.0,
                         pos=(0, 0, 4), target=(0, 0, 0), max_depth=4, lights=None, want_mean=False):
        y1 = h if y1 is None else y1
        nrm = np.ascontiguousarray(normal, np.float32)
        mat = np.ascontiguousarray(material, np.int32)
        col = np.ascontiguousarray(rgb, np.int32)
        rough = np.ascontiguousarray(roughness, np.float32)
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        lt = None if lights is None or len(lights) == 0 else np.ascontiguousarray(lights, np.float32).reshape(-1, 24)
        out = np.zeros((y1 - y0, w), np.uint32)
        mean = np.zeros((y1 - y0, w, 3), np.float32) if want_mean else None
        orc().orc_render_reference(self.h, P(nrm), P(mat), P(col), P(rough), w, h, y0, y1, focal, P(pos), P(target),
                                   samples, max_depth, 0 if lt is None else lt.shape[0], P(lt), P(out), P(mean))
        return (out, mean) if want_mean else out

    def render_bidirectional(self, normal, rgb, w, h, samples, exposure=40.0, stream=0, seed=0, y0=0, y1=None,
                             focal=2.0, pos=(0, 0, 4), target=(0, 0, 0), rtl=True, want_acc=False):
        """The restated bidirectional estimator (stream 0: the reference's per-row
        mt19937 streams; 1: Philox under seed). Rows [y0, y1)."""
        y1 = h if y1 is None else y1
        nrm = np.ascontiguousarray(normal, np.float32)
        col = np.ascontiguousarray(rgb, np.int32)
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        out = np.zeros((y1 - y0, w), np.uint32)
        acc = np.zeros((y1 - y0, w, 3), np.float32) if want_acc else None
        orc().orc_bdpt_render(self.h, P(nrm), P(col), w, h, y0, y1, focal, P(pos), P(target), int(samples),
                              float(exposure), int(stream), int(seed), int(bool(rtl)), P(out), P(acc))
        return (out, acc) if want_acc else out

    def render_metropolis(self, normal, rgb, w, h, mutations, chains, bootstrap=100000, seed=0, exposure=16.0,
                          focal=2.0, pos=(0, 0, 4), target=(0, 0, 0), rtl=True):
        """The restated many-chain Metropolis sampler: (canvas, unscaled deposits (h, w, 3), b)."""
        nrm = np.ascontiguousarray(normal, np.float32)
        col = np.ascontiguousarray(rgb, np.int32)
        pos = np.asarray(pos, np.float32)
        target = np.asarray(target, np.float32)
        img = np.zeros((h, w, 3), np.float32)
        b = ctypes.c_double(0.0)
        out = np.zeros((h, w), np.uint32)
        orc().orc_mlt_render(self.h, P(nrm), P(col), w, h, focal, P(pos), P(target), int(mutations), int(chains),
                             int(bootstrap), int(seed), float(exposure), int(bool(rtl)), P(img), ctypes.byref(b),
                             P(out))
        return out, img, b.value

    def __del__(self):
        try:
            orc().orc_bvh_free(self.h)
        except Exception:
            pass


class OrcPhysScene:
    """The oracle restatement of the physical estimator over a scene dict
    (vertices, albedo, emission, material, material_param)."""

    def __init__(self, sc: dict):
        self._keep = [np.ascontiguousarray(sc["vertices"], np.float32), np.ascontiguousarray(sc["albedo"], np.float32),
                      np.ascontiguousarray(sc["emission"], np.float32), np.ascontiguousarray(sc["material"], np.int32),
                      np.ascontiguousarray(sc["material_param"], np.float32)]
        v, a, e, m, p = self._keep
        self.h = orc().orc_pt_scene_new(v.shape[0], P(v), P(a), P(e), P(m), P(p))

    def render_sums(self, cam: dict, spp: int, max_depth: int, rr_depth: int, seed: int, offset: int = 0,
                    env=(0.0, 0.0, 0.0), pixels=None, double: bool = False) -> np.ndarray:
        """Per-pixel radiance SUMS over samples [offset, offset + spp), float64 (n, 3)."""
        c10 = np.array(list(cam["position"]) + list(cam["target"]) + list(cam["up"]) + [cam["vfov_deg"]], np.float32)
        envv = np.asarray(env, np.float32)
        w, h = cam["width"], cam["height"]
        px = None if pixels is None else np.ascontiguousarray(pixels, np.int32)
        n = w * h if px is None else px.size
        out = np.zeros((n, 3), np.float64)
        orc().orc_pt_render(self.h, P(c10), w, h, spp, max_depth, rr_depth, seed, offset, P(envv),
                            0 if px is None else px.size, P(px), 1 if double else 0, P(out))
        return out

    def backward(self, cam: dict, spp: int, max_depth: int, rr_depth: int, seed: int, d_image, offset: int = 0,
                 env=(0.0, 0.0, 0.0), double: bool = True):
        """Path-replay gradient: (dL/d albedo, dL/d emission), float64 (n, 3) each."""
        c10 = np.array(list(cam["position"]) + list(cam["target"]) + list(cam["up"]) + [cam["vfov_deg"]], np.float32)
        envv = np.asarray(env, np.float32)
        g = np.ascontiguousarray(d_image, np.float32).reshape(-1)
        n = self._keep[0].shape[0]
        ga = np.zeros((n, 3), np.float64)
        ge = np.zeros((n, 3), np.float64)
        orc().orc_pt_backward(self.h, P(c10), cam["width"], cam["height"], spp, max_depth, rr_depth, seed, offset,
                              P(envv), P(g), 1 if double else 0, P(ga), P(ge))
        return ga, ge

    def count_queries(self, cam: dict, spp: int, max_depth: int, rr_depth: int, seed: int, offset: int = 0,
                      env=(0.0, 0.0, 0.0), pixels=None) -> dict:
        """Reference-order query counts of the FP32 estimator on the listed pixels:
        closest / any-hit queries and their node-box and triangle tests."""
        c10 = np.array(list(cam["position"]) + list(cam["target"]) + list(cam["up"]) + [cam["vfov_deg"]], np.float32)
        envv = np.asarray(env, np.float32)
        px = None if pixels is None else np.ascontiguousarray(pixels, np.int32)
        out = np.zeros(6, np.int64)
        orc().orc_pt_count(self.h, P(c10), cam["width"], cam["height"], spp, max_depth, rr_depth, seed, offset,
                           P(envv), 0 if px is None else px.size, P(px), P(out))
        keys = ("closest", "any", "closest_boxes", "closest_tris", "any_boxes", "any_tris")
        return {k: int(v) for k, v in zip(keys, out)}

    def __del__(self):
        try:
            orc().orc_pt_scene_free(self.h)
        except Exception:
            pass
