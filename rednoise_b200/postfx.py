"""Canvas post-processing on the GPU with the reference's semantics
(toneMap, applyBloom, applyFXAA and AccumBuffer, src/Renderer.cpp:1353-1470).

Canvases are (height, width) uint32 arrays of 0xAARRGGBB pixels, as returned by
``Scene.render_reference`` / ``render_raytraced`` / ``render_photon_mapped``.
Each function returns a processed copy.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native


def _canvas(c) -> np.ndarray:
    a = np.ascontiguousarray(c, np.uint32).copy()
    if a.ndim != 2:
        raise ValueError("a canvas is a (height, width) uint32 array")
    return a


def tonemap(canvas, exposure: float = 1.0, gamma: float = 2.2) -> np.ndarray:
    """Reinhard tone mapping of the exposure-scaled colour, then gamma."""
    a = _canvas(canvas)
    h, w = a.shape
    _native.check(_native.load().rn_pt_tonemap(a.ctypes.data, w, h, ctypes.c_float(exposure), ctypes.c_float(gamma),
                                               0, None), "rn_pt_tonemap")
    return a


def bloom(canvas, threshold: float = 0.75, intensity: float = 0.7) -> np.ndarray:
    """Bright pass above ``threshold``, three separable 13-tap box blurs, added back."""
    a = _canvas(canvas)
    h, w = a.shape
    _native.check(_native.load().rn_pt_bloom(a.ctypes.data, w, h, ctypes.c_float(threshold),
                                             ctypes.c_float(intensity), 0, None), "rn_pt_bloom")
    return a


def fxaa(canvas) -> np.ndarray:
    """Blend interior pixels on luma edges towards their 4-neighbour average."""
    a = _canvas(canvas)
    h, w = a.shape
    _native.check(_native.load().rn_pt_fxaa(a.ctypes.data, w, h, 0, None), "rn_pt_fxaa")
    return a


class AccumBuffer:
    """Running per-pixel sum of canvases; ``resolve`` returns their mean canvas."""

    def __init__(self, width: int, height: int):
        self.width, self.height = int(width), int(height)
        self.sum = np.zeros(self.width * self.height * 3, np.float32)
        self.count = 0

    def add(self, canvas) -> None:
        a = np.ascontiguousarray(canvas, np.uint32)
        if a.shape != (self.height, self.width):
            raise ValueError("canvas size does not match the buffer")
        _native.check(_native.load().rn_pt_accum_add(self.sum.ctypes.data, a.ctypes.data, self.width, self.height,
                                                     0, None), "rn_pt_accum_add")
        self.count += 1

    def resolve(self) -> np.ndarray:
        out = np.zeros((self.height, self.width), np.uint32)
        _native.check(_native.load().rn_pt_accum_resolve(self.sum.ctypes.data, self.count, out.ctypes.data,
                                                         self.width, self.height, 0, None), "rn_pt_accum_resolve")
        return out
