"""Image comparison helpers shared by the reference-mode GPU tests (tests only)."""
from __future__ import annotations

import numpy as np


def argb_to_rgba(c):
    """Canvas 0xAARRGGBB -> (h, w, 4) uint8 RGBA."""
    c = np.asarray(c, np.uint32)
    return np.stack([(c >> 16) & 255, (c >> 8) & 255, c & 255, c >> 24], -1).astype(np.uint8)


def agree(a, b, min_equal=0.99, max_outlier_frac=0.01):
    """At least min_equal of channel values identical, at most max_outlier_frac off by more than 2."""
    a = np.asarray(a).astype(np.int32)
    b = np.asarray(b).astype(np.int32)
    eq = (a == b).mean()
    outliers = (np.abs(a - b) > 2).mean()
    assert eq >= min_equal, f"only {eq:.5f} of channel values identical"
    assert outliers <= max_outlier_frac, f"{outliers:.5f} of values differ by more than 2"
    return eq


def light_records(lights):
    """rn_light structures -> the reference shim's 24-float light records."""
    out = []
    for L in lights:
        r = np.zeros(24, np.float32)
        r[0] = L.type
        r[1:4] = L.position[:]
        r[4:7] = L.direction[:]
        r[7:10] = L.colour[:]
        r[10] = L.intensity
        r[11] = L.radius
        r[12] = L.cone_cos
        r[13:16] = (L.atten_constant, L.atten_linear, L.atten_quadratic)
        r[16:19] = L.u_axis[:]
        r[19:22] = L.v_axis[:]
        out.append(r)
    return np.stack(out)
