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


def oracle_float_frame(orc, cam, spp, depth, rr, seed=1, offset=0):
    """The oracle's FP32 physical-mode frame formed the way the GPU forms it: each
    sample's radiance (a one-sample sum in double holds the float exactly), summed in
    float32 in sample order, times the float 1 / spp; (pixels, 3) float32."""
    acc = np.zeros((cam["width"] * cam["height"], 3), np.float32)
    for k in range(spp):
        one = orc.render_sums(cam, 1, depth, rr, seed=seed, offset=offset + k)
        assert np.array_equal(one.astype(np.float32).astype(np.float64), one)
        acc = (acc + one.astype(np.float32)).astype(np.float32)
    return (acc * (np.float32(1.0) / np.float32(spp))).astype(np.float32)


def assert_bit_equal(got, want):
    """Two float images with the same bits in every channel."""
    g = np.ascontiguousarray(got, np.float32).reshape(-1, 3)
    w = np.ascontiguousarray(want, np.float32).reshape(-1, 3)
    bad = np.any(g.view(np.uint32) != w.view(np.uint32), axis=1)
    assert not bad.any(), (int(bad.sum()), np.nonzero(bad)[0][:8], g[bad][:3], w[bad][:3])
