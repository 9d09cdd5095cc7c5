"""The GPU-built linear BVH (rn_pt_scene_build_lbvh): closest hits agree with the
reference tree's, any-hits are identical, and renders agree on the same samples.

Nearest-first traversal of a different tree returns the nearest intersected
triangle, so it can differ from the reference tree only where two triangles are
hit at exactly the same distance (shared edges: the tie is broken by leaf
position, not by the reference's visit order), where two hits a few ULP apart are
kept or pruned by different box tests, or where a ray grazes a triangle at the
face of one tree's box but not the other's (rays aimed at vertices and edges).
"""
import numpy as np
import pytest

import raysets
import rednoise_b200 as rn
from rednoise_b200 import scenes

pytestmark = pytest.mark.gpu


def ulp_diff(a, b):
    a = a.view(np.int32).astype(np.int64)
    b = b.view(np.int32).astype(np.int64)
    return np.abs(a - b)


@pytest.mark.parametrize("kind", ["icosphere", "soup", "box"])
def test_lbvh_closest_hits_agree_with_reference_tree(kind):
    if kind == "icosphere":
        v9 = scenes.icosphere_scene(level=5)["vertices"]
    elif kind == "soup":
        v9 = scenes.soup_scene(50000, 7)["vertices"]
    else:
        v9 = scenes.cornell_box()["vertices"]
    s = rn.Scene.from_arrays(v9)
    ms = s.build_lbvh()
    assert ms > 0.0
    lo, hi = raysets.scene_bounds(v9)
    o1, d1 = raysets.random_rays(40000, 3, lo, hi)
    o2, d2 = raysets.towards_rays(20000, 4, v9, lo, hi)
    o, d = np.concatenate([o1, o2]), np.concatenate([d1, d2])
    ri, rt, _, _ = s.trace_closest(o, d)
    li, lt, _, _ = s.trace_closest(o, d, lbvh=True)
    hit = ri >= 0
    assert (hit == (li >= 0)).mean() > 0.9995
    both = hit & (li >= 0)
    # the same triangle, or a tie: another triangle at bit-identical distance
    agree = (ri == li) | (both & (rt.view(np.uint32) == lt.view(np.uint32))) | (~hit & (li < 0))
    n1 = o1.shape[0]
    assert agree[:n1].mean() > 0.999, agree[:n1].mean()  # random rays
    # rays aimed at vertices and edges meet near-ties, where which of two triangles a
    # few ULP apart is kept depends on the tree's box tests
    assert agree[n1:].mean() > 0.99, agree[n1:].mean()
    # random rays: where the triangles differ, the distances are near-ties
    b1 = both[:n1]
    assert (ulp_diff(rt[:n1][b1], lt[:n1][b1]) <= 64).mean() > 0.9999
    tmax = np.where(np.arange(o.shape[0]) % 3 == 0, 1e6, 2.0).astype(np.float32)
    occ_ref = s.trace_any(o, d, tmax)
    occ_gpu = s.trace_any(o, d, tmax, lbvh=True)
    assert (occ_ref != occ_gpu).mean() < 1e-3


def test_lbvh_render_agrees_with_reference_tree():
    sc = scenes.icosphere_scene(level=3)
    s = rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                             material=sc["material"], material_param=sc["material_param"])
    s.build_lbvh()
    c = scenes.camera(64, 48)
    cam = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], 64, 48)
    for integ in (1, 2):
        st = rn.Settings.make(spp=8, max_depth=6, rr_depth=3, seed=2, integrator=integ)
        a = s.render_physical(cam, st, nearest_first=True).astype(np.float64)
        b = s.render_physical(cam, st, lbvh=True).astype(np.float64)
        l1 = np.abs(a - b).sum() / np.abs(a).sum()
        assert l1 < 2e-3, l1


def test_lbvh_required_before_use():
    s = rn.Scene.from_arrays(scenes.cornell_box()["vertices"])
    o = np.zeros((1, 3), np.float32)
    d = np.array([[0, 0, -1]], np.float32)
    with pytest.raises(rn.RnError):
        s.trace_closest(o, d, lbvh=True)
    s.build_lbvh()
    s.trace_closest(o, d, lbvh=True)
