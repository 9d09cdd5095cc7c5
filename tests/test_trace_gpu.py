"""GPU parity of closest-hit / any-hit traversal against the reference BVH.

Bar: triangle index bit-exact, t/u/v bit-exact (the kernels use the reference's
IEEE operation order), occlusion identical. Golden data come from the reference
build (tests/golden/make_golden.py); larger cases are checked against the CPU
oracle (pinned to the reference by tests/test_oracle.py) computed live.
"""
import os

import numpy as np
import pytest

import oracle
import raysets
import rednoise_b200 as rn
from rednoise_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "trace_ref.npz")), np.load(os.path.join(GOLD, "assets_ref.npz"))


def _v9(name, assets):
    return scenes.cornell_box()["vertices"] if name == "box" else assets[f"{name}_v"]


def ulp_distance(a, b):
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(ia - ib)


def nearest_consistent(idx, t, ref_idx, ref_t, max_frac=0.01):
    """Nearest-first traversal returns the (t, rank)-minimal hit. It departs from
    the reference only where the reference's float slab test pruned a leaf whose
    triangle lies a hair nearer (coplanar triangles, rays through a shared edge or
    vertex, where the two triangles' t differ by their rounding): there the hit
    must be no farther than the reference's and within 64 ULP of it."""
    bad = np.nonzero(idx != ref_idx)[0]
    assert bad.size <= max_frac * idx.size, bad.size
    assert (ref_idx[bad] >= 0).all() and (idx[bad] >= 0).all()
    assert (t[bad] <= ref_t[bad]).all()
    assert (ulp_distance(t[bad], ref_t[bad]) <= 64).all()
    same = idx == ref_idx
    assert np.array_equal(t[same].view(np.uint32), ref_t[same].view(np.uint32))
    return bad.size


@pytest.mark.parametrize("name", ["cornell", "sphere", "box"])
@pytest.mark.parametrize("mode", ["width4", "width2", "nearest"])
def test_closest_hit_matches_reference_golden(gold, name, mode):
    trace, assets = gold
    s = rn.Scene.from_arrays(_v9(name, assets))
    o, d = trace[f"{name}_o"], trace[f"{name}_d"]
    kw = {"nearest_first": mode == "nearest", "width2": mode == "width2"}
    idx, t, u, v = s.trace_closest(o, d, **kw)
    if mode == "nearest":
        nearest_consistent(idx, t, trace[f"{name}_idx"], trace[f"{name}_t"].view(np.float32))
        return
    # Reference order, 2-wide or 4-wide layout: bit-exact.
    assert np.array_equal(idx, trace[f"{name}_idx"]), np.nonzero(idx != trace[f"{name}_idx"])[0][:10]
    assert np.array_equal(t.view(np.uint32), trace[f"{name}_t"])
    assert np.array_equal(u.view(np.uint32), trace[f"{name}_u"])
    assert np.array_equal(v.view(np.uint32), trace[f"{name}_v"])
    if name != "box":
        ig = trace[f"{name}_ignore"]
        idx_i, t_i, _, _ = s.trace_closest(o, d, ignore=ig, **kw)
        assert np.array_equal(idx_i, trace[f"{name}_idx_ig"])
        assert np.array_equal(t_i.view(np.uint32), trace[f"{name}_t_ig"])


@pytest.mark.parametrize("name", ["cornell", "sphere", "box"])
@pytest.mark.parametrize("width2", [False, True])
def test_any_hit_matches_reference_golden(gold, name, width2):
    trace, assets = gold
    s = rn.Scene.from_arrays(_v9(name, assets))
    occ = s.trace_any(trace[f"{name}_o"], trace[f"{name}_d"], trace[f"{name}_tmax"], trace[f"{name}_ignore"],
                      width2=width2)
    assert np.array_equal(occ, trace[f"{name}_occ"])


def test_fan_kat(gold):
    """tests/tests.cpp:174-197 on the GPU: the 400-ray fan hits what brute force hits."""
    trace, assets = gold
    s = rn.Scene.from_arrays(assets["cornell_v"])
    o, d = raysets.fan_rays()
    idx, t, _, _ = s.trace_closest(o, d)
    assert (idx >= 0).sum() > 100
    assert np.array_equal(idx, trace["cornell_idx"][:400])


def test_triangle_kat():
    """tests/tests.cpp:150-165: t = 2 hit, reversed ray misses, nearer triangle wins at t = 1."""
    v = np.array([[-1, -1, -2, 1, -1, -2, 0, 1, -2], [-1, -1, -1, 1, -1, -1, 0, 1, -1]], np.float32)
    one = rn.Scene.from_arrays(v[:1])
    idx, t, _, _ = one.trace_closest([[0, 0, 0], [0, 0, 0]], [[0, 0, -1], [0, 0, 1]])
    assert idx[0] == 0 and abs(t[0] - 2.0) < 1e-4 and idx[1] == -1 and np.isinf(t[1])
    two = rn.Scene.from_arrays(v)
    idx, t, _, _ = two.trace_closest([[0, 0, 0]], [[0, 0, -1]])
    assert idx[0] == 1 and abs(t[0] - 1.0) < 1e-4
    assert two.trace_any([[0, 0, 0]], [[0, 0, -1]], [0.5])[0] == 0
    assert two.trace_any([[0, 0, 0]], [[0, 0, -1]], [1.5])[0] == 1


@pytest.mark.parametrize("count,seed", [(100000, 11), (400000, 12)])
def test_large_soup_matches_oracle(count, seed):
    sc = scenes.soup_scene(count, seed)
    v9 = sc["vertices"]
    lo, hi = raysets.scene_bounds(v9)
    o1, d1 = raysets.random_rays(40000, seed, lo, hi)
    o2, d2 = raysets.towards_rays(40000, seed + 1, v9, lo, hi)
    o, d = np.concatenate([o1, o2]), np.concatenate([d1, d2])
    orc = oracle.OrcBvh(v9)
    ri, rt, ru, rv = orc.intersect(o, d)
    s = rn.Scene.from_arrays(v9)
    for width2 in (False, True):
        gi, gt, gu, gv = s.trace_closest(o, d, width2=width2)
        bad = np.nonzero(gi != ri)[0]
        assert bad.size == 0, (width2, bad[:10])
        assert np.array_equal(gt.view(np.uint32), rt.view(np.uint32))
        assert np.array_equal(gu.view(np.uint32), ru.view(np.uint32))
    gi, gt, _, _ = s.trace_closest(o, d, nearest_first=True)
    nearest_consistent(gi, gt, ri, rt)
    tmax = np.random.default_rng(seed).random(o.shape[0]).astype(np.float32) * 5
    want = orc.occluded(o, d, tmax)
    assert np.array_equal(s.trace_any(o, d, tmax), want)
    assert np.array_equal(s.trace_any(o, d, tmax, width2=True), want)


def test_device_pointer_path_with_torch():
    torch = pytest.importorskip("torch")
    sc = scenes.soup_scene(20000, 21)
    v9 = sc["vertices"]
    lo, hi = raysets.scene_bounds(v9)
    o, d = raysets.random_rays(10000, 21, lo, hi)
    s = rn.Scene.from_arrays(v9)
    hi_idx, hi_t, _, _ = s.trace_closest(o, d)
    lib = rn._native.load()
    to = torch.from_numpy(o).cuda()
    td = torch.from_numpy(d).cuda()
    tri = torch.empty(o.shape[0], dtype=torch.int32, device="cuda")
    tt = torch.empty(o.shape[0], dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.rn_pt_trace_closest(s.handle, o.shape[0], to.data_ptr(), td.data_ptr(), None,
                                 rn._native.RN_PT_DEVICE_POINTERS, stream, tri.data_ptr(), tt.data_ptr(), None, None)
    assert st == 0
    torch.cuda.synchronize()
    assert np.array_equal(tri.cpu().numpy(), hi_idx)
    assert np.array_equal(tt.cpu().numpy().view(np.uint32), hi_t.view(np.uint32))


def test_scene_info_and_depth():
    sc = scenes.soup_scene(50000, 5)
    s = rn.Scene.from_arrays(sc["vertices"])
    info = s.info()
    assert info["num_triangles"] == 50036
    assert 1 < info["depth"] < 64
    assert info["device_bytes"] > 50036 * 48
