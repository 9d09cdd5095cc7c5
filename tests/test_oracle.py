"""Pin the CPU oracle (oracle/rn_oracle.cpp) against the reference itself.

Golden data: the reference's own known-answer tests for this path
(tests/tests.cpp:150-165 triangle KATs, 174-197 BVH-vs-brute fan) and the
fixtures that tests/golden/make_golden.py generated from the reference build.
Where the reference build (oracle/_ref) is present it is also run directly.
"""
import numpy as np
import pytest

import oracle
import raysets
from rednoise_b200 import scenes

GOLD = raysets.os.path.join(raysets.os.path.dirname(raysets.os.path.abspath(raysets.__file__)), "golden")


def load(name):
    return np.load(raysets.os.path.join(GOLD, name))


@pytest.fixture(scope="module")
def assets():
    return load("assets_ref.npz")


@pytest.fixture(scope="module")
def trace():
    return load("trace_ref.npz")


def test_triangle_kat():
    """tests/tests.cpp:150-165: t = 2 hit, reversed ray misses, nearer triangle wins at t = 1."""
    v = np.array([[-1, -1, -2, 1, -1, -2, 0, 1, -2]], np.float32)
    b = oracle.OrcBvh(v)
    idx, t, _, _ = b.intersect([[0, 0, 0]], [[0, 0, -1]])
    assert idx[0] == 0 and abs(t[0] - 2.0) < 1e-4
    idx, _, _, _ = b.intersect([[0, 0, 0]], [[0, 0, 1]])
    assert idx[0] == -1
    v2 = np.concatenate([v, np.array([[-1, -1, -1, 1, -1, -1, 0, 1, -1]], np.float32)])
    b2 = oracle.OrcBvh(v2)
    idx, t, _, _ = b2.intersect([[0, 0, 0]], [[0, 0, -1]])
    assert idx[0] == 1 and abs(t[0] - 1.0) < 1e-4


@pytest.mark.parametrize("name", ["cornell", "sphere", "box"])
def test_oracle_trace_matches_reference_golden(name, assets, trace):
    v9 = assets[f"{name}_v"] if name != "box" else scenes.cornell_box()["vertices"]
    b = oracle.OrcBvh(v9)
    o, d = trace[f"{name}_o"], trace[f"{name}_d"]
    idx, t, u, v = b.intersect(o, d)
    assert np.array_equal(idx, trace[f"{name}_idx"])
    assert np.array_equal(t.view(np.uint32), trace[f"{name}_t"])
    assert np.array_equal(u.view(np.uint32), trace[f"{name}_u"])
    assert np.array_equal(v.view(np.uint32), trace[f"{name}_v"])
    occ = b.occluded(o, d, trace[f"{name}_tmax"], trace[f"{name}_ignore"])
    assert np.array_equal(occ, trace[f"{name}_occ"])
    if name != "box":
        idx_i, t_i, _, _ = b.intersect(o, d, trace[f"{name}_ignore"])
        assert np.array_equal(idx_i, trace[f"{name}_idx_ig"])
        assert np.array_equal(t_i.view(np.uint32), trace[f"{name}_t_ig"])


def test_fan_bvh_equals_brute_force(assets, trace):
    """tests/tests.cpp:174-197 on the golden Cornell box: BVH hit == brute force, 0 mismatches."""
    fan = trace["cornell_idx"][:400]
    assert (fan >= 0).sum() > 0
    if oracle.ref_available():
        m = oracle.RefModel.from_arrays(assets["cornell_v"])
        o, d = raysets.fan_rays()
        bi, bt = m.brute(o, d)
        assert np.array_equal(bi, fan)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("seed,count", [(1, 5), (2, 37), (3, 1000), (4, 20000)])
def test_oracle_bvh_tree_matches_reference(seed, count):
    """Median-split build: identical triangle order, node boxes and links (src/BVH.cpp:6-63)."""
    rng = np.random.default_rng(seed)
    c = rng.random((count, 3)).astype(np.float32) * 4 - 2
    v9 = np.concatenate([c, c + rng.normal(scale=0.05, size=(count, 3)), c + rng.normal(scale=0.05, size=(count, 3))],
                        1).astype(np.float32)
    if seed == 2:  # coincident centroids and duplicated triangles
        v9[10:20] = v9[0]
    r = oracle.RefModel.from_arrays(v9).dump_bvh()
    o = oracle.OrcBvh(v9).dump()
    assert np.array_equal(r["order"], o["order"])
    assert np.array_equal(r["bounds"].view(np.uint32), o["bounds"].view(np.uint32))
    assert np.array_equal(r["links"], o["links"])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_oracle_trace_matches_reference_live():
    sc = scenes.soup_scene(3000, seed=7)
    v9 = sc["vertices"]
    lo, hi = raysets.scene_bounds(v9)
    o, d = raysets.random_rays(20000, 5, lo, hi)
    ref = oracle.RefModel.from_arrays(v9)
    orc = oracle.OrcBvh(v9)
    ri, rt, ru, rv = ref.intersect(o, d)
    oi, ot, ou, ov = orc.intersect(o, d)
    assert np.array_equal(ri, oi)
    assert np.array_equal(rt.view(np.uint32), ot.view(np.uint32))
    tmax = np.full(o.shape[0], 3.0, np.float32)
    assert np.array_equal(ref.occluded(o, d, tmax), orc.occluded(o, d, tmax))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_oracle_reference_render_matches_reference(assets):
    """The oracle's restated renderPathTraced is bit-exact with the reference on the CPU."""
    v9 = assets["cornell_v"]
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], assets["cornell_material"],
                                    assets["cornell_roughness"], assets["cornell_normal"])
    w, h, spp = 48, 36, 4
    ref_canvas = m.render(w, h, spp)
    orc = oracle.OrcBvh(v9)
    got = orc.render_reference(assets["cornell_normal"], assets["cornell_material"], assets["cornell_rgb"],
                               assets["cornell_roughness"], w, h, spp)
    assert np.array_equal(ref_canvas, got)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_oracle_light_types_match_reference(assets):
    """Every visibility branch (src/Renderer.cpp:390-498): oracle == reference build, bit for bit."""
    import rednoise_b200 as rn
    from test_refmode_gpu import LIGHT_CASES, _records

    v9 = assets["cornell_v"]
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], assets["cornell_material"],
                                    assets["cornell_roughness"], assets["cornell_normal"])
    orc = oracle.OrcBvh(v9)
    for case, kws in sorted(LIGHT_CASES.items()):
        lights = None if kws is None else _records([rn.Light.default(**kw) for kw in kws])
        want = m.render(40, 30, 2, lights=lights)
        got = orc.render_reference(assets["cornell_normal"], assets["cornell_material"], assets["cornell_rgb"],
                                   assets["cornell_roughness"], 40, 30, 2, lights=lights)
        assert np.array_equal(want, got), case


def test_golden_render_is_reference_c_abi(assets):
    """The golden rn_render image equals the oracle's restatement of renderPathTraced."""
    g = load("render_ref.npz")["rgba_64x48_4"]
    orc = oracle.OrcBvh(assets["cornell_v"])
    canvas = orc.render_reference(assets["cornell_normal"], assets["cornell_material"], assets["cornell_rgb"],
                                  assets["cornell_roughness"], 64, 48, 4)
    rgba = np.stack([(canvas >> 16) & 255, (canvas >> 8) & 255, canvas & 255, canvas >> 24], -1).astype(np.uint8)
    assert np.array_equal(rgba, g)


def _channels(canvas):
    c = np.asarray(canvas, np.uint32)
    return np.stack([(c >> 16) & 255, (c >> 8) & 255, c & 255], -1).astype(np.float64)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("w,h,spp,pos", [(40, 30, 4, (0, 0, 4)), (48, 36, 3, (0.3, 0.2, 3.5))])
def test_oracle_bidirectional_matches_reference(assets, w, h, spp, pos):
    """The restated renderBidirectional (reference per-row mt19937 streams) equals the
    reference build's canvas bit for bit; with the two random constructor arguments
    evaluated left to right instead it does not (GCC's order is right to left)."""
    v9 = assets["cornell_v"]
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], assets["cornell_material"],
                                    assets["cornell_roughness"], assets["cornell_normal"])
    want = m.render_bidirectional(w, h, spp, pos=pos)
    orc = oracle.OrcBvh(v9)
    got = orc.render_bidirectional(assets["cornell_normal"], assets["cornell_rgb"], w, h, spp, pos=pos)
    assert np.array_equal(want, got)
    ltr = orc.render_bidirectional(assets["cornell_normal"], assets["cornell_rgb"], w, h, spp, pos=pos, rtl=False)
    assert (ltr == want).mean() < 0.5
    rows = orc.render_bidirectional(assets["cornell_normal"], assets["cornell_rgb"], w, h, spp, y0=5, y1=9, pos=pos)
    assert np.array_equal(rows, want[5:9])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_oracle_bidirectional_counter_stream_estimates_the_same_image(assets):
    """The counter-stream estimator converges to the reference's image: at 64 spp the
    mean 8-bit level agrees within 1% and the per-pixel difference is noise-sized."""
    v9 = assets["cornell_v"]
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], assets["cornell_material"],
                                    assets["cornell_roughness"], assets["cornell_normal"])
    want = _channels(m.render_bidirectional(32, 24, 64))
    orc = oracle.OrcBvh(v9)
    got = _channels(orc.render_bidirectional(assets["cornell_normal"], assets["cornell_rgb"], 32, 24, 64, stream=1,
                                             seed=11))
    assert abs(got.mean() - want.mean()) < 0.01 * want.mean()
    assert np.abs(got - want).mean() < 4.0


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_oracle_metropolis_estimates_the_reference_image(assets):
    """The many-chain Metropolis restatement and the reference's 16-chain sampler
    estimate the same image: equal mean level within 1.5%, per-pixel differences
    within twice the reference's own run-to-run spread at 4x the mutations."""
    v9 = assets["cornell_v"]
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], assets["cornell_material"],
                                    assets["cornell_roughness"], assets["cornell_normal"])
    w, h, muts = 32, 24, 200000
    want = _channels(m.render_metropolis(w, h, muts))
    want4 = _channels(m.render_metropolis(w, h, 4 * muts))
    orc = oracle.OrcBvh(v9)
    canvas, img, b = orc.render_metropolis(assets["cornell_normal"], assets["cornell_rgb"], w, h, muts, muts // 64,
                                           bootstrap=20000, seed=5)
    got = _channels(canvas)
    assert b > 0 and img.sum() > 0
    assert abs(got.mean() - want4.mean()) < 0.015 * want4.mean()
    spread = np.abs(want - want4).mean()
    assert np.abs(got - want4).mean() < 2.0 * spread + 1.0
