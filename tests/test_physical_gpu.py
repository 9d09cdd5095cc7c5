"""GPU parity of the physical-mode integrators against the CPU oracle.

The GPU and the oracle draw the same counter-based uniforms for every path and
compute each sample's radiance with the same IEEE float operations in the same
order (no multiply-add contraction on either side), so with common random numbers
a frame equals the oracle's per-sample radiance summed in float in sample order and
scaled by 1 / spp, bit for bit. Statistical checks (independent seeds, Russian
roulette, the FP64 estimator) use per-pixel confidence intervals or relative
tolerances.
"""
import numpy as np
import pytest

import oracle
import rednoise_b200 as rn
from imgcheck import assert_bit_equal, oracle_float_frame
from rednoise_b200 import scenes

pytestmark = pytest.mark.gpu


def make_scene(sc):
    return rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                                material=sc["material"], material_param=sc["material_param"])


def cam(w, h):
    return scenes.camera(w, h)


def gpu_render(s, c, spp, depth, rr=None, seed=1, offset=0, nearest=False, integrator=0):
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], c["width"], c["height"])
    st = rn.Settings.make(spp=spp, max_depth=depth, rr_depth=rr, seed=seed, sample_offset=offset,
                          integrator=integrator)
    return s.render_physical(camera, st, nearest_first=nearest)


def crn_agree(gpu_mean, orc_mean, rel_l1=2e-3, pix_frac=0.01):
    """Common-random-number agreement: image-level relative L1 and the fraction
    of pixels whose values differ by more than 1e-3 of the image's peak."""
    g = gpu_mean.reshape(-1, 3).astype(np.float64)
    o = orc_mean.reshape(-1, 3)
    l1 = np.abs(g - o).sum() / max(np.abs(o).sum(), 1e-30)
    peak = max(o.max(), 1e-30)
    frac = (np.abs(g - o).max(axis=1) > 1e-3 * peak).mean()
    assert l1 < rel_l1, f"relative L1 {l1:.2e}"
    assert frac < pix_frac, f"{frac:.4f} of pixels differ"
    return l1, frac


def oracle_frame(sc, c, spp, depth, rr, seed=1, offset=0):
    return oracle_float_frame(oracle.OrcPhysScene(sc), c, spp, depth, rr, seed=seed, offset=offset)


bit_equal = assert_bit_equal


@pytest.fixture(scope="module")
def box():
    return scenes.cornell_box()


def test_cornell_box_matches_oracle_crn(box):
    s = make_scene(box)
    c = cam(64, 48)
    spp, depth = 32, 5
    g = gpu_render(s, c, spp, depth)
    assert g.mean() > 0
    bit_equal(g, oracle_frame(box, c, spp, depth, depth))


def test_fp64_oracle_agrees(box):
    """FP32 GPU vs the oracle's FP64 estimator on the same samples."""
    s = make_scene(box)
    c = cam(48, 36)
    g = gpu_render(s, c, 32, 5)
    o = oracle.OrcPhysScene(box).render_sums(c, 32, 5, 5, seed=1, double=True) / 32
    crn_agree(g, o, rel_l1=5e-3, pix_frac=0.03)


@pytest.mark.parametrize("integrator", [1, 2])
def test_mixed_materials_match_oracle_crn(integrator):
    """Lambert, GGX and dielectric triangles, roulette from vertex 3: bit for bit."""
    sc = scenes.icosphere_scene(level=3)
    s = make_scene(sc)
    c = cam(64, 48)
    g = gpu_render(s, c, 16, 8, rr=3, integrator=integrator)
    bit_equal(g, oracle_frame(sc, c, 16, 8, 3))


def test_reference_order_equals_nearest_order_renders(box):
    s = make_scene(box)
    c = cam(48, 36)
    a = gpu_render(s, c, 16, 5, nearest=False)
    b = gpu_render(s, c, 16, 5, nearest=True)
    crn_agree(a, b, rel_l1=1e-3, pix_frac=0.01)


def test_accumulate_resume_is_bit_exact(box):
    """A render split over sample offsets equals one call, bit for bit."""
    s = make_scene(box)
    c = cam(40, 30)
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], 40, 30)
    one = np.zeros(40 * 30 * 3, np.float32)
    s.accumulate(camera, rn.Settings.make(spp=12, max_depth=5, seed=3), one)
    two = np.zeros(40 * 30 * 3, np.float32)
    s.accumulate(camera, rn.Settings.make(spp=5, max_depth=5, seed=3), two)
    s.accumulate(camera, rn.Settings.make(spp=7, max_depth=5, seed=3, sample_offset=5), two)
    assert np.array_equal(one.view(np.uint32), two.view(np.uint32))


def test_independent_seeds_within_confidence(box):
    """Two independent estimates agree within a per-pixel 99.9 % interval (Welch)."""
    s = make_scene(box)
    c = cam(24, 18)
    k = 8
    runs_a = np.stack([gpu_render(s, c, 64, 5, seed=100 + i) for i in range(k)])
    runs_b = np.stack([gpu_render(s, c, 64, 5, seed=200 + i) for i in range(k)])
    ma, mb = runs_a.mean(0), runs_b.mean(0)
    va, vb = runs_a.var(0, ddof=1) / k, runs_b.var(0, ddof=1) / k
    z = np.abs(ma - mb) / np.sqrt(va + vb + 1e-30)
    assert (z > 3.29).mean() < 0.01


def test_russian_roulette_is_unbiased():
    """Frame means with and without roulette agree within 4 standard errors
    (independent seeds, bright-light box)."""
    s = make_scene(scenes.cornell_box(light_scale=10.0))
    c = cam(32, 24)
    a = np.array([gpu_render(s, c, 64, 8, rr=8, seed=i).mean() for i in range(12)])
    b = np.array([gpu_render(s, c, 64, 8, rr=2, seed=50 + i).mean() for i in range(12)])
    z = abs(a.mean() - b.mean()) / np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)
    assert z < 4.0, (a.mean(), b.mean(), z)


@pytest.mark.parametrize("nearest", [False, True])
def test_wavefront_equals_megakernel(nearest):
    """Same estimator, same uniforms, same per-pixel summation order."""
    sc = scenes.icosphere_scene(level=3)
    s = make_scene(sc)
    c = cam(64, 48)
    a = gpu_render(s, c, 12, 8, rr=3, nearest=nearest, integrator=1)
    b = gpu_render(s, c, 12, 8, rr=3, nearest=nearest, integrator=2)
    bit_equal(b, a)
    # a second wavefront frame replays the captured graph with new sample indices
    b2 = gpu_render(s, c, 12, 8, rr=3, nearest=nearest, integrator=2, offset=12)
    a2 = gpu_render(s, c, 12, 8, rr=3, nearest=nearest, integrator=1, offset=12)
    bit_equal(b2, a2)
    assert not np.array_equal(a, a2)


def test_wavefront_static_and_refetch_agree():
    """One ray per lane vs lanes refetching rays: same hits, same image."""
    sc = scenes.icosphere_scene(level=3)
    s = make_scene(sc)
    c = cam(64, 48)
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], 64, 48)
    st = rn.Settings.make(spp=8, max_depth=8, rr_depth=3, seed=4, integrator=2)
    a = s.render_physical(camera, st)
    b = s.render_physical(camera, st, wavefront_static=True)
    m = s.render_physical(camera, rn.Settings.make(spp=8, max_depth=8, rr_depth=3, seed=4, integrator=1))
    bit_equal(a, b)
    bit_equal(a, m)


@pytest.mark.parametrize("static,level,w,h,spp", [(False, 3, 64, 48, 8), (True, 3, 64, 48, 8),
                                                  (False, 6, 320, 240, 32), (False, 3, 37, 23, 8),
                                                  (False, 2, 5, 3, 8)])
def test_ray_binning_changes_no_path(static, level, w, h, spp):
    """Binning each bounce's rays only reorders the queue: the image is bit-identical
    to the unbinned wavefront's and agrees with the megakernel's. The 320x240x32 case
    (2.46 M paths, 82k triangles) fills origin cells with thousands of rays each, so the
    second sort level places large cells by direction cell. The 37x23 and 5x3 frames
    are not whole 8 x 4 pixel tiles: the first queue's tile order then covers a ragged
    right and bottom strip, or the strips alone."""
    sc = scenes.icosphere_scene(level=level)
    s = make_scene(sc)
    c = cam(w, h)
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], w, h)
    st = rn.Settings.make(spp=spp, max_depth=8, rr_depth=3, seed=6, integrator=2)
    plain = s.render_physical(camera, st, wavefront_static=static, ray_sort=False)
    binned = s.render_physical(camera, st, wavefront_static=static, ray_sort=True)
    assert np.array_equal(plain.view(np.uint32), binned.view(np.uint32))
    m = s.render_physical(camera, rn.Settings.make(spp=spp, max_depth=8, rr_depth=3, seed=6, integrator=1))
    bit_equal(binned, m)
    # a second binned frame replays the captured graph
    binned2 = s.render_physical(camera, st, wavefront_static=static, ray_sort=True)
    assert np.array_equal(binned.view(np.uint32), binned2.view(np.uint32))


def test_autotune_reports_ray_binning():
    sc = scenes.icosphere_scene(level=3)
    s = make_scene(sc)
    c = cam(64, 48)
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], 64, 48)
    t = s.autotune(camera, rn.Settings.make(spp=8, max_depth=6, seed=1))
    assert t["ray_sort"] in (0, 1) and t["integrator"] in (1, 2)
    a = s.render_physical(camera, rn.Settings.make(spp=8, max_depth=6, seed=1))
    b = s.render_physical(camera, rn.Settings.make(spp=8, max_depth=6, seed=1, integrator=1))
    bit_equal(a, b)


def test_wavefront_matches_oracle_crn(box):
    s = make_scene(box)
    c = cam(48, 36)
    g = gpu_render(s, c, 16, 5, integrator=2)
    bit_equal(g, oracle_frame(box, c, 16, 5, 5))


def test_batched_wavefront_equals_per_job_megakernel():
    """Scenes of different sizes, resolutions and spp in one wave schedule (one
    captured graph) give the same images as per-job megakernel renders."""
    jobs, refs = [], []
    specs = [(scenes.soup_scene(800, 1), 32, 24, 4), (scenes.cornell_box(), 48, 36, 9),
             (scenes.soup_scene(5000, 2), 24, 40, 6), (scenes.icosphere_scene(level=2), 40, 30, 3)]
    keep = []
    for sc, w, h, spp in specs:
        s = make_scene(sc)
        keep.append(s)
        c = cam(w, h)
        camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], w, h)
        settings = rn.Settings.make(spp=spp, max_depth=6, seed=7, integrator=1)
        jobs.append((s, camera, settings))
        refs.append(s.render_physical(camera, settings))
    for integ, binning in ((2, None), (2, True), (1, None), (0, None), (0, True)):
        b = rn.Batch(jobs, integrator=integ, ray_sort=binning)
        assert b.integrator in (1, 2)
        outs = b.render()
        for o, r in zip(outs, refs):
            bit_equal(o, r)
        outs2 = b.render(sample_offset=1000)
        assert not np.array_equal(outs2[1], outs[1])
        b.close()


def test_traversal_counters_match_oracle():
    """The GPU's reference-traversal counters (roofline numerator) match the
    oracle's instrumented reference traversal over the same estimator's rays."""
    sc = scenes.icosphere_scene(level=4)
    s = make_scene(sc)
    c = cam(64, 48)
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], 64, 48)
    g = s.count_traversal(camera, rn.Settings.make(spp=4, max_depth=8, rr_depth=3, seed=5))
    o = oracle.OrcPhysScene(sc).count_queries(c, 4, 8, 3, seed=5)
    assert g["samples"] == 64 * 48 * 4
    for k in ("closest", "any", "closest_boxes", "closest_tris", "any_boxes", "any_tris"):
        assert abs(g[k] - o[k]) <= 0.01 * o[k] + 16, (k, g[k], o[k])


def test_invalid_settings_rejected(box):
    s = make_scene(box)
    c = rn.Camera.make((0, 0, 5), (0, 0, 5), width=8, height=8)
    with pytest.raises(rn.RnError):
        s.render_physical(c, rn.Settings.make(spp=1))
    c = rn.Camera.make((0, 0, 5), (0, 0, 0), width=8, height=8)
    with pytest.raises(rn.RnError):
        s.render_physical(c, rn.Settings.make(spp=1, max_depth=0))


def test_profile_wavefront_equals_render_and_times_every_stage():
    """The profiled frame (kernel by kernel, events between stages) renders the same
    image as rn_pt_render's captured frame and accounts for every stage."""
    sc = scenes.icosphere_scene(level=3)
    s = make_scene(sc)
    c = cam(64, 48)
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], 64, 48)
    for sort in (False, True):
        st = rn.Settings.make(spp=8, max_depth=6, rr_depth=3, seed=4, integrator=2)
        want = s.render_physical(camera, st, ray_sort=sort, wavefront_static=True)
        got, t = s.profile_wavefront(camera, st, ray_sort=sort, wavefront_static=True)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        assert t["ray_sort"] == int(sort) and t["dynamic_fetch"] == 0
        for k in ("camera_ms", "extend_ms", "shade_ms", "shadow_ms", "accumulate_ms"):
            assert t[k] > 0, (k, t)
        parts = sum(t[k] for k in ("camera_ms", "ray_sort_ms", "extend_ms", "shade_ms", "shadow_sort_ms",
                                   "shadow_ms", "accumulate_ms"))
        assert abs(parts - t["total_ms"]) <= 1e-3 * t["total_ms"] + 1e-3, (parts, t)
        # camera + accumulate, 3 stages per bounce, and 4 kernels per sort (count, column
        # scan, scatter, refine): 5 ray sorts and 6 shadow sorts at depth 6
        per_wave = 2 + 3 * 6 + (4 * 5 + 4 * 6 if sort else 0)
        assert t["launches"] == t["waves"] * per_wave + 1, t


def test_read_probe_measures_bandwidth():
    import ctypes

    import torch

    from rednoise_b200 import _native

    lib = _native.load()
    buf = torch.zeros(16 << 20, dtype=torch.uint8, device="cuda")
    ms = ctypes.c_float(0.0)
    _native.check(lib.rn_pt_probe_read(ctypes.c_void_p(buf.data_ptr()), buf.numel(), 8, 10, 1, None,
                                       ctypes.byref(ms)), "rn_pt_probe_read")
    gbs = buf.numel() * 8 * 10 / (ms.value / 1e3) / 1e9
    assert 100 < gbs < 200000, gbs
    assert lib.rn_pt_probe_read(ctypes.c_void_p(buf.data_ptr() + 4), 1024, 1, 1, 1, None,
                                ctypes.byref(ms)) == _native.RN_ERR_INVALID_ARGUMENT
    assert lib.rn_pt_probe_read(ctypes.c_void_p(buf.data_ptr()), 1024, 0, 1, 1, None,
                                ctypes.byref(ms)) == _native.RN_ERR_INVALID_ARGUMENT
