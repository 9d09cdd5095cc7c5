"""Parity of the physical estimator at the benchmarked configuration.

The 1.31M-triangle displaced icosphere in the Cornell box (60 % Lambert, 25 % GGX
metal, 15 % dielectric by seeded hash), 1920x1080, depth 8, Russian roulette from
vertex 3: the GPU's megakernel and its wavefront (autotuned, one wave per frame)
against the CPU oracle on the 512 seeded pixels of the FP64 reference
(tests/golden/fp64_ref.npz).

* Common random numbers: both sides draw the same counter-based uniforms, use the
  reference traversal (bit-exact closest hits), IEEE division and square roots,
  the same quarter-turn sin/cos and no multiply-add contraction, so each sample's
  radiance is the same float on both sides, bit for bit, through every material
  branch (the NEE structure restated from src/Metropolis.cpp:64-74).
* A multi-sample frame is the float sum of those samples in sample order, scaled
  by 1 / spp: bit-exact as well.
* Against the FP64 estimator at 65536 spp: 16 independent 64-spp frames per pixel
  lie within their Monte-Carlo confidence interval of the FP64 mean.
"""
import os

import numpy as np
import pytest

import oracle
import raysets
import rednoise_b200 as rn
from rednoise_b200 import _native, scenes

pytestmark = pytest.mark.gpu

W, H, DEPTH, RR, SEED = 1920, 1080, 8, 3, 1
FP64_REF = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fp64_ref.npz")


@pytest.fixture(scope="module")
def c2():
    sc = scenes.icosphere_scene(level=8)
    s = rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                             material=sc["material"], material_param=sc["material_param"])
    s.prepare()
    ref = np.load(FP64_REF)
    assert list(ref["c2_spec"][:4]) == [W, H, DEPTH, RR]
    px = ref["c2_pixels"]
    c = scenes.camera(W, H)
    camera = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], W, H)
    yield {"sc": sc, "s": s, "orc": oracle.OrcPhysScene(sc), "px": px, "cam": c, "camera": camera,
           "fp64_mean": ref["c2_mean"], "fp64_var": ref["c2_var"]}
    s.close()


def oracle_samples(d, offsets):
    """Per-sample FP32 radiance of the oracle at the subset pixels: (len(offsets), n, 3)
    float32 (a one-sample sum in double holds the float exactly)."""
    out = [d["orc"].render_sums(d["cam"], 1, DEPTH, RR, seed=SEED, offset=k, pixels=d["px"]) for k in offsets]
    out = np.stack(out)
    assert np.array_equal(out.astype(np.float32).astype(np.float64), out)
    return out.astype(np.float32)


def gpu_frame(d, spp, offset, integrator, **kw):
    st = rn.Settings.make(spp=spp, max_depth=DEPTH, rr_depth=RR, seed=SEED, sample_offset=offset,
                          integrator=integrator)
    return d["s"].render_physical(d["camera"], st, **kw).reshape(-1, 3)[d["px"]]


def report(got, want):
    bad = np.any(got.view(np.uint32) != want.view(np.uint32), axis=-1)
    return int(bad.sum()), bad


@pytest.mark.parametrize("integrator", [_native.RN_PT_MEGAKERNEL, _native.RN_PT_WAVEFRONT])
def test_c2_every_sample_bit_exact(c2, integrator):
    """Four samples of every subset pixel, one frame per sample index: each sample's
    radiance equals the oracle's FP32 radiance bit for bit."""
    want = oracle_samples(c2, range(4))
    assert (want.sum(axis=(1, 2)) > 0).all()
    # the subset's paths reach every material
    mats = c2["sc"]["material"]
    assert len(np.unique(mats)) == 3
    for k in range(4):
        got = gpu_frame(c2, 1, k, integrator)
        n_bad, bad = report(got, want[k])
        assert n_bad == 0, (k, n_bad, np.nonzero(bad)[0][:8], got[bad][:4], want[k][bad][:4])


def test_c2_one_wave_frames_bit_exact(c2):
    """A 4-spp frame through the autotuned integrator (one wave of 8.3M paths on the
    wavefront) and through the megakernel: the float sum of the oracle's samples in
    sample order, times 1/4."""
    want_k = oracle_samples(c2, range(8, 12))
    want = np.zeros_like(want_k[0])
    for k in range(4):
        want = (want + want_k[k]).astype(np.float32)
    want = (want * np.float32(0.25)).astype(np.float32)
    st = rn.Settings.make(spp=4, max_depth=DEPTH, rr_depth=RR, seed=SEED, sample_offset=8)
    tuned = c2["s"].autotune(c2["camera"], st)
    frames = {"auto": gpu_frame(c2, 4, 8, _native.RN_PT_AUTO),
              "wavefront_binned": gpu_frame(c2, 4, 8, _native.RN_PT_WAVEFRONT, ray_sort=True),
              "megakernel": gpu_frame(c2, 4, 8, _native.RN_PT_MEGAKERNEL)}
    for name, got in frames.items():
        n_bad, bad = report(got, want)
        assert n_bad == 0, (name, tuned, n_bad, got[bad][:4], want[bad][:4])


def test_c2_within_confidence_of_fp64(c2):
    """16 independent 64-spp frames (1024 samples per pixel): each subset pixel's mean
    lies within its Monte-Carlo confidence interval of the FP64 65536-spp mean. The
    interval's variance is the frames' sample variance plus the FP64 mean's own;
    |z| > 3.29 (two-sided 0.1 %) may occur at most at 1 % of the 1536 pixel channels
    (heavy-tailed caustic paths make a 16-frame variance estimate short at a few)."""
    frames = np.stack([gpu_frame(c2, 64, 64 * (100 + b), _native.RN_PT_AUTO).astype(np.float64)
                       for b in range(16)])
    mean = frames.mean(0)
    var = frames.var(0, ddof=1) / frames.shape[0]
    z = (mean - c2["fp64_mean"]) / np.sqrt(var + c2["fp64_var"] + 1e-30)
    assert np.mean(np.abs(z) > 3.29) < 0.01, np.sort(np.abs(z).ravel())[-8:]
    assert abs(z.mean()) < 0.15, z.mean()
    # the subset's mean level: within 4 standard errors of the FP64 level
    se = np.sqrt((var + c2["fp64_var"]).sum()) / mean.size
    assert abs(mean.mean() - c2["fp64_mean"].mean()) < 4 * se, (mean.mean(), c2["fp64_mean"].mean(), se)


def test_c2_hits_match_the_reference_bvh(c2):
    """The reference's own BVH (src/BVH.cpp built from its sources, oracle/_ref) over the
    1.31M-triangle scene against the GPU's speculative 4-wide traversal: 60 000 seeded
    rays -- aimed at random points of random triangles (15 % at edges and vertices)
    from inside the room, and secondary rays from their hit points in random
    directions ignoring the hit triangle -- closest-hit index, t, u, v bit for bit,
    and occlusion of shadow rays towards the emitter identical."""
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    sc = c2["sc"]
    v9 = sc["vertices"]
    ref = oracle.RefModel.from_arrays(v9, sc["ref_rgb"], sc["ref_material"], sc["ref_roughness"])
    o1, d1 = raysets.towards_rays(30000, 31, v9, (-2.5, -2.5, -2.5), (2.5, 2.5, 2.5))
    s = c2["s"]
    idx, t, u, v = s.trace_closest(o1, d1)
    ri, rt, ru, rv = ref.intersect(o1, d1)
    assert np.array_equal(idx, ri), np.nonzero(idx != ri)[0][:8]
    assert np.array_equal(t.view(np.uint32), rt.view(np.uint32))
    assert np.array_equal(u.view(np.uint32), ru.view(np.uint32))
    assert np.array_equal(v.view(np.uint32), rv.view(np.uint32))
    hit = idx >= 0
    assert hit.mean() > 0.9
    rng = np.random.default_rng(32)
    p = (o1[hit] + d1[hit] * t[hit, None]).astype(np.float32)
    d2 = rng.normal(size=p.shape).astype(np.float32)
    d2 = scenes.glm_normalize(d2)
    ig = idx[hit].astype(np.int32)
    idx2, t2, _, _ = s.trace_closest(p, d2, ignore=ig)
    ri2, rt2, _, _ = ref.intersect(p, d2, ignore=ig)
    assert np.array_equal(idx2, ri2) and np.array_equal(t2.view(np.uint32), rt2.view(np.uint32))
    # shadow rays to random points of the emitter
    em = np.nonzero(sc["emission"].sum(1) > 0)[0]
    e = v9[rng.choice(em, size=p.shape[0])].reshape(-1, 3, 3).astype(np.float64)
    w = rng.random((p.shape[0], 3))
    w /= w.sum(1, keepdims=True)
    q = (e * w[:, :, None]).sum(1)
    dd = q - p
    dist = np.linalg.norm(dd, axis=1)
    d3 = scenes.glm_normalize(dd.astype(np.float32))
    tmax = (dist * 0.999).astype(np.float32)
    occ = s.trace_any(p, d3, tmax, ignore=ig)
    rocc = ref.occluded(p, d3, tmax, ignore=ig)
    assert np.array_equal(np.asarray(occ).astype(bool), np.asarray(rocc).astype(bool))
    assert 0.05 < np.mean(occ) < 0.95


def test_c2_albedo_gradient_matches_central_differences(c2):
    """The gradient the bench times -- d loss / d albedo over all 1,310,756 x 3 albedos
    of the 1.31M-triangle scene at 512x512, 32 spp, depth 6 -- against central
    differences (eps 1e-3, common random numbers, roulette off so the fixed-sample
    estimator is a polynomial in the albedo) on 16 seeded parameters of the room's
    wall and box triangles, each within 2 %. The sphere's triangles cover a tenth of
    a pixel each at this size, so their differences drown in the float rounding of
    the 786 432-value loss; they are checked against the FP64 oracle's gradient in
    tests/test_adjoint_gpu.py instead."""
    sc = c2["sc"]
    s = c2["s"]
    cam = scenes.camera(512, 512)
    camera = rn.Camera.make(cam["position"], cam["target"], cam["up"], cam["vfov_deg"], 512, 512)
    st = rn.Settings.make(spp=32, max_depth=6, rr_depth=6, seed=3, integrator=_native.RN_PT_MEGAKERNEL)
    room = np.nonzero(sc["emission"][:36].sum(1) == 0)[0]
    rng = np.random.default_rng(0x5EED0004)
    alb_t = sc["albedo"].copy()
    alb_t[room] = np.clip(alb_t[room] + rng.normal(0, 0.1, (room.size, 3)), 0.05, 0.95)
    s.set_materials(albedo=alb_t)
    target = s.render_physical(camera, st).astype(np.float64)
    s.set_materials(albedo=sc["albedo"])

    def loss():
        img = s.render_physical(camera, st).astype(np.float64)
        return ((img - target) ** 2).sum(), 2 * (img - target)

    try:
        L0, dI = loss()
        ga, _ = s.backward([(camera, st)], [dI.astype(np.float32)])
        assert ga.shape == (sc["vertices"].shape[0], 3)
        cand = [(int(t), c) for t in room for c in range(3)]
        pick = np.random.default_rng(16).permutation(len(cand))[:16]
        eps = 1e-3
        errs = []
        for i in pick:
            tri, ch = cand[i]
            alb = sc["albedo"].copy()
            alb[tri, ch] += eps
            s.set_materials(albedo=alb)
            Lp, _ = loss()
            alb[tri, ch] -= 2 * eps
            s.set_materials(albedo=alb)
            Lm, _ = loss()
            fd = (Lp - Lm) / (2 * eps)
            if fd == 0.0:
                assert ga[tri, ch] == 0.0
                continue
            errs.append((abs(fd - ga[tri, ch]) / abs(fd), tri, ch, fd, float(ga[tri, ch])))
        assert len(errs) >= 12
        assert max(errs)[0] < 0.02, sorted(errs)[-3:]
    finally:
        s.set_materials(albedo=sc["albedo"])
