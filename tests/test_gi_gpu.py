"""GPU parity of the bidirectional path tracer and the Metropolis sampler
(renderBidirectional, src/BDPT.cpp:65-144; renderMetropolis, src/Metropolis.cpp:85-192).

Bidirectional, reference stream: the GPU draws every image row from the
reference's own std::mt19937(9871 + y) in the reference's order, so its canvas is
compared with the reference build pixel by pixel (including a frame split into
several column chunks). Counter stream: compared with the oracle's restatement on
the same Philox numbers. Metropolis: the GPU chains are compared with the oracle's
restatement of the same many-chain scheme on the same random numbers (equal up to
last-bit libm differences and the order of the GPU's atomic adds),
and with the reference's own 16-chain sampler statistically.
"""
import os

import numpy as np
import pytest

import oracle
import rednoise_b200 as rn
from imgcheck import agree, argb_to_rgba

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EXACT = dict(min_equal=0.999, max_outlier_frac=0.001)


@pytest.fixture(scope="module")
def assets():
    return np.load(os.path.join(GOLD, "assets_ref.npz"))


def _scene(assets):
    return rn.Scene.from_arrays(assets["cornell_v"], ref_rgb=assets["cornell_rgb"],
                                ref_material=assets["cornell_material"], ref_normal=assets["cornell_normal"],
                                ref_roughness=assets["cornell_roughness"])


def _ref(assets):
    return oracle.RefModel.from_arrays(assets["cornell_v"], assets["cornell_rgb"], assets["cornell_material"],
                                       assets["cornell_roughness"], assets["cornell_normal"])


def _channels(canvas):
    c = np.asarray(canvas, np.uint32)
    return np.stack([(c >> 16) & 255, (c >> 8) & 255, c & 255], -1).astype(np.float64)


@pytest.mark.parametrize("w,h,spp,pos", [(64, 48, 8, (0, 0, 4)), (40, 30, 5, (0.3, 0.2, 3.5))])
def test_bidirectional_reference_stream_matches_reference(assets, w, h, spp, pos):
    want = _ref(assets).render_bidirectional(w, h, spp, pos=pos)
    got = _scene(assets).render_bidirectional(w, h, spp, position=pos)
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_bidirectional_reference_stream_across_column_chunks(assets):
    """320 x 192 at 64 spp needs two column chunks of subpath records (each row's
    stream continues from one chunk into the next)."""
    w, h, spp = 320, 192, 64
    want = _ref(assets).render_bidirectional(w, h, spp)
    got = _scene(assets).render_bidirectional(w, h, spp)
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_bidirectional_counter_stream_matches_oracle(assets):
    w, h, spp = 48, 36, 6
    s = _scene(assets)
    got, rgb = s.render_bidirectional(w, h, spp, rng="counter", seed=7, want_rgb=True)
    orc = oracle.OrcBvh(assets["cornell_v"])
    want, acc = orc.render_bidirectional(assets["cornell_normal"], assets["cornell_rgb"], w, h, spp, stream=1, seed=7,
                                         want_acc=True)
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)
    close = np.isclose(rgb, acc, rtol=1e-5, atol=1e-6).mean()
    assert close > 0.999, close
    # a different seed is a different image; the same seed reproduces
    assert not np.array_equal(s.render_bidirectional(w, h, spp, rng="counter", seed=8), got)
    assert np.array_equal(s.render_bidirectional(w, h, spp, rng="counter", seed=7), got)


def test_metropolis_matches_oracle_chains(assets):
    w, h, muts, chains, boot = 32, 24, 30000, 300, 4000
    s = _scene(assets)
    canvas, rgb, b = s.render_metropolis(w, h, muts, chains=chains, bootstrap=boot, seed=3, want_rgb=True)
    orc = oracle.OrcBvh(assets["cornell_v"])
    want, img, ob = orc.render_metropolis(assets["cornell_normal"], assets["cornell_rgb"], w, h, muts, chains,
                                          bootstrap=boot, seed=3)
    # Same bootstrap paths and summation order; the GPU's cos/sin (double, rounded
    # once) can differ from the host libm's float cosf/sinf in the last bit.
    assert abs(b - ob) <= 1e-7 * ob, (b, ob)
    scale = np.float32(b) * np.float32(w) * np.float32(h) / np.float32(muts)
    dep = rgb / scale
    err = np.abs(dep - img) / np.maximum(np.abs(img), 1e-3)
    assert (err < 1e-4).mean() > 0.995, (err < 1e-4).mean()
    assert abs(dep.sum() - img.sum()) < 1e-4 * img.sum()
    agree(argb_to_rgba(canvas), argb_to_rgba(want), min_equal=0.99, max_outlier_frac=0.005)


def test_metropolis_estimates_the_reference_image(assets):
    w, h, muts = 32, 24, 400000
    m = _ref(assets)
    want = _channels(m.render_metropolis(w, h, muts))
    want4 = _channels(m.render_metropolis(w, h, 4 * muts))
    got = _channels(_scene(assets).render_metropolis(w, h, muts, seed=1))
    assert abs(got.mean() - want4.mean()) < 0.015 * want4.mean()
    spread = np.abs(want - want4).mean()
    assert np.abs(got - want4).mean() < 2.0 * spread + 1.0


def test_bidirectional_counter_stream_converges_to_reference(assets):
    w, h = 32, 24
    want = _channels(_ref(assets).render_bidirectional(w, h, 256))
    got = _channels(_scene(assets).render_bidirectional(w, h, 256, rng="counter", seed=2))
    assert abs(got.mean() - want.mean()) < 0.005 * want.mean()
    assert np.abs(got - want).mean() < 2.0


def test_gi_invalid_arguments(assets):
    s = _scene(assets)
    with pytest.raises(rn.RnError):
        s.render_bidirectional(16, 16, 0)
    with pytest.raises(ValueError):
        s.render_bidirectional(16, 16, 4, rng="sobol")
    with pytest.raises(rn.RnError):
        s.render_metropolis(16, 16, 0)
    with pytest.raises(rn.RnError):
        s.render_metropolis(16, 16, 100, chains=200)
    with pytest.raises(rn.RnError):
        s.render_metropolis(16, 16, 1000, bootstrap=0)


def test_metropolis_black_scene_leaves_cleared_canvas():
    """No surface sees the emitter: b = 0, and the reference returns its cleared canvas."""
    v = np.array([[-1, -2, -1, 1, -2, -1, 0, -2, 1]], np.float32)  # one triangle below the camera's view
    s = rn.Scene.from_arrays(v, ref_rgb=np.array([[200, 200, 200]], np.int32))
    canvas, rgb, b = s.render_metropolis(16, 12, 2000, bootstrap=500, want_rgb=True)
    assert b == 0.0 and not canvas.any() and not rgb.any()
