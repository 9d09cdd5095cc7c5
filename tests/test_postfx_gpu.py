"""GPU parity of the canvas post-processing with the reference's toneMap,
applyBloom, applyFXAA and AccumBuffer (src/Renderer.cpp:1353-1470): identical
pixels (the tone map's pow is the only libm call; one differing pixel in ten
thousand is allowed for a last-bit difference at a truncation boundary)."""
import numpy as np
import pytest

import oracle
from rednoise_b200 import postfx

pytestmark = pytest.mark.gpu


def _canvas(seed, h=61, w=83):
    rng = np.random.default_rng(seed)
    rgb = rng.integers(0, 256, (h, w, 3)).astype(np.uint32)
    # smooth regions, hard edges and bright spots
    rgb[10:30, 5:40] = (250, 240, 230)
    rgb[35:60, 50:80] = (12, 20, 30)
    rgb[:, 41] = 255
    return (255 << 24) | (rgb[..., 0] << 16) | (rgb[..., 1] << 8) | rgb[..., 2]


def _same(a, b, frac=1e-4):
    diff = (a != b).mean()
    assert diff <= frac, f"{diff:.5f} of pixels differ"


@pytest.mark.parametrize("args", [(1.0, 2.2), (2.5, 1.8), (0.4, 2.4)])
def test_tonemap_matches_reference(args):
    c = _canvas(1)
    _same(postfx.tonemap(c, *args), oracle.ref_postfx("tonemap", c, *args))


@pytest.mark.parametrize("args", [(0.75, 0.7), (0.3, 1.5)])
def test_bloom_matches_reference(args):
    c = _canvas(2)
    _same(postfx.bloom(c, *args), oracle.ref_postfx("bloom", c, *args))


def test_fxaa_matches_reference():
    c = _canvas(3)
    got = postfx.fxaa(c)
    _same(got, oracle.ref_postfx("fxaa", c))
    assert (got[0] == c[0]).all() and (got[:, -1] == c[:, -1]).all()  # borders untouched


def test_accum_buffer_matches_reference():
    frames = np.stack([_canvas(10 + k) for k in range(5)])
    acc = postfx.AccumBuffer(frames.shape[2], frames.shape[1])
    for f in frames:
        acc.add(f)
    _same(acc.resolve(), oracle.ref_accum(frames))
