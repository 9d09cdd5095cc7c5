"""GPU parity of the photon mapper (renderPhotonMapped, src/Renderer.cpp:1177-1349).

The reference draws every photon from one std::mt19937(777) stream, one photon
after the other; the GPU resolves each photon's start in that stream in parallel
(every candidate start traced, the chain resolved by pointer doubling), stores the
photons at the reference's indices and gathers them in the reference's order, so
the images are compared with the reference build pixel by pixel.
"""
import os

import numpy as np
import pytest

import oracle
import rednoise_b200 as rn
from imgcheck import agree, argb_to_rgba, light_records

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EXACT = dict(min_equal=0.999, max_outlier_frac=0.001)


@pytest.fixture(scope="module")
def assets():
    return np.load(os.path.join(GOLD, "assets_ref.npz"))


def _pair(assets, material=None):
    v9 = assets["cornell_v"]
    mat = assets["cornell_material"] if material is None else material
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], mat, assets["cornell_roughness"],
                                    assets["cornell_normal"])
    s = rn.Scene.from_arrays(v9, ref_rgb=assets["cornell_rgb"], ref_material=mat,
                             ref_normal=assets["cornell_normal"], ref_roughness=assets["cornell_roughness"])
    return m, s


@pytest.mark.parametrize("photons", [2000, 50000])
def test_photon_map_matches_reference(assets, photons):
    """The asset's mirror and glass boxes: reflected and refracted photons (caustics)."""
    m, s = _pair(assets)
    want = m.render_photon_mapped(64, 48, photons)
    got, stored = s.render_photon_mapped(64, 48, photons, return_count=True)
    m.close()
    assert stored > photons // 4
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_metal_and_lights_match_reference(assets):
    mat = assets["cornell_material"].copy()
    mat[[4, 5]] = 6  # metal back wall
    m, s = _pair(assets, mat)
    lights = [rn.Light.default(position=(0.2, 0.8, 0.1), intensity=30.0),
              rn.Light.default(type=1, direction=(0.3, -1.0, -0.4), intensity=20.0)]
    want = m.render_photon_mapped(48, 36, 20000, lights=light_records(lights), pos=(0.3, 0.2, 3.5))
    got = s.render_photon_mapped(48, 36, 20000, lights=lights, position=(0.3, 0.2, 3.5))
    m.close()
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_final_gather_matches_reference(assets):
    """gather_rays > 0: every row draws its gather directions from its own stream."""
    m, s = _pair(assets)
    want = m.render_photon_mapped(32, 24, 10000, gather_rays=3)
    got = s.render_photon_mapped(32, 24, 10000, gather_rays=3)
    m.close()
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_photon_arguments_rejected(assets):
    s = rn.Scene.from_arrays(assets["cornell_v"])
    with pytest.raises(rn.RnError):
        s.render_photon_mapped(8, 8, 0)
    with pytest.raises(rn.RnError):
        s.render_photon_mapped(8, 8, 100, gather_rays=-1)
