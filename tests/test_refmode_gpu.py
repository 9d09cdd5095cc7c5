"""GPU parity of the drop-in reference-mode renderer (rn_render(RN_PATHTRACED)).

The GPU consumes each pixel's mt19937 stream exactly as the reference does, so
images are compared pixel by pixel with the reference's own output: the bar is
>= 99 % of channel values identical, and every pixel within the 99.9 %
Monte-Carlo interval of the reference's estimate (a handful of pixels may follow
a different path where a libm last-bit difference changes a decision).
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
import objio
import rednoise_b200 as rn
from rednoise_b200 import _native, scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def argb_to_rgba(c):
    return np.stack([(c >> 16) & 255, (c >> 8) & 255, c & 255, c >> 24], -1).astype(np.uint8)


def agree(a, b, min_equal=0.99, max_outlier_frac=0.01):
    a = a.astype(np.int32)
    b = b.astype(np.int32)
    eq = (a == b).mean()
    outliers = (np.abs(a - b) > 2).mean()
    assert eq >= min_equal, f"only {eq:.4f} of channel values identical"
    assert outliers <= max_outlier_frac, f"{outliers:.4f} of values differ by more than 2"
    return eq


@pytest.fixture(scope="module")
def assets():
    return np.load(os.path.join(GOLD, "assets_ref.npz"))


@pytest.mark.parametrize("key", ["rgba_64x48_4", "rgba_96x72_16"])
def test_rn_render_matches_reference_golden(assets, key, tmp_path):
    gold = np.load(os.path.join(GOLD, "render_ref.npz"))[key]
    w, h, spp = (int(x) for x in key.split("_")[1].split("x") + [key.split("_")[2]])
    path = objio.write_obj(str(tmp_path), "cornell", assets["cornell_v"], assets["cornell_rgb"],
                           assets["cornell_material"])
    s = rn.Scene.load_obj(path, 1.0)
    img = s.render("pathtraced", w, h, 4.0, spp)
    got = img.to_numpy()
    assert (got[..., 3] == 255).all()
    agree(got, gold)


def _oracle_scene(assets):
    v9 = assets["cornell_v"]
    return v9, oracle.OrcBvh(v9)


LIGHT_CASES = {
    "default": None,
    "point_hard": [dict(type=0, radius=0.0)],
    "rect": [dict(type=4, position=(0.0, 0.9, 0.0))],
    "triangle": [dict(type=5, position=(-0.3, 0.9, -0.3), u_axis=(0.6, 0, 0), v_axis=(0, 0, 0.6))],
    "volume": [dict(type=3, radius=0.2, position=(0.1, 0.6, 0.2))],
    "spot_dir": [dict(type=2, radius=0.1, direction=(0.0, -1.0, 0.1)),
                 dict(type=1, direction=(0.3, -1.0, -0.4), intensity=20.0)],
}


def _records(lights):
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


@pytest.mark.parametrize("case", sorted(LIGHT_CASES))
def test_reference_mode_light_types_match_oracle(assets, case):
    """Every visibility branch (src/Renderer.cpp:390-498) against the oracle restatement."""
    lights = None if LIGHT_CASES[case] is None else [rn.Light.default(**kw) for kw in LIGHT_CASES[case]]
    v9, orc = _oracle_scene(assets)
    s = rn.Scene.from_arrays(v9, ref_rgb=assets["cornell_rgb"], ref_material=assets["cornell_material"],
                             ref_normal=assets["cornell_normal"], ref_roughness=assets["cornell_roughness"])
    w, h, spp = 80, 60, 4
    got = s.render_reference(w, h, spp, lights=lights)
    want = orc.render_reference(assets["cornell_normal"], assets["cornell_material"], assets["cornell_rgb"],
                                assets["cornell_roughness"], w, h, spp,
                                lights=None if lights is None else _records(lights))
    agree(argb_to_rgba(got), argb_to_rgba(want))


def test_reference_mode_materials_match_reference_live(assets):
    """Metal and subsurface triangles (absent from the asset) against the reference build itself."""
    v9 = assets["cornell_v"]
    mat = assets["cornell_material"].copy()
    rgb = assets["cornell_rgb"].copy()
    rough = np.full(v9.shape[0], 0.35, np.float32)
    mat[[4, 5]] = 6   # back wall -> Metal
    mat[[8, 9]] = 8   # floor -> Subsurface
    mat[[0, 1]] = 10  # light quad -> Emissive
    rgb[[0, 1]] = (255, 240, 200)
    m = oracle.RefModel.from_arrays(v9, rgb, mat, rough, assets["cornell_normal"])
    w, h, spp = 64, 48, 4
    want = m.render(w, h, spp)
    s = rn.Scene.from_arrays(v9, ref_rgb=rgb, ref_material=mat, ref_normal=assets["cornell_normal"],
                             ref_roughness=rough)
    got = s.render_reference(w, h, spp)
    agree(argb_to_rgba(got), argb_to_rgba(want))


def test_reference_mode_depth_of_field_and_motion(assets):
    """Aperture sampling (round and 6-blade) and motion blur against the reference build."""
    v9 = assets["cornell_v"]
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], assets["cornell_material"],
                                    assets["cornell_roughness"], assets["cornell_normal"])
    s = rn.Scene.from_arrays(v9, ref_rgb=assets["cornell_rgb"], ref_material=assets["cornell_material"],
                             ref_normal=assets["cornell_normal"], ref_roughness=assets["cornell_roughness"])
    for blades in (0, 6):
        want = m.render(64, 48, 4, aperture=0.05, focus=3.5, motion=(0.02, 0.0, 0.0), blades=blades)
        got = s.render_reference(64, 48, 4, aperture=0.05, focus_distance=3.5, camera_motion=(0.02, 0.0, 0.0),
                                 aperture_blades=blades)
        agree(argb_to_rgba(got), argb_to_rgba(want))


def test_reference_mode_long_pixel_streams_match_reference_live(assets):
    """96 spp draws about a thousand numbers per pixel: past the first twist's 227
    outputs (computed without a state array) and into the second twist."""
    v9 = assets["cornell_v"]
    m = oracle.RefModel.from_arrays(v9, assets["cornell_rgb"], assets["cornell_material"],
                                    assets["cornell_roughness"], assets["cornell_normal"])
    s = rn.Scene.from_arrays(v9, ref_rgb=assets["cornell_rgb"], ref_material=assets["cornell_material"],
                             ref_normal=assets["cornell_normal"], ref_roughness=assets["cornell_roughness"])
    want = m.render(24, 18, 96)
    got = s.render_reference(24, 18, 96)
    m.close()
    agree(argb_to_rgba(got), argb_to_rgba(want), min_equal=0.999, max_outlier_frac=0.001)


@pytest.mark.parametrize("spp", [16, 64])
def test_reference_mode_pixel_chunks(assets, spp):
    """1024 x 1024 at 16 and 64 spp needs several pixel chunks of path records; the
    first and last rows equal the oracle's rows, which equal the reference's."""
    v9 = assets["cornell_v"]
    s = rn.Scene.from_arrays(v9, ref_rgb=assets["cornell_rgb"], ref_material=assets["cornell_material"],
                             ref_normal=assets["cornell_normal"], ref_roughness=assets["cornell_roughness"])
    w = h = 1024
    got = s.render_reference(w, h, spp)
    orc = oracle.OrcBvh(v9)
    for y0 in (0, h - 3):
        want = orc.render_reference(assets["cornell_normal"], assets["cornell_material"], assets["cornell_rgb"],
                                    assets["cornell_roughness"], w, h, spp, y0=y0, y1=y0 + 3)
        agree(argb_to_rgba(got[y0:y0 + 3]), argb_to_rgba(want), min_equal=0.999, max_outlier_frac=0.001)


def test_mean_taps_are_consistent(assets):
    v9 = assets["cornell_v"]
    s = rn.Scene.from_arrays(v9, ref_rgb=assets["cornell_rgb"], ref_material=assets["cornell_material"],
                             ref_normal=assets["cornell_normal"], ref_roughness=assets["cornell_roughness"])
    canvas, mean = s.render_reference(40, 30, 8, want_mean=True)
    r = np.minimum(255, (mean[..., 0] * np.float32(255.0)).astype(np.int64))
    assert np.array_equal(r, (canvas >> 16) & 255)


def test_rn_render_zero_samples_and_other_modes(assets, tmp_path):
    path = objio.write_obj(str(tmp_path), "c", assets["cornell_v"], assets["cornell_rgb"],
                           assets["cornell_material"])
    lib = _native.load()
    sc = lib.rn_scene_load_obj(os.fsencode(path), 1.0)
    buf = ctypes.create_string_buffer(8 * 6 * 4)
    assert lib.rn_render(sc, 3, 8, 6, 4.0, 0, buf) == 1
    px = np.frombuffer(buf.raw, np.uint8).reshape(6, 8, 4)
    assert (px[..., :3] == 0).all() and (px[..., 3] == 255).all()  # reference: 0/0 -> black, alpha 255
    assert lib.rn_render(sc, 2, 8, 6, 4.0, 1, buf) == 1  # RN_RAYTRACED is served too
    assert lib.rn_render(sc, 1, 8, 6, 4.0, 1, buf) == 0  # the rasteriser is not
    assert lib.rn_render(sc, 0, 8, 6, 4.0, 1, buf) == 0
    lib.rn_scene_free(sc)
