"""GPU parity of the Whitted ray tracer (rn_render(RN_RAYTRACED), renderRaytraced).

The renderer is deterministic, so images are compared pixel by pixel with the
reference's own output: the committed golden canvases, and the reference build
(oracle/_ref) called live for materials, shading models, light types and fog.
The bar is >= 99.9 % of channel values identical and at most 0.1 % off by more
than 2 (a last-bit difference of pow/exp can move a specular highlight or a
Fresnel weight by one step of the 8-bit output).
"""
import os

import numpy as np
import pytest

import objio
import oracle
import rednoise_b200 as rn
from imgcheck import agree, argb_to_rgba, light_records
from rednoise_b200 import _native, scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EXACT = dict(min_equal=0.999, max_outlier_frac=0.001)


@pytest.fixture(scope="module")
def assets():
    return np.load(os.path.join(GOLD, "assets_ref.npz"))


@pytest.mark.parametrize("key", ["cornell_96x72", "cornell_64x48", "sphere_80x60"])
def test_rn_render_raytraced_matches_reference_golden(assets, key, tmp_path):
    gold = np.load(os.path.join(GOLD, "raytraced_ref.npz"))[key]
    name, size = key.split("_")
    w, h = (int(x) for x in size.split("x"))
    path = objio.write_obj(str(tmp_path), name, assets[f"{name}_v"], assets[f"{name}_rgb"],
                           assets[f"{name}_material"], share_vertices=True)
    s = rn.Scene.load_obj(path, 1.0)
    got = s.render("raytraced", w, h, 4.0, 1).to_numpy()
    assert (got[..., 3] == 255).all()
    agree(got, gold, **EXACT)


def _material_scene(assets, tmp_path):
    """The Cornell asset with every reference material on some triangles, and
    smoothed vertex normals (from loading it as an indexed OBJ)."""
    v9 = assets["cornell_v"]
    rgb = assets["cornell_rgb"].copy()
    mat = assets["cornell_material"].copy()
    n = v9.shape[0]
    cycle = [1, 2, 3, 4, 5, 6, 7, 8, 9, 0]
    for i in range(2, n):
        mat[i] = cycle[(i // 2) % len(cycle)]
    mat[[0, 1]] = 10
    rgb[[0, 1]] = (255, 240, 200)
    path = objio.write_obj(str(tmp_path), "cornell", v9, assets["cornell_rgb"], assets["cornell_material"],
                           share_vertices=True)
    vn = rn.Scene.load_obj(path, 1.0).vertex_normals()
    return v9, rgb, mat, vn


def _pair(assets, v9, rgb, mat, vn):
    m = oracle.RefModel.from_arrays(v9, rgb, mat, assets["cornell_roughness"], assets["cornell_normal"])
    m.set_vertex_normals(vn)
    s = rn.Scene.from_arrays(v9, ref_rgb=rgb, ref_material=mat, ref_normal=assets["cornell_normal"],
                             ref_roughness=assets["cornell_roughness"], ref_vertex_normals=vn)
    return m, s


@pytest.mark.parametrize("shading", [0, 1, 2])
def test_materials_and_shading_models_match_reference(assets, shading, tmp_path):
    """Mirror, glass, dispersive, metal, emissive, procedural and bump surfaces
    under flat, Gouraud and Phong shading, against the reference build."""
    v9, rgb, mat, vn = _material_scene(assets, tmp_path)
    m, s = _pair(assets, v9, rgb, mat, vn)
    w, h = 80, 60
    want = m.render_raytraced(w, h, shading=shading)
    got = s.render_raytraced(w, h, shading=shading)
    m.close()
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


LIGHT_CASES = {
    "point_hard": [dict(type=0, radius=0.0)],
    "rect": [dict(type=4, position=(0.0, 0.9, 0.0))],
    "triangle": [dict(type=5, position=(-0.3, 0.9, -0.3), u_axis=(0.6, 0, 0), v_axis=(0, 0, 0.6))],
    "volume": [dict(type=3, radius=0.2, position=(0.1, 0.6, 0.2))],
    "spot_dir": [dict(type=2, radius=0.1, direction=(0.0, -1.0, 0.1)),
                 dict(type=1, direction=(0.3, -1.0, -0.4), intensity=20.0)],
}


@pytest.mark.parametrize("case", sorted(LIGHT_CASES))
def test_light_types_and_depth_match_reference(assets, case, tmp_path):
    v9, rgb, mat, vn = _material_scene(assets, tmp_path)
    m, s = _pair(assets, v9, rgb, mat, vn)
    lights = [rn.Light.default(**kw) for kw in LIGHT_CASES[case]]
    w, h = 64, 48
    want = m.render_raytraced(w, h, lights=light_records(lights))
    got = s.render_raytraced(w, h, lights=lights)
    m.close()
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_fog_and_camera_match_reference(assets, tmp_path):
    v9, rgb, mat, vn = _material_scene(assets, tmp_path)
    m, s = _pair(assets, v9, rgb, mat, vn)
    kw = dict(focal=1.2, pos=(0.6, 0.3, 3.0), target=(0.0, -0.1, 0.0))
    want = m.render_raytraced(72, 54, fog_density=0.25, fog_colour=(180.0, 190.0, 220.0), **kw)
    got = s.render_raytraced(72, 54, focal_length=1.2, position=(0.6, 0.3, 3.0), target=(0.0, -0.1, 0.0),
                             fog_density=0.25, fog_colour=(180.0, 190.0, 220.0))
    m.close()
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_large_mesh_matches_reference():
    """The 20k-triangle displaced icosphere inside the box (4-wide traversal on a real tree)."""
    sc = scenes.icosphere_scene(level=5)
    v9 = sc["vertices"]
    mat = sc["ref_material"]
    m = oracle.RefModel.from_arrays(v9, sc["ref_rgb"], mat, sc["ref_roughness"])
    s = rn.Scene.from_arrays(v9, ref_rgb=sc["ref_rgb"], ref_material=mat, ref_roughness=sc["ref_roughness"])
    pos = (0.0, 0.0, scenes.CAMERA_Z)
    want = m.render_raytraced(96, 64, focal=1.0, pos=pos)
    got = s.render_raytraced(96, 64, focal_length=1.0, position=pos)
    m.close()
    agree(argb_to_rgba(got), argb_to_rgba(want), **EXACT)


def test_invalid_arguments_rejected(assets):
    s = rn.Scene.from_arrays(assets["cornell_v"])
    with pytest.raises(rn.RnError):
        s.render_raytraced(16, 16, shading=3)
    with pytest.raises(rn.RnError):
        s.render_raytraced(16, 16, max_depth=9)
    assert _native.RN_PT_SHADING_PHONG == 2
