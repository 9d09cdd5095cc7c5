"""CPU tests of the product library's host side (no GPU calls)."""
import ctypes
import os
import re
import struct
import zlib

import numpy as np
import pytest

import oracle
import objio
import raysets
import rednoise_b200 as rn
from rednoise_b200 import _native, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
REF_ASSETS = os.path.join(oracle.reference_dir() or "", "assets")


def declared_functions():
    names = []
    for h in ("rednoise.h", "rednoise_pt.h"):
        src = open(os.path.join(ROOT, "include", "rednoise", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(rn_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = declared_functions()
    assert "rn_render" in names and "rn_pt_trace_closest" in names
    for n in names:
        assert hasattr(lib, n), n
    # the ctypes table covers the whole header
    assert set(names) <= set(_native.SIGNATURES), set(names) - set(_native.SIGNATURES)


def test_version_matches_reference():
    assert rn.version() == "0.1.2"


def test_invalid_arguments_without_gpu(tmp_path):
    lib = _native.load()
    buf = ctypes.create_string_buffer(16)
    assert lib.rn_render(None, 3, 2, 2, 4.0, 1, buf) == 0
    assert lib.rn_scene_load_obj(None, 1.0) is None
    assert lib.rn_scene_load_obj(os.fsencode(str(tmp_path / "missing.obj")), 1.0) is None
    assert lib.rn_scene_triangle_count(None) == 0
    lib.rn_scene_free(None)
    out = ctypes.c_void_p()
    assert lib.rn_pt_scene_create(None, ctypes.byref(out)) == 1
    with pytest.raises(rn.RnError):
        rn.Scene.from_arrays(np.full((1, 9), np.nan, np.float32))
    with pytest.raises(rn.RnError):
        rn.Scene.from_arrays(np.zeros((1, 9), np.float32), material=[7])
    # a face that references a missing vertex is rejected instead of read out of bounds
    p = tmp_path / "bad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nf 1/ 2/ 3/\n")
    assert lib.rn_scene_load_obj(os.fsencode(str(p)), 1.0) is None
    assert b"vertex" in lib.rn_pt_last_error()
    p.write_text("v 0 0 0\nf x y z\n")
    assert lib.rn_scene_load_obj(os.fsencode(str(p)), 1.0) is None


def test_png_writer_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, size=(37, 53, 4), dtype=np.uint8)
    path = tmp_path / "x.png"
    assert _native.load().rn_save_png(os.fsencode(str(path)), 53, 37, img.ctypes.data) == 1
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, hdr = 8, b"", None
    while pos < len(data):
        (ln,) = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + ln]
        assert struct.unpack(">I", data[pos + 8 + ln:pos + 12 + ln])[0] == zlib.crc32(typ + body)
        if typ == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        if typ == b"IDAT":
            idat += body
        pos += 12 + ln
    assert hdr[:4] == (53, 37, 8, 6)
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(37, 53 * 4 + 1)
    assert (raw[:, 0] == 0).all()
    assert np.array_equal(raw[:, 1:].reshape(37, 53, 4), img)


def _assets():
    return np.load(os.path.join(GOLD, "assets_ref.npz"))


@pytest.mark.parametrize("name", ["cornell", "sphere"])
def test_obj_loader_matches_reference_loader(name, tmp_path):
    """OBJ/MTL loader semantics (src/ObjLoader.cpp:23-214) against the reference's loaded arrays."""
    a = _assets()
    v9, rgb, mat, nrm = a[f"{name}_v"], a[f"{name}_rgb"], a[f"{name}_material"], a[f"{name}_normal"]
    path = objio.write_obj(str(tmp_path), name, v9, rgb, mat)
    s = rn.Scene.load_obj(path, 1.0)
    t = s.triangles()
    assert np.array_equal(t["vertices"].view(np.uint32), v9.view(np.uint32))
    assert np.array_equal(t["ref_rgb"], rgb)
    assert np.array_equal(t["ref_material"], mat)
    assert np.array_equal(t["normal"].view(np.uint32), nrm.view(np.uint32))


@pytest.mark.skipif(not os.path.isdir(REF_ASSETS), reason="reference assets absent")
@pytest.mark.parametrize("fname", ["cornell-box.obj", "sphere.obj", "terrain.obj"])
def test_obj_loader_on_reference_assets(fname):
    path = os.path.join(REF_ASSETS, fname)
    m = oracle.RefModel.from_obj(path, 0.35)
    r = m.arrays()
    s = rn.Scene.load_obj(path, 0.35)
    t = s.triangles()
    assert s.triangle_count == m.count
    assert np.array_equal(t["vertices"].view(np.uint32), r["v"].view(np.uint32))
    assert np.array_equal(t["ref_rgb"], r["rgb"])
    assert np.array_equal(t["ref_material"], r["material"])
    assert np.array_equal(t["normal"].view(np.uint32), r["normal"].view(np.uint32))


def _tree_equal(scene_arrays_v9):
    s = rn.Scene.from_arrays(scene_arrays_v9)
    got = s.bvh()
    want = oracle.OrcBvh(scene_arrays_v9).dump()
    assert np.array_equal(got["order"], want["order"])
    assert np.array_equal(got["bounds"].view(np.uint32), want["bounds"].view(np.uint32))
    assert np.array_equal(got["links"], want["links"])
    if oracle.ref_available():
        r = oracle.RefModel.from_arrays(scene_arrays_v9).dump_bvh()
        assert np.array_equal(got["order"], r["order"])
        assert np.array_equal(got["links"], r["links"])


@pytest.mark.parametrize("kind", ["cornell", "sphere", "box", "soup", "tiny", "dups", "threaded"])
def test_host_bvh_equals_reference_tree(kind):
    """The product's host build yields the reference's exact tree (src/BVH.cpp:6-63);
    "threaded" is large enough for the build to split subtrees across threads."""
    a = _assets()
    if kind in ("cornell", "sphere"):
        v9 = a[f"{kind}_v"]
    elif kind == "box":
        v9 = scenes.cornell_box()["vertices"]
    elif kind == "soup":
        v9 = scenes.soup_scene(5000, seed=3)["vertices"]
    elif kind == "threaded":
        v9 = scenes.soup_scene(300000, seed=4)["vertices"]
    elif kind == "tiny":
        v9 = a["cornell_v"][:3]
    else:
        v9 = np.repeat(a["cornell_v"][:2], 9, axis=0)
    _tree_equal(v9)


def test_icosphere_generator_shape():
    s = scenes.icosphere(3)
    assert s.shape == (20 * 4 ** 3, 3, 3)
    r = np.linalg.norm(s.reshape(-1, 3), axis=1)
    assert np.allclose(r, 1.0)
    box = scenes.cornell_box()
    assert box["vertices"].shape == (36, 9)
    assert (box["emission"].max(axis=1) > 0).sum() == 2


def test_workload_generators_are_seeded_and_in_range():
    from rednoise_b200 import scenes

    a, b = scenes.batch_jobs(), scenes.batch_jobs()
    assert a == b and len(a) == 64
    for j in a:
        assert 1000 <= j["triangles"] <= 500000
        assert (j["width"], j["height"]) in ((256, 256), (512, 384), (1024, 768))
        assert 4 <= j["spp"] <= 64 and j["max_depth"] == 6
    v = scenes.views()
    assert v == scenes.views() and len(v) == 16
    for c in v:
        assert -1.5 <= c["position"][0] <= 1.5 and 2.0 <= c["position"][2] <= 2.6
        assert -2.0 <= c["target"][2] <= -1.0 and c["width"] == c["height"] == 384


@pytest.mark.parametrize("name", ["sphere", "cornell", "icosphere", "box"])
def test_loader_vertex_normals_match_reference_loader(name, tmp_path):
    """Per-corner smoothed normals (src/ObjLoader.cpp:178-204) equal the reference
    loader's bit for bit on OBJ files whose faces share vertices."""
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    a = _assets()
    if name in ("sphere", "cornell"):
        v9, rgb, mat = a[f"{name}_v"], a[f"{name}_rgb"], a[f"{name}_material"]
    elif name == "icosphere":
        v9 = scenes.icosphere(2).reshape(-1, 9).astype(np.float32)
        rgb, mat = np.full((v9.shape[0], 3), 200, np.int32), np.zeros(v9.shape[0], np.int32)
    else:
        sc = scenes.cornell_box()
        v9, rgb, mat = sc["vertices"], sc["ref_rgb"], sc["ref_material"]
    path = objio.write_obj(str(tmp_path), name, v9, rgb, mat, share_vertices=True)
    got = rn.Scene.load_obj(path, 1.0).vertex_normals()
    m = oracle.RefModel.from_obj(path, 1.0)
    want = m.vertex_normals()
    m.close()
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    if name in ("sphere", "icosphere"):  # smoothing happened somewhere
        face = np.repeat(rn.Scene.load_obj(path, 1.0).triangles()["normal"], 3, axis=0).reshape(-1, 9)
        assert not np.array_equal(got, face)
