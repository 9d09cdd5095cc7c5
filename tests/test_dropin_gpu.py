"""Drop-in use through the reference's own, unchanged C consumer (GPU part).

oracle/_ref/c_consumer is the reference's examples/c_consumer.c, unchanged,
compiled by oracle/Makefile against this repository's include/rednoise/rednoise.h
and linked to librednoise_b200.so (built where the reference tree is present; the
binary travels with the build). It loads an OBJ at scale 0.35, prints the version
and triangle count, renders 320x240 with rn_render(RN_RAYTRACED, cam_z 4, 8
samples) and writes a PPM. The test gives it the reference's Cornell box (the
committed fixture written back as OBJ + MTL) and compares its image with the
reference library's own rn_render of the same file (oracle/_ref/librn_ref.so):
at least 99.9 % of channel values identical, at most 0.1 % off by more than 2,
the bar of the Whitted parity tests.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import objio
import oracle
from imgcheck import agree

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CONSUMER = os.path.join(ROOT, "oracle", "_ref", "c_consumer")
GOLD = os.path.join(ROOT, "tests", "golden")


def read_ppm(path):
    with open(path, "rb") as f:
        data = f.read()
    head = data.split(b"\n", 3)
    assert head[0] == b"P6"
    w, h = (int(x) for x in head[1].split())
    assert head[2] == b"255"
    return np.frombuffer(head[3], np.uint8).reshape(h, w, 3)


@pytest.mark.skipif(not os.path.isfile(CONSUMER) or not oracle.ref_available(),
                    reason="c_consumer / reference build absent")
def test_reference_c_consumer_renders_through_this_library(tmp_path):
    a = np.load(os.path.join(GOLD, "assets_ref.npz"))
    v9 = (a["cornell_v"].astype(np.float64) / 0.35).astype(np.float32)
    obj = objio.write_obj(str(tmp_path), "cornell-box", v9, a["cornell_rgb"], a["cornell_material"],
                          share_vertices=True)
    out = str(tmp_path / "capi.ppm")
    env = dict(os.environ)
    env.pop("RN_B200_LIBRARY", None)
    p = subprocess.run([CONSUMER, obj, out], cwd=str(tmp_path), capture_output=True, text=True, timeout=300,
                       env=env)
    assert p.returncode == 0, p.stderr
    assert "rednoise 0.1.2" in p.stdout and "loaded 32 triangles" in p.stdout and "wrote" in p.stdout
    got = read_ppm(out)
    assert got.shape == (240, 320, 3)

    ref = oracle.ref()
    sc = ref.rn_scene_load_obj(obj.encode(), ctypes.c_float(0.35))
    assert sc
    want = np.zeros((240, 320, 4), np.uint8)
    assert ref.rn_render(sc, 2, 320, 240, ctypes.c_float(4.0), 8, oracle.P(want)) == 1
    ref.rn_scene_free(sc)
    assert want[..., :3].mean() > 10
    agree(got, want[..., :3], min_equal=0.999, max_outlier_frac=0.001)
