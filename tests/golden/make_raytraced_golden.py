"""Golden canvases of the reference's Whitted ray tracer (rn_render(RN_RAYTRACED)).

Run where the reference build exists (``make -C oracle``):
    python tests/golden/make_raytraced_golden.py

Writes raytraced_ref.npz: the reference's RGBA8 output of rn_render(RN_RAYTRACED)
through its C ABI, for the Cornell-box and sphere assets (arrays in
assets_ref.npz) written as OBJ files whose faces share vertices, so the loader's
vertex-normal smoothing is exercised. Keys: <asset>_<w>x<h>.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import objio  # noqa: E402
import oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = (("cornell", 96, 72), ("cornell", 64, 48), ("sphere", 80, 60))


def main() -> None:
    a = np.load(os.path.join(HERE, "assets_ref.npz"))
    lib = oracle.ref()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, w, h in CASES:
            path = objio.write_obj(d, name, a[f"{name}_v"], a[f"{name}_rgb"], a[f"{name}_material"],
                                   share_vertices=True)
            sc = lib.rn_scene_load_obj(os.fsencode(path), 1.0)
            buf = np.zeros((h, w, 4), np.uint8)
            assert lib.rn_render(sc, 2, w, h, 4.0, 1, oracle.P(buf)) == 1
            lib.rn_scene_free(sc)
            out[f"{name}_{w}x{h}"] = buf
    np.savez_compressed(os.path.join(HERE, "raytraced_ref.npz"), **out)
    print("raytraced_ref.npz", os.path.getsize(os.path.join(HERE, "raytraced_ref.npz")), "bytes")


if __name__ == "__main__":
    main()
