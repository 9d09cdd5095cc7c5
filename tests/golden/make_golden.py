"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run in a container that has the reference tree and its build
(``make -C oracle``):  python tests/golden/make_golden.py [reference_dir]

Writes:
  assets_ref.npz   triangle arrays produced by the reference's loadOBJ for
                   assets/cornell-box.obj (scale 0.35) and assets/sphere.obj
                   (scale 0.35): vertices, Colour, Material, face normal, roughness
  trace_ref.npz    seeded ray sets with the reference BVH::intersect / occluded
                   results (triangle index, t/u/v bits, occlusion) on those
                   meshes and on the 36-triangle Cornell box of rednoise_b200.scenes
  render_ref.npz   reference renderPathTraced canvases (0xAARRGGBB) of the
                   loaded cornell-box.obj through the C ABI camera
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from rednoise_b200 import scenes  # noqa: E402
import raysets  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def model_arrays(m):
    a = m.arrays()
    return {k: a[k] for k in ("v", "rgb", "material", "normal", "roughness")}


def rays_for(v9, seed):
    lo, hi = raysets.scene_bounds(v9)
    o1, d1 = raysets.random_rays(3000, seed, lo, hi)
    o2, d2 = raysets.towards_rays(3000, seed + 1, v9, lo, hi)
    fo, fd = raysets.fan_rays()
    o = np.concatenate([fo, o1, o2])
    d = np.concatenate([fd, d1, d2])
    rng = np.random.default_rng(seed + 2)
    tmax = (rng.random(o.shape[0]) * 4.0).astype(np.float32)
    tmax[rng.random(o.shape[0]) < 0.1] = np.float32(1e6)
    ignore = np.where(rng.random(o.shape[0]) < 0.2, rng.integers(0, v9.shape[0], o.shape[0]), -1).astype(np.int32)
    return o, d, tmax, ignore


def main(refdir: str) -> None:
    assets = {}
    trace = {}
    for name, fname, scale in (("cornell", "cornell-box.obj", 0.35), ("sphere", "sphere.obj", 0.35)):
        m = oracle.RefModel.from_obj(os.path.join(refdir, "assets", fname), scale)
        arr = model_arrays(m)
        for k, v in arr.items():
            assets[f"{name}_{k}"] = v
        o, d, tmax, ignore = rays_for(arr["v"], 1234 + len(name))
        idx, t, u, v = m.intersect(o, d)
        idx_i, t_i, _, _ = m.intersect(o, d, ignore)
        occ = m.occluded(o, d, tmax, ignore)
        trace.update({f"{name}_o": o, f"{name}_d": d, f"{name}_tmax": tmax, f"{name}_ignore": ignore,
                      f"{name}_idx": idx, f"{name}_t": t.view(np.uint32), f"{name}_u": u.view(np.uint32),
                      f"{name}_v": v.view(np.uint32), f"{name}_idx_ig": idx_i, f"{name}_t_ig": t_i.view(np.uint32),
                      f"{name}_occ": occ})
        m.close()
    box = scenes.cornell_box()
    m = oracle.RefModel.from_arrays(box["vertices"])
    o, d, tmax, ignore = rays_for(box["vertices"], 99)
    idx, t, u, v = m.intersect(o, d)
    occ = m.occluded(o, d, tmax, ignore)
    trace.update({"box_o": o, "box_d": d, "box_tmax": tmax, "box_ignore": ignore, "box_idx": idx,
                  "box_t": t.view(np.uint32), "box_u": u.view(np.uint32), "box_v": v.view(np.uint32),
                  "box_occ": occ})
    m.close()
    np.savez_compressed(os.path.join(HERE, "assets_ref.npz"), **assets)
    np.savez_compressed(os.path.join(HERE, "trace_ref.npz"), **trace)

    # renderPathTraced through the C ABI camera, on the loaded Cornell box.
    lib = oracle.ref()
    sc = lib.rn_scene_load_obj(os.fsencode(os.path.join(refdir, "assets", "cornell-box.obj")), 0.35)
    renders = {}
    for (w, h, spp) in ((64, 48, 4), (96, 72, 16)):
        buf = np.zeros((h, w, 4), np.uint8)
        assert lib.rn_render(sc, 3, w, h, 4.0, spp, oracle.P(buf)) == 1
        renders[f"rgba_{w}x{h}_{spp}"] = buf
    lib.rn_scene_free(sc)
    np.savez_compressed(os.path.join(HERE, "render_ref.npz"), **renders)
    for f in ("assets_ref.npz", "trace_ref.npz", "render_ref.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RN_REFERENCE_DIR", "/root/reference"))
