"""FP64 CPU reference radiance for the RMSE measurements (oracle, 65536 spp).

A full-frame FP64 render at 65536 spp is out of reach of a host CPU, so the
reference is computed on a seeded subset of pixels of each workload and stored
with the pixel indices:

  python tests/golden/make_fp64_reference.py            (about 3 minutes on 8 cores)

fp64_ref.npz keys, for workload in (c1, c2):
  <w>_pixels   int32 pixel indices (row-major)
  <w>_mean     float64 (n, 3) mean radiance of 65536 samples
  <w>_var      float64 (n, 3) variance of the 65536-sample mean (from 16 batches)
  <w>_spec     [width, height, max_depth, rr_depth, spp, seed]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rednoise_b200 import scenes  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
SPP = 65536
BATCHES = 16
SEED = 0xF64F64


def run(name, sc, w, h, depth, rr, npix):
    cam = scenes.camera(w, h)
    rng = np.random.default_rng(1234 if name == "c1" else 5678)
    px = np.sort(rng.choice(w * h, npix, replace=False)).astype(np.int32)
    o = oracle.OrcPhysScene(sc)
    per = SPP // BATCHES
    batch_means = []
    t0 = time.time()
    for b in range(BATCHES):
        s = o.render_sums(cam, per, depth, rr, SEED, offset=b * per, pixels=px, double=True)
        batch_means.append(s / per)
    bm = np.stack(batch_means)
    mean = bm.mean(0)
    var = bm.var(0, ddof=1) / BATCHES
    print(name, f"{time.time() - t0:.1f}s", "mean radiance", mean.mean(0))
    return {f"{name}_pixels": px, f"{name}_mean": mean, f"{name}_var": var,
            f"{name}_spec": np.array([w, h, depth, rr, SPP, SEED], np.int64)}


def main():
    out = {}
    out.update(run("c1", scenes.cornell_box(), 320, 240, 5, 5, 1024))
    out.update(run("c2", scenes.icosphere_scene(), 1920, 1080, 8, 3, 512))
    np.savez_compressed(os.path.join(HERE, "fp64_ref.npz"), **out)


if __name__ == "__main__":
    main()
