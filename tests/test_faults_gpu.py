"""Failed device allocations fail cleanly (host-side fault injection).

rn_pt_inject_allocation_failure(k) makes the k-th next device allocation report
out-of-memory, once. For every k up to the workload's allocation count, each call
of a workload that touches every renderer must either succeed or raise
RN_ERR_OUT_OF_MEMORY, and afterwards the same scene object must render exactly
what a scene that never saw a failure renders. Nothing here faults the GPU: the
failure is made on the host, before cudaMalloc is called.
"""
import ctypes

import numpy as np
import pytest

import rednoise_b200 as rn
from rednoise_b200 import _native, scenes

pytestmark = pytest.mark.gpu


def _inject(k: int) -> None:
    _native.load().rn_pt_inject_allocation_failure(ctypes.c_longlong(k))


def _scene():
    box = scenes.cornell_box()
    return rn.Scene.from_arrays(box["vertices"], **{k: box[k] for k in ("albedo", "emission", "material",
                                                                       "material_param", "ref_rgb",
                                                                       "ref_material", "ref_roughness")})


def _workload(s):
    c = scenes.camera(32, 24)
    cam = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], 32, 24)
    out = [s.render_physical(cam, rn.Settings.make(spp=4, max_depth=4, seed=3, integrator=2)),
           s.render_physical(cam, rn.Settings.make(spp=4, max_depth=4, seed=3, integrator=1)),
           s.render_reference(32, 24, 2, position=(0, 0, scenes.CAMERA_Z)),
           s.render_raytraced(32, 24, position=(0, 0, scenes.CAMERA_Z)),
           s.render_bidirectional(32, 24, 2, position=(0, 0, scenes.CAMERA_Z)),
           s.render_photon_mapped(32, 24, 2000, position=(0, 0, scenes.CAMERA_Z))]
    s.build_lbvh()
    out.append(s.render_physical(cam, rn.Settings.make(spp=2, max_depth=4, seed=5, integrator=2), lbvh=True))
    return out


def test_allocation_failures_fail_cleanly():
    ok = _scene()
    want = _workload(ok)
    ok.close()
    failures = 0
    finished = False
    for k in range(200):
        s = None
        _inject(k)
        try:
            s = _scene()
            _workload(s)
            finished = True
        except rn.RnError as e:
            assert e.status == _native.RN_ERR_OUT_OF_MEMORY, str(e)
            failures += 1
        finally:
            _inject(-1)
        if s is not None:
            again = _workload(s)
            for a, b in zip(again, want):
                assert np.array_equal(a, b), f"results differ after the failed allocation {k}"
            s.close()
        if finished:
            break
    assert finished and failures >= 10, (finished, failures)
