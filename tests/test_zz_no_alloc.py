"""rn_pt_render_static: the physical-mode render whose scratch is a fixed array
inside the library (no allocation), checked against rn_pt_render through the
C ABI on consecutive calls that share that array.

Named to be collected last, so it also runs after every other GPU test has
used the library in the same process.
"""
import ctypes

import numpy as np
import pytest
import torch

import rednoise_b200 as rn
from rednoise_b200 import _native, scenes

pytestmark = pytest.mark.gpu


def _scene(sc):
    s = rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                             material=sc["material"], material_param=sc["material_param"])
    s.prepare()
    return s


def _camera(w, h):
    c = scenes.camera(w, h)
    return rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], w, h)


def _render_static(s, camera, settings):
    lib = _native.load()
    out = torch.full((camera.height * camera.width * 3,), float("nan"), device="cuda:0")
    torch.cuda.synchronize()
    st = lib.rn_pt_render_static(s._handle, ctypes.byref(camera), ctypes.byref(settings), 0, None,
                                 ctypes.c_void_p(out.data_ptr()))
    _native.check(st, "rn_pt_render_static")
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _render_reference_path(s, camera, settings):
    return s.render_physical(camera, settings).reshape(-1)


def test_static_scratch_render_matches_rn_pt_render():
    torch.cuda.set_device(0)
    s = _scene(scenes.icosphere_scene(level=3))
    # two calls in a row: the second is smaller and reuses the array the first filled
    for (w, h, spp, seed) in ((96, 72, 8, 11), (40, 30, 5, 12)):
        camera = _camera(w, h)
        settings = rn.Settings.make(spp=spp, max_depth=8, rr_depth=3, seed=seed, integrator=_native.RN_PT_MEGAKERNEL)
        got = _render_static(s, camera, settings)
        want = _render_reference_path(s, camera, settings)
        assert np.isfinite(got).all()
        assert want.mean() > 0
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6)
    s.close()


def test_static_scratch_rejects_oversize_image():
    torch.cuda.set_device(0)
    s = _scene(scenes.cornell_box())
    lib = _native.load()
    camera = _camera(513, 512)
    assert camera.width * camera.height > _native.RN_PT_STATIC_MAX_PIXELS
    settings = rn.Settings.make(spp=1, max_depth=2)
    out = torch.zeros(16, device="cuda:0")
    st = lib.rn_pt_render_static(s._handle, ctypes.byref(camera), ctypes.byref(settings), 0, None,
                                 ctypes.c_void_p(out.data_ptr()))
    assert st == 6  # RN_ERR_CAPACITY, before any GPU work
    assert b"512 x 512" in lib.rn_pt_last_error()
    s.close()
