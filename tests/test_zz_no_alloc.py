"""rn_pt_render_static: the physical-mode render whose scratch is a fixed array
inside the library, for callers that must not allocate GPU memory while they
render (a host that owns a fixed memory budget, a framework whose allocator must
not be bypassed, a real-time loop). Checked through the C ABI on consecutive
calls that share that array: against rn_pt_render (the same megakernel with
scene-owned scratch) and against the CPU oracle on the same random numbers, bit
for bit; the
calls succeed while the next device allocation is armed to fail, and they do not
change the device's free memory.

Named to be collected last, so it also runs after every other GPU test has
used the library in the same process.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import rednoise_b200 as rn
from imgcheck import assert_bit_equal, oracle_float_frame
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


def _call_static(s, camera, settings, out):
    lib = _native.load()
    return lib.rn_pt_render_static(s._handle, ctypes.byref(camera), ctypes.byref(settings), 0, None,
                                   ctypes.c_void_p(out.data_ptr()))


def test_static_scratch_render_matches_rn_pt_render_and_oracle():
    torch.cuda.set_device(0)
    sc = scenes.icosphere_scene(level=3)
    s = _scene(sc)
    orc = oracle.OrcPhysScene(sc)
    lib = _native.load()
    # Set-up call: the first call on a device resolves the array's address (and the
    # driver loads the module that holds the array); later calls only render.
    warm = torch.empty(8 * 6 * 3, device="cuda:0")
    _native.check(_call_static(s, _camera(8, 6), rn.Settings.make(spp=1, max_depth=2), warm), "rn_pt_render_static")
    torch.cuda.synchronize()
    # two calls in a row: the second is smaller and reuses the array the first filled
    for (w, h, spp, seed) in ((96, 72, 8, 11), (40, 30, 5, 12)):
        camera = _camera(w, h)
        settings = rn.Settings.make(spp=spp, max_depth=8, rr_depth=3, seed=seed, integrator=_native.RN_PT_MEGAKERNEL)
        out = torch.full((h * w * 3,), float("nan"), device="cuda:0")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        # The next device allocation the library makes would fail: this call makes none.
        lib.rn_pt_inject_allocation_failure(ctypes.c_longlong(0))
        try:
            st = _call_static(s, camera, settings, out)
        finally:
            lib.rn_pt_inject_allocation_failure(ctypes.c_longlong(-1))
        _native.check(st, "rn_pt_render_static")
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        got = out.cpu().numpy()
        want = s.render_physical(camera, settings).reshape(-1)
        assert np.isfinite(got).all()
        assert want.mean() > 0
        # the same megakernel with the same summation order: the same bits, and the
        # oracle's float frame bit for bit
        assert_bit_equal(got, want)
        assert_bit_equal(got, oracle_float_frame(orc, scenes.camera(w, h), spp, 8, 3, seed=seed))
    s.close()


def test_static_scratch_rejects_oversize_image():
    torch.cuda.set_device(0)
    s = _scene(scenes.cornell_box())
    lib = _native.load()
    camera = _camera(513, 512)
    assert camera.width * camera.height > _native.RN_PT_STATIC_MAX_PIXELS
    settings = rn.Settings.make(spp=1, max_depth=2)
    out = torch.zeros(16, device="cuda:0")
    assert _call_static(s, camera, settings, out) == _native.RN_ERR_CAPACITY  # before any GPU work
    assert b"512 x 512" in lib.rn_pt_last_error()
    s.close()


def test_static_scratch_rejects_host_output():
    """A host buffer is refused before any kernel could write to it."""
    torch.cuda.set_device(0)
    s = _scene(scenes.cornell_box())
    camera = _camera(8, 6)
    settings = rn.Settings.make(spp=1, max_depth=2)
    for pinned in (False, True):
        out = torch.zeros(8 * 6 * 3, pin_memory=pinned)
        assert _call_static(s, camera, settings, out) == _native.RN_ERR_INVALID_ARGUMENT
        assert (out == 0).all()
    s.close()
