"""PyTorch binding of the differentiable path tracer.

``render(albedo, emission, scene, views, adjoint)`` renders every view's mean
radiance image on the GPU and is differentiable with respect to the per-triangle
``albedo`` and ``emission`` tensors (n x 3, float32, CUDA). The backward pass
calls the path-replay adjoint kernel (rn_pt_backward) with the views' adjoint
settings: every path is regenerated from its RNG key, so memory stays O(pixels).
All work is enqueued on PyTorch's current CUDA stream with device pointers; no
host copies are made.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import torch

from . import _native


def _stream_handle() -> ctypes.c_void_p:
    h = torch.cuda.current_stream().cuda_stream
    # The legacy default stream is handle 0 in PyTorch; name it explicitly
    # (cudaStreamLegacy) so the library does not substitute its own stream.
    return ctypes.c_void_p(h if h else 1)


def _check_params(t: torch.Tensor, n: int, name: str) -> torch.Tensor:
    if not t.is_cuda or t.dtype != torch.float32 or t.shape != (n, 3):
        raise ValueError(f"{name} must be a CUDA float32 tensor of shape ({n}, 3)")
    return t.contiguous()


class _PathTrace(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, emission, scene, views, adjoint):
        lib = _native.load()
        n = scene.triangle_count
        albedo = _check_params(albedo, n, "albedo")
        emission = _check_params(emission, n, "emission")
        stream = _stream_handle()
        flags = _native.RN_PT_DEVICE_POINTERS
        _native.check(lib.rn_pt_scene_set_materials(scene.handle, ctypes.c_void_p(albedo.data_ptr()),
                                                    ctypes.c_void_p(emission.data_ptr()), flags, stream),
                      "rn_pt_scene_set_materials")
        images = []
        for camera, settings in views:
            img = torch.empty((camera.height, camera.width, 3), dtype=torch.float32, device=albedo.device)
            _native.check(lib.rn_pt_render(scene.handle, ctypes.byref(camera), ctypes.byref(settings), flags, stream,
                                           ctypes.c_void_p(img.data_ptr())), "rn_pt_render")
            images.append(img)
        # The scene holds one set of materials: backward puts this call's back before
        # replaying the paths, so another forward in between (another parameter set on
        # the same scene) does not change what this call differentiates.
        ctx.save_for_backward(albedo, emission)
        ctx.scene = scene
        ctx.adjoint = adjoint
        ctx.device = albedo.device
        return tuple(images)

    @staticmethod
    def backward(ctx, *grads):
        lib = _native.load()
        scene, adjoint = ctx.scene, ctx.adjoint
        n = scene.triangle_count
        nv = len(adjoint)
        gimgs = [g.contiguous() if g is not None else torch.zeros(
            (c.height, c.width, 3), dtype=torch.float32, device=ctx.device) for g, (c, _) in zip(grads, adjoint)]
        cams = (_native.Camera * nv)(*[v[0] for v in adjoint])
        sets = (_native.Settings * nv)(*[v[1] for v in adjoint])
        ptrs = (ctypes.c_void_p * nv)(*[g.data_ptr() for g in gimgs])
        d_alb = torch.empty((n, 3), dtype=torch.float32, device=ctx.device)
        d_em = torch.empty((n, 3), dtype=torch.float32, device=ctx.device)
        albedo, emission = ctx.saved_tensors
        stream = _stream_handle()
        _native.check(lib.rn_pt_scene_set_materials(scene.handle, ctypes.c_void_p(albedo.data_ptr()),
                                                    ctypes.c_void_p(emission.data_ptr()),
                                                    _native.RN_PT_DEVICE_POINTERS, stream),
                      "rn_pt_scene_set_materials")
        _native.check(lib.rn_pt_backward(scene.handle, nv, cams, sets, ptrs, _native.RN_PT_DEVICE_POINTERS,
                                         stream, ctypes.c_void_p(d_alb.data_ptr()),
                                         ctypes.c_void_p(d_em.data_ptr())), "rn_pt_backward")
        return d_alb, d_em, None, None, None


def render(albedo: torch.Tensor, emission: torch.Tensor, scene, views: Sequence[Tuple], adjoint: Sequence[Tuple] = None
           ) -> List[torch.Tensor]:
    """Render views [(Camera, Settings)] of ``scene`` with the given materials.

    ``adjoint`` gives each view's (Camera, Settings) for the backward pass
    (default: the same settings, i.e. the same samples as the primal).
    """
    adjoint = list(views) if adjoint is None else list(adjoint)
    if len(adjoint) != len(views):
        raise ValueError("one adjoint setting per view")
    return list(_PathTrace.apply(albedo, emission, scene, list(views), adjoint))
