"""Multi-view inverse rendering of per-triangle albedo on the device.

Every step renders all views with one batched launch (the views' frames share
one wave schedule, captured once as a CUDA graph, when the batch runs the
wavefront), forms the L2 image loss against the targets on the device, runs the
path-replay adjoint of all views in one launch, and takes an Adam step on the
albedo, which is written back into the scene's shading records without a host
round trip. The renders and the adjoint use disjoint sample indices, so the
gradient estimate is unbiased for the expected loss.
"""
from __future__ import annotations

import ctypes
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _native


def _cam(c) -> "_native.Camera":
    if isinstance(c, _native.Camera):
        return c
    return _native.Camera.make(c["position"], c["target"], c.get("up", (0.0, 1.0, 0.0)), c.get("vfov_deg", 40.0),
                               c["width"], c["height"])


class AlbedoFit:
    """Adam on the per-triangle albedo of ``scene`` (an ``rednoise_b200.Scene``)
    against ``targets`` (one (h, w, 3) image per view, host or CUDA)."""

    def __init__(self, scene, views: Sequence, targets: Sequence, albedo0, spp: int = 16, max_depth: int = 5,
                 lr: float = 0.02, seed: int = 1, bounds=(0.01, 0.99)):
        import torch

        from . import Batch

        self.torch = torch
        self.scene = scene
        self.cams = [_cam(v) for v in views]
        self.spp, self.max_depth, self.seed = int(spp), int(max_depth), int(seed)
        self.bounds = bounds
        self.stream = torch.cuda.Stream()
        self.sptr = ctypes.c_void_p(self.stream.cuda_stream)
        dev = torch.device("cuda")
        self.targets = [torch.as_tensor(t if torch.is_tensor(t) else np.asarray(t, np.float32),
                                        device=dev).reshape(-1) for t in targets]
        self.n_values = sum(t.numel() for t in self.targets)
        self.albedo = torch.as_tensor(np.asarray(albedo0, np.float32), device=dev).reshape(-1, 3).clone()
        self.albedo.requires_grad_(True)
        self.opt = torch.optim.Adam([self.albedo], lr=lr)
        self.images = [torch.empty(c.height * c.width * 3, device=dev) for c in self.cams]
        self.d_images = [torch.empty_like(i) for i in self.images]
        self.g_alb = torch.empty(self.albedo.numel(), device=dev)
        self.g_em = torch.empty(self.albedo.numel(), device=dev)
        self.lib = _native.load()
        torch.cuda.synchronize()
        self._push_albedo()
        self.stream.synchronize()
        jobs = [(scene, c, _native.Settings.make(spp=self.spp, max_depth=self.max_depth, rr_depth=self.max_depth,
                                                 seed=self.seed)) for c in self.cams]
        self.batch = Batch(jobs, integrator=_native.RN_PT_AUTO)
        self._out_ptrs = (ctypes.c_void_p * len(self.images))(*[i.data_ptr() for i in self.images])
        self._d_ptrs = (ctypes.c_void_p * len(self.d_images))(*[g.data_ptr() for g in self.d_images])
        self._cams_arr = (_native.Camera * len(self.cams))(*self.cams)
        self.step_index = 0

    def _push_albedo(self):
        _native.check(self.lib.rn_pt_scene_set_materials(self.scene.handle, ctypes.c_void_p(self.albedo.data_ptr()),
                                                         None, _native.RN_PT_DEVICE_POINTERS, self.sptr),
                      "rn_pt_scene_set_materials")

    def render(self, sample_offset: int):
        """Render every view into ``self.images`` (one batched launch)."""
        _native.check(self.lib.rn_pt_batch_render(self.batch._handle, int(sample_offset),
                                                  _native.RN_PT_DEVICE_POINTERS, self.sptr, self._out_ptrs),
                      "rn_pt_batch_render")

    def adjoint(self, sample_offset: int):
        """d loss / d albedo of the current image gradients (all views, one launch)."""
        sets = (_native.Settings * len(self.cams))(*[
            _native.Settings.make(spp=self.spp, max_depth=self.max_depth, rr_depth=self.max_depth, seed=self.seed,
                                  sample_offset=sample_offset) for _ in self.cams])
        _native.check(self.lib.rn_pt_backward(self.scene.handle, len(self.cams), self._cams_arr, sets, self._d_ptrs,
                                              _native.RN_PT_DEVICE_POINTERS, self.sptr,
                                              ctypes.c_void_p(self.g_alb.data_ptr()),
                                              ctypes.c_void_p(self.g_em.data_ptr())), "rn_pt_backward")

    def step(self):
        """One Adam step; returns the loss (a device scalar, not synchronised)."""
        torch = self.torch
        k = self.step_index
        self.step_index += 1
        with torch.cuda.stream(self.stream):
            self.render(sample_offset=2 * k * self.spp)
            loss = torch.zeros((), device=self.albedo.device)
            for img, tgt, g in zip(self.images, self.targets, self.d_images):
                r = img - tgt
                loss = loss + (r * r).sum()
                torch.mul(r, 2.0 / self.n_values, out=g)
            loss = loss / self.n_values
            self.adjoint(sample_offset=(2 * k + 1) * self.spp)
            self.albedo.grad = self.g_alb.view_as(self.albedo)
            self.opt.step()
            with torch.no_grad():
                self.albedo.clamp_(*self.bounds)
            self._push_albedo()
        return loss

    def run(self, steps: int, on_step: Optional[Callable] = None) -> List[float]:
        """``steps`` Adam steps; returns the losses (one host synchronisation at the end)."""
        losses = []
        for i in range(steps):
            loss = self.step()
            if on_step is not None:
                on_step(i, loss)
            losses.append(loss)
        self.torch.cuda.synchronize()
        return [float(x) for x in losses]

    def close(self):
        self.batch.close()
