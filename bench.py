#!/usr/bin/env python
"""Benchmark of the path-tracing hot path on B200.

Workload (one step = one full frame): the 1.31M-triangle displaced-icosphere
Cornell box (seeded synthetic scene, rednoise_b200.scenes.icosphere_scene),
1920x1080, 64 samples per pixel, max depth 8, Russian roulette from vertex 3,
physical estimator. Metric: samples/s (whole job). Multi-GPU: weak scaling,
each rank renders its own 64 samples per pixel (disjoint sample indices) with
no data-path collective.

  python bench.py [--gpus N --steps K --warmup W]
  python bench.py --impl reference      # the reference's CPU renderPathTraced

Printed: one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "samples/s (path-traced samples per second)"
UNIT = "samples/s"
WORKLOAD = "icosphere-cornell-1.31M-tris 1920x1080 64spp depth8"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    p.add_argument("--spp", type=int, default=64)
    p.add_argument("--depth", type=int, default=8)
    p.add_argument("--rr", type=int, default=3)
    p.add_argument("--level", type=int, default=8, help="icosphere subdivision level (8 = 1.31M triangles)")
    p.add_argument("--integrator", default="auto", choices=["auto", "megakernel", "wavefront"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-grad", action="store_true", help="skip the gradient-vs-primal timing")
    p.add_argument("--no-extra", action="store_true",
                   help="skip the 64-scene batch and the 16-view inverse rendering keys of the frame line")
    p.add_argument("--workload", default="frame", choices=["frame", "batch64", "inverse", "raytraced", "photon", "lbvh",
                                                       "bidirectional", "metropolis", "dropin"],
                   help="frame: the 1.31M-triangle 1080p frame (the bench line); batch64: 64 scenes per "
                        "launch; inverse: 16-view albedo recovery; raytraced: Whitted ray tracing; "
                        "photon: photon mapping; lbvh: the GPU-built BVH; bidirectional: bidirectional path "
                        "tracing; metropolis: Metropolis light transport; dropin: the rn_render path tracer "
                        "(reference semantics) alone")
    p.add_argument("--small", action="store_true",
                   help="bidirectional / metropolis / dropin: the small case used for profiles (160x120 at 16 spp, "
                        "400 000 mutations, 480x270 at 1 spp)")
    p.add_argument("--inverse-steps", type=int, default=200)
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(
        os.environ.get("WORLD_SIZE", "1"))


def free_port() -> int:
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_entry(rank: int, world: int, port: int, target, targs):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    target(*targs)


def spawn_ranks(world: int, target, *targs) -> None:
    """One process per GPU when bench.py is started without a launcher: ranks
    0..world-1 get RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT as
    torchrun sets them, then run target(*targs)."""
    import torch.multiprocessing as mp

    mp.start_processes(_rank_entry, args=(world, free_port(), target, targs), nprocs=world, join=True,
                       start_method="spawn")


def shard_sample_offset(step: int, rank: int, world: int, spp: int) -> int:
    """First sample index of this rank's frame at this step: ranks and steps take
    consecutive, disjoint blocks of spp sample indices, so the ranks' frames sum to
    one render of world * spp samples (weak scaling, no data-path exchange)."""
    return (step * world + rank) * spp


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum of per-rank timings (the slowest rank sets the job time)."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


# ---- clocks sampled during the timed region ------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.rows = []
        self.proc = None
        self.index = index

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for k, name in enumerate(names):
                    if r[3 + k].lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- CPU baseline: the reference's renderPathTraced (oracle/_ref) ---------------------

def reference_model(sc):
    import oracle

    return oracle.RefModel.from_arrays(sc["vertices"], sc["ref_rgb"], sc["ref_material"], sc["ref_roughness"])


def reference_focal(height: int) -> float:
    # f = focalLength * 150 pixels gives the 40-degree vertical field of view.
    return (height / 2.0) / math.tan(math.radians(20.0)) / 150.0


def time_reference_step(model, w, h, spp) -> float:
    from rednoise_b200 import scenes

    t0 = time.perf_counter()
    model.render(w, h, spp, focal=reference_focal(h), pos=(0.0, 0.0, scenes.CAMERA_Z), target=(0.0, 0.0, 0.0))
    return time.perf_counter() - t0


def reference_bvh_build_s(model, reps: int = 2) -> float:
    """Seconds of one reference BVH build over the model (renderPathTraced rebuilds it
    on every call)."""
    import oracle

    lib = oracle.ref()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        bvh = lib.refsh_bvh_new(model.h)
        best = min(best, time.perf_counter() - t0)
        lib.refsh_bvh_free(bvh)
    return best


def reference_rate(model, w, h, spp, calls, warmup=0, min_s=0.0, full_spp=64) -> dict:
    """The reference renderPathTraced timed over whole-frame calls of spp samples.
    Each call rebuilds the BVH, as the reference does; the rate charges that build
    once per full_spp samples per pixel, as one call rendering the whole workload
    would, so a bounded sample of few spp is not dominated by it."""
    for _ in range(warmup):
        time_reference_step(model, w, h, spp)
    dts = []
    while len(dts) < calls or sum(dts) < min_s:
        dts.append(time_reference_step(model, w, h, spp))
    build = reference_bvh_build_s(model)
    total = sum(dts)
    charged = total - len(dts) * build * (1.0 - spp / float(full_spp))
    samples = w * h * spp * len(dts)
    return {"value": samples / charged, "calls": len(dts), "seconds": total, "bvh_build_s": build,
            "per_call_value": samples / total, "samples": samples}


def cpu_baseline(sc, w=1920, h=1080, target_s=12.0) -> dict:
    model = reference_model(sc)
    r = reference_rate(model, w, h, 2, calls=1, min_s=target_s)
    return {"value": r["value"], "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "sample": f"reference renderPathTraced (oracle/_ref, OpenMP, reference semantics: depth 4, default "
                      f"light) on the same 1.31M-triangle geometry and camera: {r['calls']} calls of {w}x{h} at "
                      f"2 spp ({r['samples']} samples, {r['seconds']:.1f} s); each call rebuilds the BVH "
                      f"({r['bvh_build_s']:.2f} s), charged once per 64 spp; uncharged rate "
                      f"{r['per_call_value']:.4g} samples/s"}


def cpu_physical_baseline(sc, cam, args, target_s=8.0) -> dict:
    """The restated FP32 physical integrator (the oracle: same estimator, materials and
    emitter sampling as the GPU) on all host cores, over a seeded pixel subset."""
    import oracle

    orc = oracle.OrcPhysScene(sc)
    rng = np.random.default_rng(7)
    n_pix = cam["width"] * cam["height"]
    npx, spp = 2048, 4
    while True:
        px = rng.choice(n_pix, npx, replace=False).astype(np.int32)
        t0 = time.perf_counter()
        orc.render_sums(cam, spp, args.depth, args.rr, seed=1, pixels=px)
        dt = time.perf_counter() - t0
        if dt > target_s / 3 or (npx >= n_pix and spp >= 64):
            break
        grow = max(2.0, target_s / 3 / max(dt, 1e-3))
        if npx < n_pix:
            npx = min(n_pix, int(npx * grow))
        else:
            spp = min(64, int(spp * grow))
    return {"value": npx * spp / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"oracle FP32 physical integrator (OpenMP), {npx} seeded pixels of the "
                      f"{cam['width']}x{cam['height']} frame at {spp} spp, depth {args.depth}, RR from {args.rr} "
                      f"({dt:.1f} s)"}


def gradient_timing(scene, lib, stream, sptr, l2, size=512, spp=32, depth=6) -> dict:
    """One albedo/emission gradient by the path-replay adjoint against one primal render:
    the same 1.31M-triangle scene at 512x512, 32 spp primal + 32 spp adjoint, depth 6,
    L2 loss against a render with another seed."""
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import _native, scenes

    c = scenes.camera(size, size)
    cam = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], size, size)
    flags = _native.RN_PT_DEVICE_POINTERS
    npx = size * size * 3
    img = torch.empty(npx, device="cuda")
    target = torch.empty(npx, device="cuda")
    n = scene.triangle_count
    g_alb = torch.empty(n * 3, device="cuda")
    g_em = torch.empty(n * 3, device="cuda")

    def primal(out, seed):
        st = rn.Settings.make(spp=spp, max_depth=depth, rr_depth=depth, seed=seed)
        _native.check(lib.rn_pt_render(scene.handle, ctypes.byref(cam), ctypes.byref(st), flags, sptr,
                                       ctypes.c_void_p(out.data_ptr())), "rn_pt_render")

    with torch.cuda.stream(stream):
        primal(target, 99)
        primal(img, 1)  # first call at this shape: autotune + graph capture
        d_img = (2.0 / npx) * (img - target)
        ptrs = (ctypes.c_void_p * 1)(d_img.data_ptr())
        st = rn.Settings.make(spp=spp, max_depth=depth, rr_depth=depth, seed=1)

        def adjoint():
            _native.check(lib.rn_pt_backward(scene.handle, 1, ctypes.byref(cam), ctypes.byref(st), ptrs, flags,
                                             sptr, ctypes.c_void_p(g_alb.data_ptr()),
                                             ctypes.c_void_p(g_em.data_ptr())), "rn_pt_backward")

        adjoint()
        torch.cuda.synchronize()
        tp, ta = [], []
        for _ in range(3):
            for fn, acc in ((lambda: primal(img, 1), tp), (adjoint, ta)):
                l2.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                acc.append(e0.elapsed_time(e1))
    p_ms, a_ms = float(np.median(tp)), float(np.median(ta))
    return {"workload": f"{size}x{size}, {spp} spp primal + {spp} spp adjoint, depth {depth}, "
                        f"d loss / d albedo ({n} x 3) and emission",
            "primal_ms": p_ms, "adjoint_ms": a_ms, "adjoint_over_primal": a_ms / p_ms,
            "grad_nonzero": int((g_alb != 0).sum().item())}


def time_to_rmse(scene, lib, stream, sptr, cam, args, fp64, W, H, target=0.5, frame_spp=64, max_frames=32):
    """Time for each integrator to bring the frame's relative RMSE against the FP64
    65536-spp reference (its seeded 512-pixel subset) below `target`: 64-spp frames of
    consecutive sample indices are accumulated (rn_pt_render_accumulate) until the
    running mean reaches the target. Both integrators render the same samples to the
    same floats, so they need the same number of frames; the time is the sum of the
    frames' device times (CUDA events; the RMSE check between frames is not timed).
    Also the relative RMSE of single 64-spp frames over 8 sample blocks: a few
    subset pixels see rare, bright caustic paths (light reaching the emitter-lit
    surfaces through the dielectric triangles), so one 64-spp block's error depends
    on whether such a path was drawn."""
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import _native

    px = torch.as_tensor(fp64["c2_pixels"].astype(np.int64), device="cuda")
    mref = torch.as_tensor(fp64["c2_mean"], device="cuda", dtype=torch.float64)
    ref_norm = float(torch.sqrt((mref ** 2).mean()))
    acc = torch.zeros(H * W * 3, dtype=torch.float32, device="cuda")
    base = 1 << 24  # sample indices not used by the timed frames

    def rel_rmse(mean_flat):
        m = mean_flat.view(-1, 3)[px].to(torch.float64)
        return float(torch.sqrt(((m - mref) ** 2).mean())) / ref_norm

    def frame(code, k):
        st = rn.Settings.make(spp=frame_spp, max_depth=args.depth, rr_depth=args.rr, integrator=code, seed=1,
                              sample_offset=base + k * frame_spp)
        _native.check(lib.rn_pt_render_accumulate(scene.handle, ctypes.byref(cam), ctypes.byref(st),
                                                  _native.RN_PT_DEVICE_POINTERS, sptr,
                                                  ctypes.c_void_p(acc.data_ptr())), "rn_pt_render_accumulate")

    out = {"target_relative_rmse": target, "frame_spp": frame_spp,
           "reference": "FP64 oracle estimator, 65536 spp, 512 seeded pixels (tests/golden/fp64_ref.npz)"}
    with torch.cuda.stream(stream):
        blocks = []
        for b in range(8):
            acc.zero_()
            frame(_native.RN_PT_AUTO, 1000 + b)
            torch.cuda.synchronize()
            blocks.append(rel_rmse(acc / frame_spp))
        out["single_64spp_frame_relative_rmse"] = {"min": min(blocks), "median": float(np.median(blocks)),
                                                   "max": max(blocks)}
        for name, code in (("wavefront", _native.RN_PT_AUTO), ("megakernel", _native.RN_PT_MEGAKERNEL)):
            acc.zero_()
            frame(code, 999)  # warm-up (graph capture of the accumulate path), not counted
            acc.zero_()
            ms, err, k = 0.0, None, 0
            while k < max_frames:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                frame(code, k)
                e1.record(stream)
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
                k += 1
                err = rel_rmse(acc / (k * frame_spp))
                if err < target:
                    break
            out[name] = {"frames": k, "spp": k * frame_spp, "seconds": ms / 1e3, "relative_rmse": err,
                         "reached": err < target,
                         "samples_per_s_at_target": W * H * k * frame_spp / (ms / 1e3)}
    out["wavefront_speedup_at_target"] = out["megakernel"]["seconds"] / out["wavefront"]["seconds"]
    return out


def run_reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    from rednoise_b200 import scenes

    sc = scenes.icosphere_scene(level=args.level)
    model = reference_model(sc)
    w, h, spp = args.width, args.height, 1
    r = reference_rate(model, w, h, spp, calls=args.steps, warmup=args.warmup, full_spp=args.spp)
    value = r["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / r["calls"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "reference_step": f"{w}x{h} at {spp} of the {args.spp} spp "
                                                           f"(bounded sample of the frame)",
                   "semantics": "reference renderPathTraced: depth 4, default disk light, 8-bit output",
                   "bvh_build_s": r["bvh_build_s"], "uncharged_per_call_value": r["per_call_value"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                         "sample": f"{r['calls']} calls of {w}x{h} at {spp} spp; the per-call BVH rebuild "
                                   f"charged once per {args.spp} spp"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm -----------------------------------------------------------------------

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.isfile(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_peaks(lib, stream, sptr) -> dict:
    """Read bandwidths measured on this GPU in this run (rn_pt_probe_read, CUDA events):
    an L2-resident read (8-64 MB buffers read repeatedly within each launch, about
    2 GB per launch, with loads that bypass L1; the best size) and an HBM read (a
    2 GB buffer, one pass per launch)."""
    import torch

    from rednoise_b200 import _native

    out = {}
    best = 0.0
    for mb in (8, 16, 32, 64):
        buf = torch.empty(mb << 20, dtype=torch.uint8, device="cuda")
        buf.zero_()
        torch.cuda.synchronize()
        ms = ctypes.c_float(0.0)
        passes, n = (2 << 30) // buf.numel(), 20
        _native.check(lib.rn_pt_probe_read(ctypes.c_void_p(buf.data_ptr()), buf.numel(), passes, n, 1, sptr,
                                           ctypes.byref(ms)), "rn_pt_probe_read")
        gbs = buf.numel() * passes * n / (ms.value / 1e3) / 1e9
        out[f"l2_read_{mb}MB_gbs"] = gbs
        best = max(best, gbs)
        del buf
    out["l2_read_gbs"] = best
    big = torch.empty(2 << 30, dtype=torch.uint8, device="cuda")
    big.zero_()
    torch.cuda.synchronize()
    ms = ctypes.c_float(0.0)
    _native.check(lib.rn_pt_probe_read(ctypes.c_void_p(big.data_ptr()), big.numel(), 1, 5, 1, sptr,
                                       ctypes.byref(ms)), "rn_pt_probe_read")
    out["hbm_read_gbs"] = big.numel() * 5 / (ms.value / 1e3) / 1e9
    del big
    torch.cuda.empty_cache()
    return out


def kernel_profile():
    """ncu figures of the frame's stage kernels (instructions, lanes per instruction,
    issue activity, DRAM bytes per sample), committed under profiles/ from a capture of
    the same scene and wave configuration at 480x270; per-sample traffic is set by the
    scene, the path pool and the wave, which the autotuner chooses alike at both sizes."""
    path = os.path.join(ROOT, "profiles", "traversal_kernels.json")
    if not os.path.isfile(path):
        return None
    with open(path) as f:
        return json.load(f)


def reference_semantics_rate(sc, W, H, args, spp=2) -> dict:
    """The drop-in renderer (rn_render's renderPathTraced semantics: depth 4, the
    default disk light with its 9 shadow rays per vertex, per-pixel mt19937, 8-bit
    output) on the same geometry and camera as the CPU baseline, through the C ABI
    with a host canvas: the like-for-like counterpart of cpu_baseline."""
    import rednoise_b200 as rn
    from rednoise_b200 import scenes

    s = rn.Scene.from_arrays(sc["vertices"], ref_rgb=sc["ref_rgb"], ref_material=sc["ref_material"],
                             ref_roughness=sc["ref_roughness"])
    s.prepare()
    kw = dict(position=(0.0, 0.0, scenes.CAMERA_Z), focal_length=reference_focal(H))
    s.render_reference(W, H, spp, **kw)
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        s.render_reference(W, H, spp, **kw)
    dt = (time.perf_counter() - t0) / reps
    s.close()
    return {"value": W * H * spp / dt, "unit": UNIT, "ms_per_frame": dt * 1e3,
            "workload": f"{W}x{H} at {spp} spp, reference semantics (rn_pt_render_reference, host canvas)"}


def run_ours(args):
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import _native, scenes

    rank, local_rank, world = dist_env()
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but {world} ranks were launched")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    sc = scenes.icosphere_scene(level=args.level)
    scene = rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                                 material=sc["material"], material_param=sc["material_param"])
    scene.prepare()
    info = scene.info()
    W, H, spp = args.width, args.height, args.spp
    c = scenes.camera(W, H)
    cam = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], W, H)
    integ = {"auto": 0, "megakernel": 1, "wavefront": 2}[args.integrator]
    lib = _native.load()
    stream = torch.cuda.Stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    out = torch.empty(H * W * 3, dtype=torch.float32, device="cuda")
    l2 = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    flags = _native.RN_PT_DEVICE_POINTERS
    step_counter = [0]

    def settings():
        k = step_counter[0]
        step_counter[0] += 1
        return rn.Settings.make(spp=spp, max_depth=args.depth, rr_depth=args.rr, integrator=integ, seed=1,
                                sample_offset=shard_sample_offset(k, rank, world, spp))

    def render(st):
        _native.check(lib.rn_pt_render(scene.handle, ctypes.byref(cam), ctypes.byref(st), flags, sptr,
                                       ctypes.c_void_p(out.data_ptr())), "rn_pt_render")

    # Algorithmic bytes per sample: reference-order traversal counters on the GPU.
    counts = scene.count_traversal(cam, rn.Settings.make(spp=1, max_depth=args.depth, rr_depth=args.rr, seed=99))
    bytes_per_sample = (24.0 * (counts["closest_boxes"] + counts["any_boxes"]) +
                        36.0 * (counts["closest_tris"] + counts["any_tris"])) / counts["samples"]

    # The autotuner picks megakernel vs wavefront (and the wavefront queue capacity) for
    # this frame; the timed RN_PT_AUTO renders below use its choice.
    tuned = scene.autotune(cam, rn.Settings.make(spp=spp, max_depth=args.depth, rr_depth=args.rr, seed=1))
    if integ == 1 or (integ == 0 and tuned["integrator"] == 1):
        launches_per_step = 2  # megakernel + resolve
    else:
        spw = tuned["samples_per_wave"] if integ == 0 else max(1, min(spp, (1 << 20) // (W * H)))
        waves = (spp + spw - 1) // spw
        per_wave = 2 + 3 * args.depth  # camera, 3 stages per bounce, accumulate
        if tuned["ray_sort"] and not tuned["dynamic_fetch"]:
            # two-level counting sorts (count, column scan, scatter, refine) of the ray queue
            # before bounces 1.. and of the shadow queue at every bounce
            per_wave += 4 * (args.depth - 1) + 4 * args.depth
        launches_per_step = waves * per_wave + 1  # + resolve

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            l2.zero_()
            render(settings())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        clocks = ClockSampler(local_rank)
        clocks.start()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed")  # lets a profiler capture exactly the timed frames
        t_start.record(stream)
        for i in range(args.steps):
            l2.zero_()
            ev[i][0].record(stream)
            render(settings())
            ev[i][1].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    render_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks([total_ms], dist, "cuda")[0]
    ms_per_step = total_ms / args.steps
    samples_per_step = W * H * spp
    value = world * samples_per_step / (ms_per_step / 1e3)

    # The two integrators side by side on the same frame (same estimator, same samples):
    # the plain megakernel and the wavefront (SoA queues, CUDA-graph frame).
    ref_path = os.path.join(ROOT, "tests", "golden", "fp64_ref.npz")
    fp64 = None
    if os.path.isfile(ref_path) and (W, H, args.depth, args.rr) == (1920, 1080, 8, 3) and args.level == 8:
        fp64 = np.load(ref_path)

    def rmse_of(flat):
        if fp64 is None:
            return None
        img = np.asarray(flat).reshape(-1, 3)[fp64["c2_pixels"]].astype(np.float64)
        mref = fp64["c2_mean"]
        return float(np.sqrt(((img - mref) ** 2).mean()) / max(np.sqrt((mref ** 2).mean()), 1e-30))

    compare = {}
    rmse_by = {}
    same = settings()  # every integrator renders these same samples
    with torch.cuda.stream(stream):
        for name, code, extra in (("megakernel", 1, 0), ("wavefront", 2, 0),
                                  ("wavefront_static", 2, _native.RN_PT_WAVEFRONT_STATIC),
                                  ("wavefront_binned", 2, _native.RN_PT_RAY_SORT),
                                  ("wavefront_unbinned", 2, _native.RN_PT_NO_RAY_SORT)):
            def one():
                st = rn.Settings.make(spp=spp, max_depth=args.depth, rr_depth=args.rr, integrator=code, seed=1,
                                      sample_offset=same.sample_offset)
                _native.check(lib.rn_pt_render(scene.handle, ctypes.byref(cam), ctypes.byref(st), flags | extra,
                                               sptr, ctypes.c_void_p(out.data_ptr())), "rn_pt_render")
            l2.zero_()
            one()  # warm-up (captures the wavefront graph for this frame shape)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ts = []
            for _ in range(2):
                l2.zero_()
                e0.record(stream)
                one()
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            compare[name] = samples_per_step / (min(ts) / 1e3)
            if fp64 is not None:
                rmse_by[name] = rmse_of(out.cpu().numpy())
    compare["wavefront_over_megakernel"] = compare["wavefront"] / compare["megakernel"]
    compare["auto_choice"] = {1: "megakernel", 2: "wavefront"}.get(tuned["integrator"], "?")
    compare["auto_samples_per_wave"] = tuned["samples_per_wave"]
    compare["auto_ray_fetch"] = "per-lane refetch" if tuned["dynamic_fetch"] else "one ray per lane"
    compare["auto_ray_binning"] = bool(tuned["ray_sort"])

    # End to end through the C ABI with host buffers: pinned host output, D2H inside the timed region.
    host = torch.empty(H * W * 3, dtype=torch.float32, pin_memory=True)
    hflags = 0
    e2e_steps = max(1, min(args.steps, 3))
    # one untimed call first: the host-buffer path captures its own frame graph once
    _native.check(lib.rn_pt_render(scene.handle, ctypes.byref(cam), ctypes.byref(settings()), hflags, None,
                                   ctypes.c_void_p(host.data_ptr())), "rn_pt_render (host)")
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        st = settings()
        _native.check(lib.rn_pt_render(scene.handle, ctypes.byref(cam), ctypes.byref(st), hflags, None,
                                       ctypes.c_void_p(host.data_ptr())), "rn_pt_render (host)")
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = max_over_ranks([e2e_s], dist, "cuda")[0]
    e2e_value = world * samples_per_step / e2e_s

    # RMSE of one frame against the FP64 reference on its pixel subset (when available).
    rmse = rmse_of(host.numpy())
    at_rmse = None
    if rmse_by:
        # Same samples, same estimator: both integrators reach the same RMSE at 64 spp, so
        # their times to that RMSE are their frame times.
        at_rmse = {"relative_rmse_64spp": rmse_by, "frame_ms": {k: samples_per_step / compare[k] * 1e3
                                                                for k in rmse_by},
                   "wavefront_speedup_at_equal_rmse": compare["wavefront"] / compare["megakernel"]}

    # Per-stage device times of the same frame, launched kernel by kernel with CUDA
    # events between the stages (the timed frames above replay the captured graph).
    st_prof = rn.Settings.make(spp=spp, max_depth=args.depth, rr_depth=args.rr, integrator=integ, seed=1,
                               sample_offset=same.sample_offset)
    with torch.cuda.stream(stream):
        l2.zero_()
        torch.cuda.synchronize()
        _, stages = scene.profile_wavefront(cam, st_prof)
    peaks = read_peaks(lib, stream, sptr)
    t_rmse = None
    if fp64 is not None:
        t_rmse = time_to_rmse(scene, lib, stream, sptr, cam, args, fp64, W, H)

    grad = None
    if not args.no_grad:
        grad = gradient_timing(scene, lib, stream, sptr, l2)
    like_for_like = reference_semantics_rate(sc, W, H, args)

    peak, peak_kind = measured_peaks()
    kernel_ms = float(np.mean(render_ms))
    achieved = bytes_per_sample * samples_per_step / (kernel_ms / 1e3) / 1e9
    kp = kernel_profile() or {}
    # DRAM bytes of the frame's three stage kernels (about 93 % of its device time),
    # per sample from the committed ncu capture of the same scene at 480x270
    stage_bps = sum(kp[k]["dram_bytes_per_sample"] for k in ("k_wf_extend", "k_wf_shadow", "k_wf_shade") if k in kp)
    traffic = stage_bps * samples_per_step if stage_bps else None
    # Traversal kernels against the level that holds their working set (the 4-wide tree
    # and the triangles, ~150 MB, mostly L1/L2-resident): algorithmic bytes of the
    # reference traversal per stage over the stage's device time.
    ext_bps = (24.0 * counts["closest_boxes"] + 36.0 * counts["closest_tris"]) / counts["samples"]
    sh_bps = (24.0 * counts["any_boxes"] + 36.0 * counts["any_tris"]) / counts["samples"]
    per_kernel = {}
    for name, bps, ms_key in (("k_wf_extend", ext_bps, "extend_ms"), ("k_wf_shadow", sh_bps, "shadow_ms")):
        ms = stages[ms_key]
        gbs = bps * samples_per_step / (ms / 1e3) / 1e9 if ms > 0 else None
        ent = {"ms_per_frame": ms, "launches_per_frame": args.depth, "share_of_frame": ms / stages["total_ms"],
               "algorithmic_bytes_per_sample": bps, "achieved_gbs": gbs,
               "frac_of_l2_read": gbs / peaks["l2_read_gbs"] if gbs else None,
               "frac_of_hbm": gbs / peak if gbs else None}
        if name in kp:
            ent["ncu"] = {k: v for k, v in kp[name].items() if k != "per_launch"}
        per_kernel[name] = ent
    top = per_kernel["k_wf_extend"]
    top_traffic = None
    if "k_wf_extend" in kp and kp["k_wf_extend"].get("dram_bytes_per_sample"):
        top_traffic = kp["k_wf_extend"]["dram_bytes_per_sample"] * samples_per_step / args.depth
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": spp, "max_depth": args.depth,
                   "rr_depth": args.rr, "triangles": info["num_triangles"], "integrator": args.integrator,
                   "traversal": "reference order and arithmetic (closest hits bit-exact)", "l2": "flushed (256 MB write) before each step",
                   "parallelism": f"{world} independent ranks, disjoint sample indices"},
        "gpu_launches": launches_per_step * args.steps,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": ctypes.sizeof(cam) + ctypes.sizeof(st),
                "d2h_bytes_per_step": H * W * 3 * 4, "api": "rn_pt_render with host output buffer"},
        "roofline": {"bound": "l2", "kernel": "k_wf_extend", "achieved": top["achieved_gbs"],
                     "peak": peaks["l2_read_gbs"], "unit": "GB/s", "frac": top["frac_of_l2_read"],
                     "peak_kind": "measured in this run: L2-resident read (rn_pt_probe_read, loads bypassing L1)",
                     "traffic": top_traffic,
                     "algorithmic": "24 B per node-box test + 36 B per triangle test of the reference-order "
                                    "closest-hit traversal, counted on the GPU for 1 spp of the same frame",
                     "kernel_ms_per_launch": top["ms_per_frame"] / args.depth,
                     "hbm": {"peak": peak, "peak_kind": peak_kind, "frac": top["frac_of_hbm"],
                             "read_probe_gbs": peaks["hbm_read_gbs"]},
                     "issue": ({"bound_by": "L1 throughput and instruction issue (profiles/traversal_kernels_*.md, "
                                            "profiles/k_wf_extend_*.md)",
                                "issue_active_pct": kp["k_wf_extend"]["issue_active_pct"],
                                "issue_active_pct_bounces_0_2": float(np.mean(
                                    [l["issue_pct"] for l in kp["k_wf_extend"]["per_launch"][:3]])),
                                "threads_per_instruction": kp["k_wf_extend"]["threads_per_instruction"]}
                               if "k_wf_extend" in kp else None),
                     "per_kernel": per_kernel,
                     "stages_ms": stages,
                     "frame": {"achieved": achieved, "bytes_per_sample": bytes_per_sample, "kernel_ms": kernel_ms,
                               "frac_of_l2_read": achieved / peaks["l2_read_gbs"], "frac_of_hbm": achieved / peak,
                               "dram_traffic_stage_kernels": traffic},
                     "probes": peaks},
        "time_to_rmse": t_rmse,
        "clocks": clk,
        "rmse_vs_fp64_64spp": rmse,
        "at_equal_rmse": at_rmse,
        "path_vertices_per_s": value * counts["closest"] / counts["samples"],
        "gradient": grad,
        "reference_semantics_gpu": like_for_like,
        "integrators_samples_per_s": compare,
        "scene_build_ms": info["build_ms"],
    }
    line["config"]["reference_semantics"] = (
        "the reference arm (bench.py --impl reference) and cpu_baseline time the reference's renderPathTraced, "
        "which runs the reference's estimator (depth 4, the default disk light with 9 shadow rays per diffuse "
        "vertex, 8-bit canvas) on this geometry and camera; this line's value runs the physical estimator "
        "(depth 8, emitter next-event estimation, Russian roulette). Like for like: reference_semantics_gpu "
        "(the drop-in rn_render path tracer on the same frame) against cpu_baseline, in like_for_like")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sc)
        line["cpu_physical_fp32"] = cpu_physical_baseline(sc, c, args)
        line["like_for_like"] = {
            "reference_semantics": {"gpu_samples_per_s": like_for_like["value"],
                                    "reference_cpu_samples_per_s": line["cpu_baseline"]["value"],
                                    "speedup": like_for_like["value"] / line["cpu_baseline"]["value"]},
            "physical_estimator": {"gpu_samples_per_s": value,
                                   "oracle_fp32_cpu_samples_per_s": line["cpu_physical_fp32"]["value"],
                                   "speedup": value / line["cpu_physical_fp32"]["value"]}}
    if rank == 0 and world == 1 and not args.no_extra:
        # the other two throughput workloads: 64 scenes in one batched launch, and
        # 16-view inverse rendering (200 Adam steps)
        line["batch64"] = measure_batch64(3, 1)
        line["inverse_rendering"] = measure_inverse(args.inverse_steps)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def measure_batch64(steps: int, warmup: int) -> dict:
    """The 64-scene batch: one batched launch (autotuned, normally the wavefront in
    one captured graph) against one megakernel launch per job, same samples."""
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import _native, scenes

    torch.cuda.set_device(0)
    specs = scenes.batch_jobs()
    t0 = time.perf_counter()
    keep, jobs = [], []
    for j in specs:
        sc = scenes.soup_scene(j["triangles"], j["soup_seed"])
        s = rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                                 material=sc["material"], material_param=sc["material_param"])
        s.prepare()
        keep.append(s)
        c = scenes.camera(j["width"], j["height"])
        cam = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], j["width"], j["height"])
        jobs.append((s, cam, rn.Settings.make(spp=j["spp"], max_depth=j["max_depth"], seed=3)))
    build_s = time.perf_counter() - t0
    samples = sum(j["width"] * j["height"] * j["spp"] for j in specs)
    lib = _native.load()
    stream = torch.cuda.Stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    outs = [torch.empty(c.height * c.width * 3, device="cuda") for _, c, _ in jobs]
    ptrs = (ctypes.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    l2 = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    res = {}
    for name, integ in (("batched", _native.RN_PT_AUTO), ("megakernel_per_job", _native.RN_PT_MEGAKERNEL)):
        t0 = time.perf_counter()
        b = rn.Batch(jobs, integrator=integ)
        tune_s = time.perf_counter() - t0
        ts = []
        with torch.cuda.stream(stream):
            for i in range(warmup + steps):
                l2.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                _native.check(lib.rn_pt_batch_render(b._handle, i * 64, _native.RN_PT_DEVICE_POINTERS, sptr, ptrs),
                              "rn_pt_batch_render")
                e1.record(stream)
                torch.cuda.synchronize()
                if i >= warmup:
                    ts.append(e0.elapsed_time(e1))
        res[name] = {"samples_per_s": samples / (float(np.mean(ts)) / 1e3), "ms_per_frame": float(np.mean(ts)),
                     "integrator": {1: "megakernel", 2: "wavefront"}.get(b.integrator, "?"), "create_s": tune_s}
        b.close()
    for s in keep:
        s.close()
    del l2, outs
    torch.cuda.empty_cache()
    return {"metric": METRIC, "value": res["batched"]["samples_per_s"], "unit": UNIT,
            "config": {"workload": "batch of 64 scenes (room + soup of 1e3-5e5 triangles), 256x256/512x384/"
                                   "1024x768, 4-64 spp, depth 6", "triangles": sum(j["triangles"] for j in specs),
                       "samples_per_frame": samples, "scene_build_s": build_s, "l2": "flushed before each frame",
                       "steps": steps, "warmup": warmup},
            "integrators": res,
            "batched_over_per_job_megakernel": res["batched"]["samples_per_s"] /
                                               res["megakernel_per_job"]["samples_per_s"]}


def run_batch64(args):
    r = measure_batch64(args.steps, args.warmup)
    line = {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": r["config"], "integrators": r["integrators"],
            "batched_over_per_job_megakernel": r["batched_over_per_job_megakernel"]}
    print(json.dumps(line), flush=True)


def observed_pixels(scene, views) -> np.ndarray:
    """Per-triangle count of pixel centres whose primary ray hits it first, over the
    views (the GPU's closest-hit query on pinhole rays through the pixel centres)."""
    counts = np.zeros(scene.triangle_count, np.int64)
    for v in views:
        w, h = v["width"], v["height"]
        pos = np.asarray(v["position"], np.float64)
        f = np.asarray(v["target"], np.float64) - pos
        f /= np.linalg.norm(f)
        r = np.cross(f, np.asarray(v["up"], np.float64))
        r /= np.linalg.norm(r)
        u = np.cross(r, f)
        th = math.tan(math.radians(v["vfov_deg"]) / 2)
        ys, xs = np.mgrid[0:h, 0:w]
        sx = ((xs + 0.5) / w) * 2 - 1
        sy = 1 - ((ys + 0.5) / h) * 2
        d = f + r * (sx * th * (w / h))[..., None] + u * (sy * th)[..., None]
        d /= np.linalg.norm(d, axis=-1, keepdims=True)
        o = np.broadcast_to(pos, d.shape)
        idx, _, _, _ = scene.trace_closest(o.reshape(-1, 3), d.reshape(-1, 3))
        counts += np.bincount(idx[idx >= 0], minlength=counts.size)
    return counts


def measure_inverse(steps: int) -> dict:
    """Multi-view albedo recovery: 16 views of the 36-triangle box at 384x384, 16 spp
    primal + 16 spp adjoint, depth 5, Adam (lr 0.02) from the unperturbed albedo
    towards targets rendered with albedo perturbed by N(0, 0.1) clipped to [0.05, 0.95].
    The albedo error is reported over all reflecting triangles and split by whether a
    triangle is seen directly by any of the 16 views: 13 of the 34 are not (the boxes'
    bottoms, backs and the sides that face the walls), and reach the images only
    through interreflections, whose gradients at 16 spp carry little signal."""
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import scenes
    from rednoise_b200.inverse import AlbedoFit

    torch.cuda.set_device(0)
    sc = scenes.cornell_box()
    rng = np.random.default_rng(0x5EED0005)
    truth = np.clip(sc["albedo"] + rng.normal(0.0, 0.1, sc["albedo"].shape), 0.05, 0.95).astype(np.float32)
    views = scenes.views()
    tgt_scene = rn.Scene.from_arrays(sc["vertices"], albedo=truth, emission=sc["emission"],
                                     material=sc["material"], material_param=sc["material_param"])
    targets = []
    for v in views:
        cam = rn.Camera.make(v["position"], v["target"], v["up"], v["vfov_deg"], v["width"], v["height"])
        targets.append(tgt_scene.render_physical(cam, rn.Settings.make(spp=256, max_depth=5, seed=77)))
    scene = rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                                 material=sc["material"], material_param=sc["material_param"])
    seen = observed_pixels(scene, views) > 0
    refl = sc["emission"].sum(1) == 0
    fit = AlbedoFit(scene, views, targets, sc["albedo"], spp=16, max_depth=5, lr=0.02)
    rmse0 = float(np.sqrt(((sc["albedo"][refl] - truth[refl]) ** 2).mean()))
    fit.step()  # warm-up: graph capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(fit.stream)
    losses = fit.run(steps - 1)
    e1.record(fit.stream)
    torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / max(steps - 1, 1)
    tp, ta = [], []
    for k in range(3):
        a0, a1, a2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a0.record(fit.stream)
        fit.render(sample_offset=100_000 + 64 * k)
        a1.record(fit.stream)
        fit.adjoint(sample_offset=200_000 + 64 * k)
        a2.record(fit.stream)
        torch.cuda.synchronize()
        tp.append(a0.elapsed_time(a1))
        ta.append(a1.elapsed_time(a2))
    alb = fit.albedo.detach().cpu().numpy()
    batch_integrator = fit.batch.integrator
    fit.close()

    def rmse(a, m):
        return float(np.sqrt(((a[m] - truth[m]) ** 2).mean())) if m.any() else None

    obs, hid = refl & seen, refl & ~seen
    return {"metric": "ms per inverse-rendering step", "value": ms_step, "unit": "ms",
            "config": {"workload": "16 views x 384x384 of the 36-triangle box, 16 spp primal + 16 spp adjoint, "
                                   "depth 5, Adam lr 0.02 on per-triangle albedo", "adam_steps": steps,
                       "batch_integrator": {1: "megakernel", 2: "wavefront"}.get(batch_integrator, "?")},
            "albedo_rmse": {"all_reflecting": {"triangles": int(refl.sum()), "initial": rmse0,
                                               "final": rmse(alb, refl)},
                            "seen_by_a_view": {"triangles": int(obs.sum()), "initial": rmse(sc["albedo"], obs),
                                               "final": rmse(alb, obs)},
                            "seen_by_no_view": {"triangles": int(hid.sum()), "initial": rmse(sc["albedo"], hid),
                                                "final": rmse(alb, hid)}},
            "loss_first": losses[0] if losses else None, "loss_last": losses[-1] if losses else None,
            "primal_ms": float(np.median(tp)), "adjoint_ms": float(np.median(ta)),
            "adjoint_over_primal": float(np.median(ta)) / float(np.median(tp))}


def run_inverse(args):
    r = measure_inverse(args.inverse_steps)
    line = dict(r)
    line.update({"n_gpus": 1, "steps": args.inverse_steps, "warmup": 1, "higher_is_better": False, "dtype": "f32",
                 "data": "synthetic"})
    print(json.dumps(line), flush=True)


def run_raytraced(args):
    """Whitted ray tracing (rn_render(RN_RAYTRACED) semantics: Phong, default disk
    light, depth 4) of the 1.31M-triangle scene at the bench resolution, through
    the C ABI with a host output canvas, against the reference renderRaytraced on
    the host cores (one frame of the same camera)."""
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import scenes

    torch.cuda.set_device(0)
    sc = scenes.icosphere_scene(level=args.level)
    s = rn.Scene.from_arrays(sc["vertices"], ref_rgb=sc["ref_rgb"], ref_material=sc["ref_material"],
                             ref_roughness=sc["ref_roughness"])
    s.prepare()
    W, H = args.width, args.height
    pos = (0.0, 0.0, scenes.CAMERA_Z)
    focal = reference_focal(H)
    for _ in range(args.warmup):
        s.render_raytraced(W, H, focal_length=focal, position=pos)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.render_raytraced(W, H, focal_length=focal, position=pos)
    gpu_s = (time.perf_counter() - t0) / args.steps
    model = reference_model(sc)
    w, h = W, H
    t0 = time.perf_counter()
    model.render_raytraced(w, h, focal=reference_focal(h), pos=pos)
    cpu_s = time.perf_counter() - t0
    build = reference_bvh_build_s(model)
    cpu_rate = w * h / max(cpu_s - build, 1e-9)
    line = {"metric": "pixels/s (Whitted ray tracing, end to end through the C ABI)", "value": W * H / gpu_s,
            "unit": "pixels/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": gpu_s * 1e3,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"icosphere-cornell-1.31M-tris {W}x{H} renderRaytraced (Phong, default light, "
                                   "depth 4)", "output": "host canvas, copy included"},
            "cpu_baseline": {"value": cpu_rate, "unit": "pixels/s", "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"reference renderRaytraced, one {w}x{h} frame of the same camera "
                                       f"({cpu_s:.1f} s, its BVH rebuild of {build:.2f} s excluded)"}}
    print(json.dumps(line), flush=True)


def run_photon(args):
    """Photon mapping (renderPhotonMapped: 200 000 photons from the default light,
    gather radius 0.25, no final gather) of the 1.31M-triangle scene at the bench
    resolution, through the C ABI with a host output canvas, against the reference
    on the host cores (one frame)."""
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import scenes

    torch.cuda.set_device(0)
    sc = scenes.icosphere_scene(level=args.level)
    s = rn.Scene.from_arrays(sc["vertices"], ref_rgb=sc["ref_rgb"], ref_material=sc["ref_material"],
                             ref_roughness=sc["ref_roughness"])
    s.prepare()
    W, H = args.width, args.height
    pos = (0.0, 0.0, scenes.CAMERA_Z)
    focal = reference_focal(H)
    photons = 200000
    for _ in range(args.warmup):
        s.render_photon_mapped(W, H, photons, focal_length=focal, position=pos)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        img, stored = s.render_photon_mapped(W, H, photons, focal_length=focal, position=pos, return_count=True)
    gpu_s = (time.perf_counter() - t0) / args.steps
    model = reference_model(sc)
    t0 = time.perf_counter()
    want = model.render_photon_mapped(W, H, photons, focal=focal, pos=pos)
    cpu_s = time.perf_counter() - t0
    build = reference_bvh_build_s(model)
    same = float((img == want).mean())
    line = {"metric": "frames/s (photon mapping, end to end through the C ABI)", "value": 1.0 / gpu_s,
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": gpu_s * 1e3,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"icosphere-cornell-1.31M-tris {W}x{H} renderPhotonMapped, {photons} photons",
                       "stored_photons": stored, "output": "host canvas, copy included"},
            "identical_pixels_vs_reference": same,
            "cpu_baseline": {"value": 1.0 / max(cpu_s - build, 1e-9), "unit": "frames/s", "cores": os.cpu_count(),
                             "kind": "reference",
                             "sample": f"reference renderPhotonMapped, one frame ({cpu_s:.1f} s, its BVH rebuild of "
                                       f"{build:.2f} s excluded)"}}
    print(json.dumps(line), flush=True)


def run_lbvh(args):
    """The GPU-built linear BVH on the 1.31M-triangle scene: build time (with the
    vertex upload) against the reference-tree build on the host threads, and the
    bench frame rendered on each tree (nearest-first traversal on both)."""
    import torch

    import rednoise_b200 as rn
    from rednoise_b200 import scenes

    torch.cuda.set_device(0)
    sc = scenes.icosphere_scene(level=args.level)
    s = rn.Scene.from_arrays(sc["vertices"], albedo=sc["albedo"], emission=sc["emission"],
                             material=sc["material"], material_param=sc["material_param"])
    s.prepare()
    host_ms = s.info()["build_ms"]
    builds = [s.build_lbvh() for _ in range(args.warmup + args.steps)][args.warmup:]
    W, H, spp = args.width, args.height, args.spp
    c = scenes.camera(W, H)
    cam = rn.Camera.make(c["position"], c["target"], c["up"], c["vfov_deg"], W, H)
    st = rn.Settings.make(spp=spp, max_depth=args.depth, rr_depth=args.rr, seed=1)
    rates = {}
    for name, kw in (("reference_tree_nearest", dict(nearest_first=True)), ("lbvh", dict(lbvh=True))):
        s.autotune(cam, st, nearest_first=True) if name != "lbvh" else None
        s.render_physical(cam, st, **kw)
        t0 = time.perf_counter()
        s.render_physical(cam, st, **kw)
        rates[name] = W * H * spp / (time.perf_counter() - t0)
    line = {"metric": "ms per BVH build (1.31M triangles)", "value": float(np.median(builds)), "unit": "ms",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "icosphere-cornell-1.31M-tris: GPU linear BVH build, upload included"},
            "reference_tree_host_build_ms": host_ms,
            "frame_samples_per_s": rates}
    print(json.dumps(line), flush=True)


def cornell_pair():
    """The reference's Cornell box (assets/cornell-box.obj at scale 0.35, as its app
    loads it; a committed fixture) as a GPU scene and as a reference model."""
    import oracle

    import rednoise_b200 as rn

    a = np.load(os.path.join(ROOT, "tests", "golden", "assets_ref.npz"))
    s = rn.Scene.from_arrays(a["cornell_v"], ref_rgb=a["cornell_rgb"], ref_material=a["cornell_material"],
                             ref_normal=a["cornell_normal"], ref_roughness=a["cornell_roughness"])
    s.prepare()
    m = oracle.RefModel.from_arrays(a["cornell_v"], a["cornell_rgb"], a["cornell_material"], a["cornell_roughness"],
                                    a["cornell_normal"])
    return s, m


def time_calls(fn, warmup, steps):
    for _ in range(warmup):
        fn()
    t0 = time.perf_counter()
    for _ in range(steps):
        out = fn()
    return (time.perf_counter() - t0) / steps, out


def run_bidirectional(args):
    """Bidirectional path tracing (renderBidirectional: 64 spp, exposure 40) of the
    reference's Cornell box at 640x480 with the reference's camera, through the C
    ABI with a host canvas: the reference row streams (the reference's canvas) and
    the counter streams, against the reference on the host cores (one frame)."""
    import torch

    torch.cuda.set_device(0)
    s, m = cornell_pair()
    W, H, spp = (160, 120, 16) if args.small else (640, 480, 64)
    ref_s, img = time_calls(lambda: s.render_bidirectional(W, H, spp), args.warmup, args.steps)
    ctr_s, _ = time_calls(lambda: s.render_bidirectional(W, H, spp, rng="counter"), args.warmup, args.steps)
    t0 = time.perf_counter()
    want = m.render_bidirectional(W, H, spp)
    cpu_s = time.perf_counter() - t0
    line = {"metric": "frames/s (bidirectional path tracing, end to end through the C ABI)", "value": 1.0 / ref_s,
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ref_s * 1e3,
            "higher_is_better": True, "dtype": "f32", "data": "reference asset (Cornell box, 32 triangles)",
            "config": {"workload": f"cornell-box {W}x{H} renderBidirectional, {spp} spp, exposure 40, camera (0,0,4)",
                       "rng": "reference per-row std::mt19937 streams", "output": "host canvas, copy included"},
            "samples_per_s": W * H * spp / ref_s,
            "identical_pixels_vs_reference": float((img == want).mean()),
            "counter_stream": {"value": 1.0 / ctr_s, "unit": "frames/s", "ms_per_step": ctr_s * 1e3,
                               "samples_per_s": W * H * spp / ctr_s},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "frames/s", "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"reference renderBidirectional (oracle/_ref, OpenMP), one frame ({cpu_s:.2f} s)"}}
    print(json.dumps(line), flush=True)


def run_metropolis(args):
    """Primary-sample Metropolis light transport (renderMetropolis: 4 000 000
    mutations, 100 000 bootstrap paths, exposure 16) of the reference's Cornell box
    at 640x480, through the C ABI with a host canvas, against the reference on the
    host cores (one frame)."""
    import torch

    torch.cuda.set_device(0)
    s, m = cornell_pair()
    W, H, muts = (160, 120, 400000) if args.small else (640, 480, 4000000)
    gpu_s, img = time_calls(lambda: s.render_metropolis(W, H, muts), args.warmup, args.steps)
    big_s, _ = time_calls(lambda: s.render_metropolis(W, H, 16 * muts), 1, 1)
    t0 = time.perf_counter()
    want = m.render_metropolis(W, H, muts)
    cpu_s = time.perf_counter() - t0
    ch = lambda c: np.stack([(c >> 16) & 255, (c >> 8) & 255, c & 255], -1).astype(np.float64)  # noqa: E731
    line = {"metric": "frames/s (Metropolis light transport, end to end through the C ABI)", "value": 1.0 / gpu_s,
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": gpu_s * 1e3,
            "higher_is_better": True, "dtype": "f32", "data": "reference asset (Cornell box, 32 triangles)",
            "config": {"workload": f"cornell-box {W}x{H} renderMetropolis, {muts} mutations, 100000 bootstrap paths, "
                                   "exposure 16, camera (0,0,4)",
                       "chains": muts // 16, "output": "host canvas, copy included"},
            "mutations_per_s": muts / gpu_s,
            "mutations_per_s_64M": 16 * muts / big_s,
            "mean_level": {"gpu": float(ch(img).mean()), "reference": float(ch(want).mean())},
            "mean_abs_level_difference_vs_reference": float(np.abs(ch(img) - ch(want)).mean()),
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "frames/s", "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"reference renderMetropolis (oracle/_ref, 16 OpenMP chains), one frame "
                                       f"({cpu_s:.2f} s)"}}
    print(json.dumps(line), flush=True)


def run_dropin(args):
    """The drop-in path tracer alone (rn_render's renderPathTraced semantics: depth
    4, the default disk light with its 9 shadow rays per diffuse vertex, per-pixel
    mt19937, 8-bit canvas) on the 1.31M-triangle scene at 1920x1080, 2 spp, through
    the C ABI with a host canvas."""
    import torch

    torch.cuda.set_device(0)
    from rednoise_b200 import scenes

    sc = scenes.icosphere_scene(level=args.level)
    W, H, spp = (480, 270, 1) if args.small else (1920, 1080, 2)
    r = reference_semantics_rate(sc, W, H, args, spp=spp)
    line = {"metric": "samples/s (drop-in path tracer, reference semantics, end to end through the C ABI)",
            "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": 3, "warmup": 1, "ms_per_step": r["ms_per_frame"],
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"icosphere-cornell-1.31M-tris {r['workload']}"}}
    print(json.dumps(line), flush=True)


def main(args=None):
    args = args or parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        spawn_ranks(args.gpus, main, args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "batch64":
        run_batch64(args)
    elif args.workload == "inverse":
        run_inverse(args)
    elif args.workload == "raytraced":
        run_raytraced(args)
    elif args.workload == "photon":
        run_photon(args)
    elif args.workload == "lbvh":
        run_lbvh(args)
    elif args.workload == "bidirectional":
        run_bidirectional(args)
    elif args.workload == "metropolis":
        run_metropolis(args)
    elif args.workload == "dropin":
        run_dropin(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
