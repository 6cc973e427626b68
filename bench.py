#!/usr/bin/env python
"""Benchmark: Msamples/s of the wavefront path tracer at 1920x1080.

Workload (the Disney/env-map configuration): ~1.0M triangles (64 seed-placed
icospheres of subdivision 3-6 on a 200x200 tessellated ground), per-object
Disney BSDFs, a 2048x1024 procedural HDR sky with a 0.5-degree sun of radiance
1e4 sampled through the alias tables, 1920x1080, max depth 16, seeded
synthetic data.  One step = one frame of `--spp` paths per pixel through the
whole hot path (generate, extend, shade, connect, present).

value  samples/s over K steps, device time (CUDA events around each frame,
       inputs resident), max over ranks.
e2e    samples/s through the C-ABI (bte_render + bte_read_framebuffer into a
       host buffer every step), wall clock.
Ranks (torchrun, N>1) render disjoint sample-index ranges of the same view:
weak scaling, no collective on the data path.
`--impl reference` times the reference's own integrator (its shading headers
compiled on the host, oracle/_ref) on all host cores over a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic bytes per unit of work, fixed by the reference's SoA record sizes
# (include/wavefront/wavefront_buffers.h:40-90): path state 69 B, hit 36 B,
# queue entry 4 B, shadow record 44 B.
BYTES_PER_SAMPLE_FIXED = 113      # generate 69+4, present 12+4+24
BYTES_PER_SEGMENT = 251           # extend 64 + shade 182 + 5 scene gathers
BYTES_PER_SHADOW = 112            # 44 W + 44 R + 24 radiance RMW
BYTES_PER_EXTEND_RAY = 64         # extend stage alone: queue 4 + ray 24 + hit 36
BYTES_PER_SHADE_SEGMENT = 182
BYTES_PER_CONNECT_RAY = 68        # 44 R + 24 RMW
# DRAM bytes per frame of each stage kernel on this workload (1920x1080, 2 paths per pixel, depth 16), summed
# over the frame's launches of that kernel from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the
# frame with path-ordered queues, taken before the tail kernel and the register budgets; reported per launch beside
# the algorithmic bytes.
STAGE_DRAM_BYTES_PER_FRAME = {"extend": 726.4e6, "shade": 2915.0e6, "connect": 426.2e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spp", type=int, default=2, help="paths per pixel per step")
    ap.add_argument("--depth", type=int, default=16)
    ap.add_argument("--env", default="alias", choices=["alias", "cdf"])
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="launch kernel by kernel instead of replaying the frame graph")
    ap.add_argument("--no-denoise", action="store_true", help="skip the denoised time-to-relMSE leg")
    ap.add_argument("--no-large", action="store_true", help="skip the 10M-triangle 4K leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-views and multi-scene legs")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def scene_path(args):
    from bluetruthengine_b200 import scenes
    return scenes.disney_spheres(seed=2, width=args.width, height=args.height)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix="bte_clocks_%d_" % self.gpu, suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        try:
            with open(self.path) as f:
                return parse_clock_lines(f)
        except Exception:
            return None
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass


def parse_clock_lines(lines):
    """Median SM clock, the highest max clock and the throttle reasons seen, from nvidia-smi's CSV lines (index,
    clocks.sm, clocks.max.sm, power.draw, active-reasons mask, then hw_slowdown, hw_thermal_slowdown,
    sw_thermal_slowdown and sw_power_cap as "Active" / "Not Active"); None without a sample."""
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in lines:
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx = max(mx, float(f[2]))
        except ValueError:
            continue
        for k, name in enumerate(names):
            if f[5 + k].lower().startswith("active"):
                reasons.add(name)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_bf16_tflops():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured (burst)"
    return 1590.0, "fallback"


# Denoiser FLOPs per pixel (forward): sum over its 3x3 convolutions of 2*9*Cin*Cout / 4^level,
# with the channel counts of bte_denoise.cu (input 16, levels 32/48/64/96/128, output 16).
DENOISER_CONVS = [(16, 32, 0), (32, 32, 0), (32, 48, 1), (48, 48, 1), (48, 64, 2), (64, 64, 2), (64, 96, 3), (96, 96, 3),
                  (96, 128, 4), (128, 128, 4), (224, 96, 3), (96, 96, 3), (160, 64, 2), (64, 64, 2), (112, 48, 1),
                  (48, 48, 1), (80, 32, 0), (32, 32, 0), (32, 16, 0)]
DENOISER_FLOP_PER_PIXEL = sum(2 * 9 * ci * co / 4 ** lv for ci, co, lv in DENOISER_CONVS)


def frame_launches(depth: int, tuning: dict) -> int:
    """Kernels one wavefront frame enqueues (bte_renderer.cu renderFrame / launchBounces): generate and present, an
    extend, shade and connect per bounce, the tail kernel when it is on, one ordered compaction per hand-over of the
    path-ordered bounces (buckets of bounces 0..K-1, queues of bounces 1..K-1; they need material sorting and no ray
    reordering) and two launches (bin scan, scatter) per reordered bounce."""
    n = 2 + 3 * depth + (1 if tuning.get("tailPaths", 0) > 0 else 0)
    sort_bits = tuning.get("raySortBits", 0)
    if sort_bits > 0:
        n += 2 * max(0, min(tuning.get("raySortBounces", 0), depth - 1))
    k = tuning.get("orderBounces", 0) if tuning.get("sortShading", 0) and sort_bits == 0 else 0
    k = max(0, min(k, depth))
    return n + k + max(k - 1, 0)


def e2e_copy_bytes(W: int, H: int, depth: int) -> tuple:
    """Host<->device bytes of one end-to-end step (bte_render + bte_read_framebuffer; bte_renderer.cu renderFrame):
    to the device the frame's 4-byte sample-index base (the camera and scene stay resident; the frame parameters
    travel as kernel arguments); back to the host the RGBA8 frame, the per-bounce extend and shadow-ray counters
    ((depth + 1) 32-bit words each) and the 4-byte error word."""
    return 4, W * H * 4 + 2 * (depth + 1) * 4 + 4


def denoiser_layer_bound_ms(W, H, tflops, gbs):
    """Layer-by-layer roofline of one inference: each convolution takes at least the longer of its FLOPs at the
    tensor peak and its compulsory HBM bytes (the bf16 input read once, the bf16 output written once) at the HBM
    peak.  The full-resolution layers (16-80 channels) are HBM-bound under this bound, the deep ones tensor-bound."""
    Hp = (H + 15) // 16 * 16
    t = 0.0
    for ci, co, lv in DENOISER_CONVS:
        p = (W >> lv) * (Hp >> lv)
        t += max(2 * 9 * ci * co * p / (tflops * 1e12), 2 * (ci + co) * p / (gbs * 1e9))
    return t * 1e3


def batched_views_leg(scene, args):
    """Several camera views of the bench scene in one launch sequence (bte_render_views): 8 seeded views with
    resolutions from {320x240, 640x480, 1280x720, 1920x1080} and 1, 2 or 4 samples per frame, against the
    same views rendered one bte_render at a time."""
    import bluetruthengine_b200 as bte
    r = bte.Renderer()
    base = np.asarray(scene.camera, dtype=bte.CAMERA_DTYPE).copy()
    rng = np.random.default_rng(3)
    sizes = [(320, 240), (640, 480), (1280, 720), (1920, 1080)]
    views = []
    for k in range(8):
        w, h = sizes[rng.integers(0, 4)]
        cam = base.copy()
        cam["origin"] = cam["origin"] + np.float32(0.3 * k) * cam["right"]
        cam["aspect"] = np.float32(w / h)
        views.append((cam, w, h, int(rng.choice([1, 2, 4]))))
    samples = sum(w * h * s for _, w, h, s in views)
    env = bte.ENV_ALIAS if args.env == "alias" else bte.ENV_CDF
    r.set_config(samples_per_frame=1, max_depth=args.depth, rr_start=3, env_sampling=env)
    r.reset_views()
    for _ in range(2):
        r.render_views(views)
    ms = []
    for _ in range(5):
        r.render_views(views)
        ms.append(r.stats().msTotal)
    tb = statistics.median(ms)
    seq = 0.0
    for cam, w, h, spp in views:
        r.init_camera(cam)
        r.set_config(samples_per_frame=spp, max_depth=args.depth, rr_start=3, env_sampling=env, use_graph=1)
        r.reset_accumulation(w, h)
        for _ in range(2):
            r.render(w, h)
        m = []
        for _ in range(5):
            r.render(w, h)
            m.append(r.stats().msTotal)
        seq += statistics.median(m)
    r.reset_views()
    return {"views": [[w, h, s] for _, w, h, s in views], "samples_per_frame": samples,
            "batched_ms": tb, "batched_msamples_per_s": samples / tb / 1e3,
            "one_view_at_a_time_ms": seq, "one_view_at_a_time_msamples_per_s": samples / seq / 1e3}


def multi_scene_leg(scene, args):
    """The batched configuration to completion: the bench scene in slot 0 and five seeded instanced scenes in
    slots 1-5 (2, 8, 20, 40 and 80 placements of 25,000-triangle meshes: 50k to 2M triangles, under the procedural
    sky), each with 8 seeded views from {320x240, 640x480, 1280x720, 1920x1080} (48 views), every view accumulated
    to its own sample count drawn from U{16..256}.  Each batch frame renders every unfinished view with up to 4
    samples per pixel (finished views idle) in one call (one launch of a graph holding each scene's captured view
    frame; a scene whose view set changed is captured again) until every view has its samples.  Host wall clock
    from the first frame to the end of the last, against the same frames done one scene at a time."""
    import time
    import bluetruthengine_b200 as bte
    from bluetruthengine_b200 import scenes
    r = bte.Renderer()
    env = bte.ENV_ALIAS if args.env == "alias" else bte.ENV_CDF
    rng = np.random.default_rng(4)
    sizes = [(320, 240), (640, 480), (1280, 720), (1920, 1080)]
    spf_max = 4
    plan, tris = [], []
    try:
        for slot, n_inst in enumerate([0, 2, 8, 20, 40, 80]):
            r.select_scene(slot)
            sc = scene
            if n_inst:
                sc = bte.load_scene(scenes.large_instanced(seed=10 + slot, width=640, height=480, n_instances=n_inst,
                                                           n_meshes=4, env_w=1024, env_h=512))
                r.cleanup()
                r.upload(sc)
            r.set_config(samples_per_frame=1, max_depth=args.depth, rr_start=3, env_sampling=env, use_graph=1)
            base = np.asarray(sc.camera, dtype=bte.CAMERA_DTYPE).copy()
            views = []
            for k in range(8):
                w, h = sizes[rng.integers(0, 4)]
                cam = base.copy()
                cam["origin"] = cam["origin"] + np.float32(0.3 * k) * cam["right"]
                cam["aspect"] = np.float32(w / h)
                views.append((cam, w, h, int(rng.integers(16, 257))))
            plan.append((slot, views))
            tris.append(int(len(sc.triangles)))
        r.select_scene(0)
        samples = sum(w * h * spp for _, v in plan for _, w, h, spp in v)
        frames = max((spp + spf_max - 1) // spf_max for _, v in plan for _, _, _, spp in v)

        def frame_of(k):
            return [(slot, [(cam, w, h, max(0, min(spf_max, spp - k * spf_max))) for cam, w, h, spp in views])
                    for slot, views in plan]

        def reset():
            for slot, _ in plan:
                r.select_scene(slot)
                r.reset_views()
            r.select_scene(0)

        def batch_run():
            reset()
            t0 = time.perf_counter()
            for k in range(frames):
                r.render_scene_batch([(slot, views) for slot, views in frame_of(k)
                                      if any(spf > 0 for *_, spf in views)])
            return time.perf_counter() - t0

        def serial_run():
            reset()
            t0 = time.perf_counter()
            for k in range(frames):
                for slot, views in frame_of(k):
                    if any(spf > 0 for *_, spf in views):
                        r.select_scene(slot)
                        r.render_views(views)
            r.select_scene(0)
            return time.perf_counter() - t0

        batch_run()   # captures
        tb = min(batch_run() for _ in range(2)) * 1e3
        serial_run()
        ts = min(serial_run() for _ in range(2)) * 1e3
        done = []
        for slot, views in plan:
            r.select_scene(slot)
            for i, (_, w, h, spp) in enumerate(views):
                _, total = r.read_view_accum(i, w, h)
                done.append(bool(np.isfinite(total).all()))
        r.select_scene(0)
    finally:
        for slot in range(1, len(plan)):
            r.select_scene(slot)
            r.reset_views()
            r.cleanup()
        r.select_scene(0)
        r.reset_views()
    return {"scenes": len(plan), "triangles": tris, "views": sum(len(v) for _, v in plan),
            "view_spp": [spp for _, v in plan for *_, spp in v], "samples_to_completion": samples,
            "frames": frames, "max_samples_per_frame_per_view": spf_max,
            "batch_ms_to_completion": tb, "batch_msamples_per_s": samples / tb / 1e3,
            "scene_at_a_time_ms": ts, "scene_at_a_time_msamples_per_s": samples / ts / 1e3,
            "all_views_finite": all(done)}


def denoise_leg():
    """Second half of the metric: wall time to relMSE <= 2e-3 against the FP64 16384-spp image, plain accumulation
    vs denoised low-spp, on the bench view itself (1920x1080 Disney/env-map scene, depth 16) and on the Cornell box
    (256x256, depth 8); host wall clock around the renderer calls and the image readback (first call at a size
    included for the denoised form), device time beside it, the relMSE of every image; plus the denoiser's
    inference time at 1920x1080 against the measured BF16 tensor-core peak."""
    weights = os.path.join(ROOT, "bluetruthengine_b200", "weights", "denoiser_mixed.npz")
    if not os.path.exists(weights):
        return {"unavailable": "no trained weights at bluetruthengine_b200/weights/denoiser_mixed.npz"}
    from bluetruthengine_b200.denoise_eval import evaluate
    from bluetruthengine_b200.denoiser import Denoiser
    out = {"metric": "wall ms to relMSE<=2e-3 vs FP64 16384-spp reference (device ms beside)"}
    for name in ("disney_spheres_1080p", "cornell"):
        res = evaluate(name, weights)
        keep = {k: res[k] for k in ("scene", "width", "height", "depth", "reference_spp", "reference_seconds", "bound",
                                    "reference_floor", "plain", "denoised", "denoised_sweep", "one_time_ms_at_size",
                                    "speedup_wall", "speedup_wall_first_call", "speedup_wall_warm", "speedup_device") if k in res}
        keep["plain_curve"] = res["plain_curve"][:: max(1, len(res["plain_curve"]) // 16)]
        out[name] = keep
    dn = Denoiser()
    dn.load(weights)
    rng = np.random.default_rng(0)
    H, W = 1080, 1920
    rad = rng.exponential(0.5, size=(H, W, 3)).astype(np.float32)
    feat = rng.uniform(0, 1, size=(H, W, 6)).astype(np.float32)
    for _ in range(2):
        dn.denoise(rad, feat)
    ms = []
    for _ in range(5):
        dn.denoise(rad, feat)
        ms.append(dn.last_ms())
    t = statistics.median(ms)
    flops = DENOISER_FLOP_PER_PIXEL * W * ((H + 15) // 16 * 16)
    peak, kind = measured_bf16_tflops()
    hbm, _ = measured_peaks()
    bound = denoiser_layer_bound_ms(W, H, peak, hbm)
    out["inference_1080p"] = {"ms": t, "gflop": flops / 1e9, "tflops": flops / (t / 1e3) / 1e12,
                              "peak_tflops": peak, "peak_source": kind, "frac": flops / (t / 1e3) / 1e12 / peak,
                              "layer_roofline_ms": bound, "layer_roofline_frac": bound / t}
    # one training step (forward, L1 loss, data and weight gradients, Adam) at the training configuration's
    # crop and batch, on a small seeded set of 256x256 images; the trained weights are loaded back afterwards
    n_img, crop, batch, steps = 16, 256, 8, 40
    dn.set_dataset(rng.exponential(0.5, size=(n_img, 256, 256, 3)).astype(np.float32),
                   rng.uniform(0, 1, size=(n_img, 256, 256, 6)).astype(np.float32),
                   rng.exponential(0.5, size=(n_img, 256, 256, 3)).astype(np.float32))
    step_ms = {}
    for kind in (0, 1):   # weight gradients on the warp-level kernel, then on tcgen05 (the default, left set)
        dn.set_wgrad(kind)
        dn.train(5, batch=batch, crop=crop, lr=1e-4, seed=1)
        dn.train(steps, batch=batch, crop=crop, lr=1e-4, seed=2)
        step_ms[kind] = dn.last_ms() / steps
    ms_step = step_ms[1]
    train_flops = 3 * DENOISER_FLOP_PER_PIXEL * batch * crop * crop   # forward + data + weight gradients
    out["training_step"] = {"batch": batch, "crop": crop, "ms_per_step": ms_step,
                            "tflops": train_flops / (ms_step / 1e3) / 1e12,
                            "frac": train_flops / (ms_step / 1e3) / 1e12 / peak,
                            "weight_gradient": "tcgen05", "ms_per_step_wgrad_warp_level": step_ms[0]}
    dn.load(weights)
    return out


class ReferenceCpu:
    """The reference's integrator -- its shading headers compiled on the host (oracle/_ref, -O3, OpenMP
    over all host cores) with the oracle's CPU BVH standing in for OptiX -- on the bench's view.  `scene` is
    the reference loader's flattening of the scene file (oracle.RefScene) or the product loader's identical
    arrays."""

    def __init__(self, scene, args):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        self.O = O
        self.ref = O.Ref(fast=True)
        self.view = O.SceneView(scene, env_mode=0, oracle=O.Oracle(libm=True), build_accel=True)
        self.scene = scene
        self.depth = args.depth
        self.cores = os.cpu_count() or 1
        self.rng = np.random.default_rng(7)
        self.rate = None

    def run(self, n):
        W, H = self.scene.width, self.scene.height
        pix = self.rng.integers(0, W * H, size=n).astype(np.uint32)
        t0 = time.perf_counter()
        _, _, (ext, sh) = self.O.render_samples(self.ref.lib, self.view, self.scene.camera, W, H, self.depth, pix,
                                                np.zeros(n, np.uint32), prefix="ref_", threads=self.cores)
        dt = time.perf_counter() - t0
        self.rate = n / dt
        return n, dt, ext, sh

    def sample(self, seconds):
        """One bounded sample of ~`seconds` of CPU work; returns a cpu_baseline record."""
        if self.rate is None:
            self.run(4096)
        n = int(min(max(self.rate * seconds, 4096), self.scene.width * self.scene.height * 32))
        n, dt, ext, sh = self.run(n)
        return {"value": n / dt / 1e6, "unit": "Msamples/s", "cores": self.cores, "kind": "reference",
                "sample": "%d random pixels x 1 spp of the same %dx%d view, depth %d, CDF env sampling "
                          "(the reference's own), %.1f s" % (n, self.scene.width, self.scene.height, self.depth, dt),
                "extends_per_sample": ext / n, "shadow_rays_per_sample": sh / n}


def cpu_baseline(scene, args, seconds: float):
    return ReferenceCpu(scene, args).sample(seconds)


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    # the scene file flattened by the reference's own loader (src/scene.cpp, tinyobjloader, stb_image compiled
    # from the reference tree), so this arm loads no library of this repository
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    scene = O.RefScene(scene_path(args))
    cpu = ReferenceCpu(scene, args)
    budget = max(2.0, 60.0 / max(args.steps, 1))
    for _ in range(args.warmup):
        cpu.sample(min(budget, 2.0))
    per_step = [cpu.sample(budget) for _ in range(args.steps)]
    val = statistics.median(r["value"] for r in per_step)
    r = per_step[-1]
    out = {"metric": "Msamples/s @1080p", "value": val, "unit": "Msamples/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "disney_spheres_1080p", "width": args.width, "height": args.height,
                      "max_depth": args.depth, "triangles": int(scene.triangle_count)},
           "cpu_baseline": {"value": val, "unit": "Msamples/s", "cores": r["cores"], "kind": "reference",
                            "sample": "per step: " + r["sample"]},
           "e2e": {"value": val, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def run_ours(args):
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    import bluetruthengine_b200 as bte
    scene = bte.load_scene(scene_path(args))
    W, H = scene.width, scene.height
    r = bte.Renderer()
    r.upload(scene)
    env_mode = bte.ENV_ALIAS if args.env == "alias" else bte.ENV_CDF
    r.set_config(samples_per_frame=args.spp, max_depth=args.depth, rr_start=3, env_sampling=env_mode,
                 use_graph=0 if args.no_graph else 1)
    r.reset_accumulation(W, H)
    # disjoint sample ranges per rank (every frame below draws from this rank's range)
    from bluetruthengine_b200 import distributed as D
    r.set_frame_index(D.sample_base(rank, args.steps * 2 + args.warmup + 2, args.spp))
    host_fb = torch.empty(W * H, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)

    def step_e2e():
        r.render(W, H)
        r.lib.bte_read_framebuffer(host_fb.ctypes.data_as(__import__("ctypes").c_void_p))

    for _ in range(args.warmup):
        r.render(W, H)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # --- device-timed region (value) ---
    clocks = Clocks(local)
    clocks.start()
    barrier()
    ms = []
    ext = shd = 0
    for _ in range(args.steps):
        r.render(W, H)
        st = r.stats()
        ms.append(st.msTotal)
        ext += st.extends
        shd += st.shadowRays
    barrier()
    clk = clocks.stop()
    t_dev = D.max_over_ranks(sum(ms) / 1e3, device="cuda") if world > 1 else sum(ms) / 1e3
    samples_per_rank = W * H * args.spp * args.steps
    value = samples_per_rank * world / t_dev / 1e6

    # --- end-to-end through the C-ABI with host buffers ---
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    barrier()
    t_e2e = time.perf_counter() - t0
    if world > 1:
        t_e2e = D.max_over_ranks(t_e2e, device="cuda")
    e2e = samples_per_rank * world / t_e2e / 1e6

    # --- per-stage split (separate, untimed pass) for the roofline of the dominant kernel ---
    r.set_stage_timing(True)
    r.render(W, H)
    st = r.stats()
    r.set_stage_timing(False)
    stages = {"generate": st.msGenerate, "extend": st.msExtend, "shade": st.msShade, "connect": st.msConnect,
              "present": st.msPresent, "tail": st.msTail}
    dom = max((k for k in stages if k != "tail"), key=stages.get)
    launches_per_frame = frame_launches(args.depth, r.tuning())
    ext_f, sh_f = st.extends - st.tailExtends, st.shadowRays - st.tailShadowRays   # rays of the wavefront stages
    bytes_dom = {"extend": ext_f * BYTES_PER_EXTEND_RAY, "shade": ext_f * BYTES_PER_SHADE_SEGMENT,
                 "connect": sh_f * BYTES_PER_CONNECT_RAY, "tail": 0,
                 "generate": W * H * args.spp * 73, "present": W * H * args.spp * 40}[dom]
    launches_dom = 1 if dom in ("generate", "present") else args.depth
    peak, peak_kind = measured_peaks()
    achieved = bytes_dom / (stages[dom] / 1e3) / 1e9      # GB/s over the stage's launches in the frame
    spp_samples = W * H * args.spp
    s_mean = ext / (samples_per_rank)
    r_mean = shd / (samples_per_rank)
    b_sample = BYTES_PER_SAMPLE_FIXED + BYTES_PER_SEGMENT * s_mean + BYTES_PER_SHADOW * r_mean
    out = {"metric": "Msamples/s @1080p", "value": value, "unit": "Msamples/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded procedural scene, no dataset)",
           "config": {"workload": "disney_spheres_1080p", "width": W, "height": H, "spp_per_step": args.spp,
                      "max_depth": args.depth, "triangles": int(scene.triangle_count), "env_sampling": args.env,
                      "l2": "inputs larger than L2 (path state %d MB per step)" % (spp_samples * 150 // (1 << 20)),
                      "parallelism": "replicas over sample ranges x%d" % world,
                      "frame_launch": "stream" if args.no_graph else "cuda graph", "tuning": r.tuning()},
           "e2e": {"value": e2e, "unit": "Msamples/s", "h2d_bytes_per_step": e2e_copy_bytes(W, H, args.depth)[0],
                   "d2h_bytes_per_step": e2e_copy_bytes(W, H, args.depth)[1]},
           "gpu_launches": launches_per_frame * args.steps,
           "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": peak_kind,
                        "traffic": (STAGE_DRAM_BYTES_PER_FRAME[dom] / args.depth
                                    if dom in STAGE_DRAM_BYTES_PER_FRAME and W == 1920 and H == 1080 and args.spp == 2
                                    and args.depth == 16 else None),
                        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this kernel on this "
                                          "workload, per launch: a constant from one capture of the frame with "
                                          "path-ordered queues (before the tail kernel and the register budgets); "
                                          "null on other workloads",
                        "algorithmic_bytes_per_launch": bytes_dom / launches_dom,
                        "stage_ms": stages},
           "path_stats": {"extends_per_sample": s_mean, "shadow_rays_per_sample": r_mean,
                          "bytes_per_sample": b_sample,
                          "whole_frame_hbm_frac": (value * 1e6 / world) * b_sample / (peak * 1e9)}}
    if clk is not None:
        out["clocks"] = clk
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(scene, args, seconds=args.cpu_seconds)
        except Exception as e:  # the baseline is reported, never the product
            out["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0 and world == 1 and not args.no_batch:
        try:
            out["batched_views"] = batched_views_leg(scene, args)
        except Exception as e:
            out["batched_views"] = {"unavailable": str(e)}
        try:
            out["multi_scene"] = multi_scene_leg(scene, args)
        except Exception as e:
            out["multi_scene"] = {"unavailable": str(e)}
    if rank == 0 and not args.no_denoise:
        try:
            out["denoise"] = denoise_leg()
        except Exception as e:
            out["denoise"] = {"unavailable": str(e)}
    if rank == 0 and world == 1 and not args.no_large:
        try:   # the large configuration: 10M triangles, 3840x2160, depth 24, 1 spp + denoise vs 1024-spp plain
            from bluetruthengine_b200.large_eval import run as large_run
            weights = os.path.join(ROOT, "bluetruthengine_b200", "weights", "denoiser_mixed.npz")
            out["large_scene"] = large_run(ref_spp=1024, depth=24, weights=weights, log=lambda m: None)
        except Exception as e:
            out["large_scene"] = {"unavailable": str(e)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
