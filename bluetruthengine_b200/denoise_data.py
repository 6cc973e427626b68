"""Training pairs and quality measurement for the learned denoiser, all rendered by this renderer.

* `render_pair`: a low-spp input (FP32 running mean, as the renderer accumulates it) with its first-hit
  albedo/normal features, and an independent long-run target (FP64 running sum / samples, from a
  disjoint range of sample indices).
* `reference`: an FP64-accumulated high-spp image of a view.
* `time_to_rel_mse`: wall time (host clock around the renderer calls and the readback, with the device
  time beside it) that plain accumulation needs to reach a relMSE bound against a reference, and the
  same for the denoised low-spp form (render + the renderer's denoise + readback).
"""
from __future__ import annotations

import time

import numpy as np

from . import ENV_ALIAS
from .denoiser import rel_mse

TARGET_SAMPLE_BASE = 1 << 24   # target samples use sample indices disjoint from the inputs'


def _frames(r, W, H, spp_total, spf, depth, env=ENV_ALIAS, aov=False):
    done = 0
    ms = 0.0
    while done < spp_total:
        k = min(spf, spp_total - done)
        r.set_config(samples_per_frame=k, max_depth=depth, rr_start=3, env_sampling=env, use_graph=1)
        r.render(W, H)
        ms += r.stats().msTotal
        done += k
    return ms


def render_input(r, W, H, spp, depth, sample_base=0):
    """(noisy [H,W,3], features [H,W,6], device ms) from `spp` samples starting at `sample_base`."""
    r.set_aov(True)
    r.reset_accumulation(W, H)
    r.set_frame_index(sample_base)
    ms = _frames(r, W, H, spp, min(spp, 64), depth)
    noisy = r.read_accum(W, H).reshape(H, W, 3)
    alb, nrm = r.read_aov(W, H)
    r.set_aov(False)
    return noisy, np.concatenate([alb, nrm], -1), ms


def reference(r, W, H, spp, depth, sample_base=TARGET_SAMPLE_BASE, spf=256):
    """FP64 running sum / spp over `spp` samples starting at `sample_base` -> [H,W,3] float64."""
    r.reset_accumulation(W, H)
    r.set_frame_index(sample_base)
    _frames(r, W, H, spp, spf, depth)
    return r.read_accum_f64(W, H).reshape(H, W, 3) / float(spp)


def render_pair(r, scene, spp_in, spp_target, depth=8):
    W, H = scene.width, scene.height
    r.cleanup()
    r.upload(scene)
    noisy, feat, _ = render_input(r, W, H, spp_in, depth)
    target = reference(r, W, H, spp_target, depth).astype(np.float32)
    return noisy, feat, target


def make_dataset(r, scene_paths, spp_in_choices=(2, 4, 8, 16, 32), spp_target=2048, depth=8, seed=0, log=None):
    """Pairs for every scene; `scene_paths` holds paths (rendered at `depth`) or (path, depth) pairs."""
    from . import load_scene
    rng = np.random.default_rng(seed)
    N = len(scene_paths)
    out = None
    t0 = time.perf_counter()
    for i, p in enumerate(scene_paths):
        p, d = (p, depth) if isinstance(p, str) else p
        sc = load_scene(p)
        spp_in = int(rng.choice(spp_in_choices))
        noisy, feat, target = render_pair(r, sc, spp_in, spp_target, d)
        if out is None:
            H, W = noisy.shape[:2]
            out = (np.empty((N, H, W, 3), np.float32), np.empty((N, H, W, 6), np.float32), np.empty((N, H, W, 3), np.float32))
        out[0][i], out[1][i], out[2][i] = noisy, feat, target
        if log and (i % 64 == 0 or i == N - 1):
            log("scene %d/%d spp_in %d  %.1fs" % (i + 1, N, spp_in, time.perf_counter() - t0))
    return out


def _sync():
    try:
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except ImportError:
        pass


def plain_crossing(r, W, H, ref, bound, depth, step=4, max_spp=1 << 16, env=ENV_ALIAS):
    """Smallest multiple of `step` samples at which progressive plain accumulation (the FP32 running mean
    the renderer keeps, samples 0, 1, 2, ... of every pixel) reaches relMSE <= bound against `ref`.

    The image is rendered `step` samples per frame.  relMSE is evaluated (outside any timing) on a schedule
    that follows the 1/spp convergence of the error: after each evaluation the next one is placed half way
    to the predicted crossing, and once that is within two steps, after every frame.  Returns
    (spp or None, [(spp, relMSE), ...])."""
    r.reset_accumulation(W, H)
    r.set_frame_index(0)
    r.set_config(samples_per_frame=step, max_depth=depth, rr_start=3, env_sampling=env, use_graph=1)
    spp, nxt, curve = 0, step, []
    while spp < max_spp:
        r.render(W, H)
        spp += step
        if spp < nxt:
            continue
        e = rel_mse(r.read_accum(W, H).reshape(H, W, 3), ref)
        curve.append((spp, e))
        if e <= bound:
            return spp, curve
        predicted = spp * e / bound
        gap = max(step, int((predicted - spp) * 0.5) // step * step)
        nxt = spp + (step if predicted - spp <= 2 * step else gap)
    return None, curve


def plain_wall(r, W, H, spp, depth, spf=16, env=ENV_ALIAS):
    """Host wall time (and summed device time) of plain accumulation to `spp` samples: reset, frames of
    `spf` samples, then the FP32 mean read back to the host.  Returns (wall s, device ms, image)."""
    r.set_config(samples_per_frame=min(spf, spp), max_depth=depth, rr_start=3, env_sampling=env, use_graph=1)
    _sync()
    t0 = time.perf_counter()
    r.reset_accumulation(W, H)
    r.set_frame_index(0)
    done, ms = 0, 0.0
    while done < spp:
        k = min(spf, spp - done)
        if k != min(spf, spp):
            r.set_config(samples_per_frame=k, max_depth=depth, rr_start=3, env_sampling=env, use_graph=1)
        r.render(W, H)
        ms += r.stats().msTotal
        done += k
    img = r.read_accum(W, H).reshape(H, W, 3)
    return time.perf_counter() - t0, ms, img


def denoised_wall(r, dn, W, H, spp, depth, env=ENV_ALIAS, max_spf=64):
    """Host wall time of the denoised low-spp form through the renderer API: with the denoiser toggled on,
    reset, frames of up to `max_spf` samples per pixel (one frame up to that size; the renderer denoises
    its running mean with the first-hit albedo/normal features after every frame), and the denoised image
    read back.  Returns (wall s, render ms, denoise ms, denoised image, noisy mean)."""
    spf = min(spp, max_spf)
    r.set_config(samples_per_frame=spf, max_depth=depth, rr_start=3, env_sampling=env, use_graph=1)
    _sync()
    t0 = time.perf_counter()
    r.reset_accumulation(W, H)
    r.set_frame_index(0)
    done, ms_render, ms_denoise = 0, 0.0, 0.0
    while done < spp:
        k = min(spf, spp - done)
        if k != spf:
            r.set_config(samples_per_frame=k, max_depth=depth, rr_start=3, env_sampling=env, use_graph=1)
        r.render(W, H)
        ms_render += r.stats().msTotal
        ms_denoise += dn.last_ms()
        done += k
    out = r.read_denoised(W, H)
    wall = time.perf_counter() - t0
    noisy = r.read_accum(W, H).reshape(H, W, 3)
    return wall, ms_render, ms_denoise, out, noisy


def time_to_rel_mse(r, dn, scene, ref, bound=2e-3, depth=8, step=4, plain_spf=16, plain_max_spp=1 << 16,
                    denoise_spps=(1, 2, 4, 8, 16, 32, 64, 128, 256)):
    """Wall time (and device time) plain accumulation and the denoised low-spp form need to reach
    relMSE <= bound against `ref`, on the uploaded scene's view.  The denoiser weights must be loaded.

    plain: the crossing spp from `plain_crossing`, then that many samples rendered again and timed twice
    (the first run captures the frame graphs; the second is reported as warm).
    denoised: for growing spp, one frame plus the renderer's denoise and readback; each size is timed on
    its first call (graph capture and buffers of a new size included) and again warm.  The first size
    reaching the bound is the result."""
    W, H = scene.width, scene.height
    n_cross, curve = plain_crossing(r, W, H, ref, bound, depth, step=step, max_spp=plain_max_spp)
    plain = None
    if n_cross is not None:
        cold = plain_wall(r, W, H, n_cross, depth, spf=plain_spf)
        warm = plain_wall(r, W, H, n_cross, depth, spf=plain_spf)
        plain = {"spp": n_cross, "wall_ms": warm[0] * 1e3, "wall_ms_first_run": cold[0] * 1e3,
                 "device_ms": warm[1], "rel_mse": rel_mse(warm[2], ref)}
    was_on = r.toggle_denoiser()
    if not was_on:
        raise RuntimeError("denoiser did not turn on")
    rows, den = [], None
    try:
        for n in denoise_spps:
            cold = denoised_wall(r, dn, W, H, n, depth)
            warm = denoised_wall(r, dn, W, H, n, depth)
            row = {"spp": n, "wall_ms": warm[0] * 1e3, "wall_ms_first_call": cold[0] * 1e3,
                   "device_ms_render": warm[1], "device_ms_denoise": warm[2],
                   "rel_mse": rel_mse(warm[3], ref), "rel_mse_input": rel_mse(warm[4], ref)}
            rows.append(row)
            if row["rel_mse"] <= bound:
                den = dict(row)
                break
    finally:
        r.toggle_denoiser()
    res = {"bound": bound, "plain": plain, "denoised": den, "denoised_sweep": rows, "plain_curve": curve}
    if plain and den:
        res["speedup_wall"] = plain["wall_ms"] / den["wall_ms_first_call"]
        res["speedup_wall_warm"] = plain["wall_ms"] / den["wall_ms"]
        res["speedup_device"] = plain["device_ms"] / (den["device_ms_render"] + den["device_ms_denoise"])
    return res
