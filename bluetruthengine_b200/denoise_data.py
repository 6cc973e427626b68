"""Training pairs and quality measurement for the learned denoiser, all rendered by this renderer.

* `render_pair`: a low-spp input (FP32 running mean, as the renderer accumulates it) with its albedo/normal
  features, and an independent long-run target (FP64 running sum / samples, from a
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


def reference(r, W, H, spp, depth, sample_base=TARGET_SAMPLE_BASE, spf=256, with_floor=False):
    """FP64 running sum / spp over `spp` samples starting at `sample_base` -> [H,W,3] float64.

    with_floor: also return the reference's own relMSE against the converged image, estimated from its two
    halves A and B (disjoint samples): relMSE(A, B) is about twice the error of a half, four times the error
    of the whole (errors of independent unbiased estimates add, and shrink as 1/spp)."""
    r.reset_accumulation(W, H)
    r.set_frame_index(sample_base)
    half = spp // 2
    _frames(r, W, H, half, spf, depth)
    first = r.read_accum_f64(W, H).reshape(H, W, 3).copy() if with_floor else None
    _frames(r, W, H, spp - half, spf, depth)
    total = r.read_accum_f64(W, H).reshape(H, W, 3)
    ref = total / float(spp)
    if not with_floor:
        return ref
    a, b = first / float(half), (total - first) / float(spp - half)
    return ref, rel_mse(a, b) / 4.0


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


def plain_crossing(r, W, H, ref, bound, depth, step=4, max_spp=1 << 16, env=ENV_ALIAS, floor=0.0):
    """Progressive plain accumulation (the FP32 running mean the renderer keeps, samples 0, 1, 2, ... of every
    pixel, `step` samples per frame) against `ref`, until its relMSE less the reference's own error `floor`
    reaches `bound`, or `max_spp`.  relMSE is evaluated outside the timing, on a schedule that follows the
    1/spp convergence of the error: the next evaluation at most doubles the sample count and stops at 90% of the
    predicted crossing; from there on, after every frame.  Host wall time is summed over the render
    calls alone.  Returns (crossing spp or None, [(spp, wall ms, device ms, relMSE, relMSE - floor), ...])."""
    r.set_config(samples_per_frame=step, max_depth=depth, rr_start=3, env_sampling=env, use_graph=1)
    r.reset_accumulation(W, H)
    r.set_frame_index(0)
    _sync()
    spp, nxt, curve = 0, step, []
    wall, dev = 0.0, 0.0
    while spp < max_spp:
        t0 = time.perf_counter()
        r.render(W, H)
        wall += time.perf_counter() - t0
        dev += r.stats().msTotal
        spp += step
        if spp < nxt and spp < max_spp:
            continue
        e = rel_mse(r.read_accum(W, H).reshape(H, W, 3), ref)
        curve.append((spp, wall * 1e3, dev, e, e - floor))
        if e - floor <= bound:
            return spp, curve
        predicted = spp * max(e - floor, 1e-12) / bound
        if spp >= 0.9 * predicted:
            nxt = spp + step
        else:
            nxt = max(spp + step, min(2 * spp, int(0.9 * predicted)) // step * step)
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
    its running mean with the albedo/normal features after every frame), and the denoised image
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
                    denoise_spps=(1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256), floor=0.0, denoise_max_spf=64):
    """Wall time (and device time) that plain accumulation and the denoised low-spp form need to reach
    relMSE <= bound against the converged image, on the uploaded scene's view.  The denoiser weights must be
    loaded.  Every image's relMSE against `ref` is reported as measured and less `floor`, the reference's own
    error (`reference(..., with_floor=True)`); the crossing uses the latter.

    plain: one progressive run (`plain_crossing`), its wall time summed over the render calls.  When it does not
    cross within `plain_max_spp`, the spp it needs is extrapolated from the 1/spp law its error follows (the
    median of spp x (relMSE - floor) over the curve's points from 64 spp) and its time from the measured time per
    sample; the result says so.
    denoised: for growing spp, one frame plus the renderer's denoise and readback; each sample count is timed on
    its first call (the renderer's graph capture for a new frame configuration included) and again warm, rendered
    in frames of at most `denoise_max_spf` samples per pixel.  The first sample count reaching the bound is the
    result.  The first point of the sweep also pays the one-time costs of denoising at this image size in this
    process (kernel loading, feature buffers, the denoiser's graph capture: its first call less its warm time);
    every later point's `wall_ms_cold_start` adds them back, and `speedup_wall` is taken against that cold start,
    with the first-call and warm speedups beside it."""
    W, H = scene.width, scene.height
    n_cross, curve = plain_crossing(r, W, H, ref, bound, depth, step=step, max_spp=plain_max_spp, floor=floor)
    last = curve[-1]
    if n_cross is not None:
        plain = {"spp": n_cross, "wall_ms": last[1], "device_ms": last[2], "rel_mse": last[3],
                 "rel_mse_less_floor": last[4], "extrapolated": False}
    else:
        pts = [n * e for n, _, _, _, e in curve if n >= 64 and e > 0]
        c = float(np.median(pts)) if pts else float(last[0] * last[4])
        n_need = c / bound
        plain = {"spp": n_need, "wall_ms": last[1] / last[0] * n_need, "device_ms": last[2] / last[0] * n_need,
                 "extrapolated": True, "fit_spp_times_error": c, "measured_to_spp": last[0],
                 "rel_mse_at_measured": last[3], "rel_mse_less_floor_at_measured": last[4]}
    was_on = r.toggle_denoiser()
    if not was_on:
        raise RuntimeError("denoiser did not turn on")
    rows, den, once = [], None, None
    try:
        for n in denoise_spps:
            cold = denoised_wall(r, dn, W, H, n, depth, max_spf=denoise_max_spf)
            warm = denoised_wall(r, dn, W, H, n, depth, max_spf=denoise_max_spf)
            e, e_in = rel_mse(warm[3], ref), rel_mse(warm[4], ref)
            if once is None:   # the one-time costs of the size, paid by the sweep's first point
                once = max(0.0, cold[0] - warm[0]) * 1e3
                cold_start = cold[0] * 1e3
            else:
                cold_start = cold[0] * 1e3 + once
            row = {"spp": n, "wall_ms": warm[0] * 1e3, "wall_ms_first_call": cold[0] * 1e3,
                   "wall_ms_cold_start": cold_start,
                   "device_ms_render": warm[1], "device_ms_denoise": warm[2], "rel_mse": e,
                   "rel_mse_less_floor": e - floor, "rel_mse_input": e_in, "rel_mse_input_less_floor": e_in - floor}
            rows.append(row)
            if row["rel_mse_less_floor"] <= bound:
                den = dict(row)
                break
    finally:
        r.toggle_denoiser()
    res = {"bound": bound, "reference_floor": floor, "plain": plain, "denoised": den, "denoised_sweep": rows,
           "one_time_ms_at_size": once,
           "plain_curve": [{"spp": n, "wall_ms": w, "device_ms": d, "rel_mse": e, "rel_mse_less_floor": ec}
                           for n, w, d, e, ec in curve]}
    if den:
        res["speedup_wall"] = plain["wall_ms"] / den["wall_ms_cold_start"]
        res["speedup_wall_first_call"] = plain["wall_ms"] / den["wall_ms_first_call"]
        res["speedup_wall_warm"] = plain["wall_ms"] / den["wall_ms"]
        res["speedup_device"] = plain["device_ms"] / (den["device_ms_render"] + den["device_ms_denoise"])
    return res
