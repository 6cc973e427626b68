"""Training pairs and quality measurement for the learned denoiser, all rendered by this renderer.

* `render_pair`: a low-spp input (FP32 running mean, as the renderer accumulates it) with its first-hit
  albedo/normal features, and an independent long-run target (FP64 running sum / samples, from a
  disjoint range of sample indices).
* `reference`: an FP64-accumulated high-spp image of a view.
* `time_to_rel_mse`: device time plain accumulation needs to reach a relMSE bound against a reference,
  and device time (render + denoise) the denoised low-spp form needs for the same bound.
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
    from . import load_scene
    rng = np.random.default_rng(seed)
    N = len(scene_paths)
    out = None
    t0 = time.perf_counter()
    for i, p in enumerate(scene_paths):
        sc = load_scene(p)
        spp_in = int(rng.choice(spp_in_choices))
        noisy, feat, target = render_pair(r, sc, spp_in, spp_target, depth)
        if out is None:
            H, W = noisy.shape[:2]
            out = (np.empty((N, H, W, 3), np.float32), np.empty((N, H, W, 6), np.float32), np.empty((N, H, W, 3), np.float32))
        out[0][i], out[1][i], out[2][i] = noisy, feat, target
        if log and (i % 64 == 0 or i == N - 1):
            log("scene %d/%d spp_in %d  %.1fs" % (i + 1, N, spp_in, time.perf_counter() - t0))
    return out


def time_to_rel_mse(r, dn, scene, ref, bound=2e-3, depth=8, plain_spf=16, plain_max_spp=1 << 16,
                    denoise_spps=(1, 2, 4, 8, 16, 32, 64, 128, 256)):
    """Device time for plain accumulation and for denoised low-spp to reach relMSE <= bound."""
    W, H = scene.width, scene.height
    r.cleanup()
    r.upload(scene)
    # plain accumulation (progressive, the running FP32 mean the renderer keeps)
    r.reset_accumulation(W, H)
    t_plain, spp, curve = 0.0, 0, []
    plain = None
    while spp < plain_max_spp:
        r.set_config(samples_per_frame=plain_spf, max_depth=depth, rr_start=3, env_sampling=ENV_ALIAS, use_graph=1)
        r.render(W, H)
        t_plain += r.stats().msTotal
        spp += plain_spf
        e = rel_mse(r.read_accum(W, H).reshape(H, W, 3), ref)
        curve.append((spp, t_plain, e))
        if e <= bound:
            plain = {"spp": spp, "ms": t_plain, "rel_mse": e}
            break
    # denoised: fresh low-spp renders of growing size
    den = None
    rows = []
    for n in denoise_spps:
        noisy, feat, ms_r = render_input(r, W, H, n, depth)
        out = dn.denoise(noisy, feat)
        ms_d = dn.last_ms()
        e = rel_mse(out, ref)
        e_noisy = rel_mse(noisy, ref)
        rows.append({"spp": n, "ms_render": ms_r, "ms_denoise": ms_d, "rel_mse": e, "rel_mse_input": e_noisy})
        if den is None and e <= bound:
            den = {"spp": n, "ms": ms_r + ms_d, "ms_render": ms_r, "ms_denoise": ms_d, "rel_mse": e}
            break
    return {"bound": bound, "plain": plain, "denoised": den, "denoised_sweep": rows,
            "plain_curve": curve[:: max(1, len(curve) // 24)]}
