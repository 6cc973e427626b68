"""Autotuner for the wavefront frame.

Sweeps the knobs that decide throughput on a given scene and GPU:
  * tree width and leaf size (8-wide quantised tree with 1-3 triangles per
    leaf, or the binary LBVH with SAH-collapsed leaves),
  * threads per block of the persistent stage kernels,
  * the shade kernel's register budget (2 or 3 resident blocks of 256
    threads per SM: 96 or 72 registers),
  * the leaf-test postponing threshold of the 8-wide walk,
  * material-sorted shading on or off,
  * the compaction threshold: bounce queues shorter than it finish in the
    tail kernel (one thread per remaining path) instead of the stage kernels,
  * ray reordering before the closest-hit rays of bounces 1-4 (origin cell
    bits per axis; 0 = off) and the 8-wide walk's triangle tests per step
    (0 = all of a node's at once),
  * the leading bounces whose material buckets and queues are rebuilt in
    path order (0 = atomic appends in completion order throughout),
timing whole frames on the device (CUDA events), and leaves the renderer in
the fastest configuration.  Results are deterministic in value (every
configuration renders the same bits); only speed differs.

autotune_denoiser does the same for the learned denoiser: its convolution
kernels (tcgen05 row tiles, row tiles upsampling in-kernel, pixel tiles) timed
on inference at the caller's image size, and optionally the training weight
gradient's kernel (tcgen05 pipeline shapes or the warp-level kernel) timed on
training steps.
"""
from __future__ import annotations

import itertools
import json
from dataclasses import asdict, dataclass


@dataclass
class TuneResult:
    bvh_width: int
    max_leaf: int
    block_size: int
    shade_min_blocks: int
    postpone_percent: int
    sort_shading: int
    tail_paths: int
    ray_sort_bits: int
    leaf_tests_per_step: int
    order_bounces: int
    ms_per_frame: float
    msamples_per_s: float


def autotune(renderer, width: int, height: int, samples_per_frame: int, max_depth: int, env_sampling: int,
             trees=((8, 1), (8, 2), (8, 3), (2, 1)), blocks=(64, 128, 256), shade_min_blocks=(2, 3),
             postpone=(0, 20), sort_shading=(1,), tail_paths=(0, 1 << 14), ray_sort=(0,), leaf_tests=(0,),
             order=(0, 3), frames: int = 3, verbose: bool = False):
    """Blocks run 64 to 256 threads: the stage kernels are compiled for at most 256 threads per block, which
    fixes their register budgets."""
    results = []
    for bvh_width, leaf in trees:
        renderer.set_tuning(leaf, 2, bvh_width)
        renderer.init_accel()
        for blk, smb, pp, srt, tail, rs, lt, ob in itertools.product(blocks, shade_min_blocks,
                                                                     postpone if bvh_width == 8 else (0,),
                                                                     sort_shading, tail_paths, ray_sort,
                                                                     leaf_tests if bvh_width == 8 else (0,), order):
            renderer.set_tuning(leaf, smb, bvh_width, pp, srt, tail, ray_sort_bits=rs, leaf_tests_per_step=lt,
                                order_bounces=ob)
            renderer.set_config(samples_per_frame=samples_per_frame, max_depth=max_depth, rr_start=3,
                                env_sampling=env_sampling, block_size=blk)
            renderer.render(width, height)          # warm-up at this configuration
            ms = 0.0
            for _ in range(frames):
                renderer.render(width, height)
                ms += renderer.stats().msTotal
            ms /= frames
            r = TuneResult(bvh_width, leaf, blk, smb, pp, srt, tail, rs, lt, ob, ms,
                           width * height * samples_per_frame / ms / 1e3)
            results.append(r)
            if verbose:
                print(json.dumps(asdict(r)), flush=True)
    best = min(results, key=lambda r: r.ms_per_frame)
    renderer.set_tuning(best.max_leaf, best.shade_min_blocks, best.bvh_width, best.postpone_percent, best.sort_shading,
                        best.tail_paths, ray_sort_bits=best.ray_sort_bits, leaf_tests_per_step=best.leaf_tests_per_step,
                        order_bounces=best.order_bounces)
    renderer.init_accel()
    renderer.set_config(samples_per_frame=samples_per_frame, max_depth=max_depth, rr_start=3,
                        env_sampling=env_sampling, block_size=best.block_size)
    renderer.reset_accumulation(width, height)
    return best, results


@dataclass
class DenoiserTuneResult:
    kernels: int            # convolution kernels (bte_denoiser_set_tcgen05 mode)
    wgrad: int              # training weight-gradient kernel (bte_denoiser_set_wgrad kind); -1 when not timed
    ms: float               # median device ms: one denoise, or one training step


def autotune_denoiser(dn, width: int, height: int, kernels=(2, 3, 1), wgrad=(1, 3, 4, 5, 6, 7, 0), train_steps: int = 0,
                      batch: int = 8, crop: int = 128, iters: int = 3, seed: int = 0):
    """Times the denoiser's kernel choices on this GPU and leaves the fastest in place.

    Inference: with each convolution-kernel choice (`kernels`, bte_denoiser_set_tcgen05 modes) a seeded
    width x height image is denoised once untimed (the first call at a size records its launch graph), then
    `iters` times; the median device time decides.  Training, when `train_steps` > 0 and a data set is loaded:
    with the chosen convolution kernels, each weight-gradient kernel (`wgrad`, bte_denoiser_set_wgrad kinds: the
    default list is every distinct one, kind 1 being the default pipeline shape of kind 2) runs
    one untimed step and then `train_steps` timed ones, `iters` times.  Training moves the weights, so the weights
    are put back afterwards through set_params, which also restarts Adam: tune before training.  Every choice
    computes the same convolutions (to the tolerance of their tests), so only speed differs.

    Returns (best kernels mode, best weight-gradient kind or None, every result)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    rad = rng.exponential(0.5, size=(height, width, 3)).astype(np.float32)
    feat = rng.uniform(0, 1, size=(height, width, 6)).astype(np.float32)
    results = []
    for mode in kernels:
        dn.set_tcgen05(mode)
        dn.denoise(rad, feat)
        ms = []
        for _ in range(iters):
            dn.denoise(rad, feat)
            ms.append(dn.last_ms())
        results.append(DenoiserTuneResult(mode, -1, float(np.median(ms))))
    best_mode = min((r for r in results if r.wgrad < 0), key=lambda r: r.ms).kernels
    dn.set_tcgen05(best_mode)
    best_kind = None
    if train_steps > 0 and wgrad:
        saved = dn.params()
        try:
            timed = []
            for kind in wgrad:
                dn.set_wgrad(kind)
                dn.train(1, batch=batch, crop=crop, lr=1e-4, seed=seed)
                ms = []
                for _ in range(iters):
                    dn.train(train_steps, batch=batch, crop=crop, lr=1e-4, seed=seed + 1)
                    ms.append(dn.last_ms() / train_steps)
                timed.append(DenoiserTuneResult(best_mode, kind, float(np.median(ms))))
            results += timed
            best_kind = min(timed, key=lambda r: r.ms).wgrad
            dn.set_wgrad(best_kind)
        finally:
            dn.set_params(saved)
    return best_mode, best_kind, results
