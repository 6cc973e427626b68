"""Train the denoiser on pairs this renderer generates and save its weights.

The shipped weights (bluetruthengine_b200/weights/denoiser_mixed.npz) came from two runs on one B200:

    python -m bluetruthengine_b200.train_denoiser --scenes 640 --outdoor 640 --blob 720 --spp-target 4096 \
        --spp-in 1,2,4,8,16,32,64 --steps 40000 --lr 5e-4 --out base.npz
    python -m bluetruthengine_b200.train_denoiser --init base.npz --scenes 200 --outdoor 200 --blob 400 \
        --first-seed 5000 --spp-target 4096 --spp-in 1,2,4,8,16,32,48,64 --steps 60000 --lr 2e-4 \
        --out bluetruthengine_b200/weights/denoiser_mixed.npz

(2000 scenes, 22.4 min of pair rendering and 1.8 min of training; then 800 further scenes, 8.6 min and 2.7 min;
the file's training record holds both runs' settings).

Training scenes are the seeded Cornell-box variants of `scenes.c4_scene` (wall colours, light, boxes,
1-3 dielectric spheres with IOR U[1.3, 1.8], an occasional mirror or microfacet sphere) and, with
--outdoor, sky-lit sphere groups of `scenes.outdoor_scene` (Disney, microfacet, mirror and dielectric
spheres under a procedural sky with a sun) and, with --blob, groups of mirror / dielectric / microfacet blob
meshes under soft-sun skies (`scenes.blob_scene`, the large configuration's kind), all at 256x256;
inputs mix several sample counts (--spp-in, default 2-32 spp) so that one network serves several noise levels;
targets are independent FP64-accumulated long runs.  Training runs in chunks of 250 steps; the weights of the
chunk with the lowest mean loss are kept and saved, and a chunk whose mean loss exceeds 1.5 times the best
(a blow-up: a few batches of bright caustics can throw Adam far off) returns to those weights with half the
step size.  Weights are stored as float16 (`params`) with the training record.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np


def train_chunks(dn, steps, batch, crop, lr, seed, log=lambda m: None, chunk=250, blowup=1.5):
    """Trains `dn` for `steps` steps in chunks of `chunk`, the learning rate a tenth for the last fifth.  Keeps the
    weights of the chunk with the lowest mean loss; a chunk whose mean loss exceeds `blowup` times that best returns
    to those weights (which also clears Adam's moments) with half the learning rate.  Returns (best weights, all
    step losses, best chunk loss, its step, rollbacks)."""
    losses = []
    best, best_p, best_step, rollbacks = float("inf"), None, 0, 0
    for s in range(0, steps, chunk):
        k = min(chunk, steps - s)
        lr_s = lr * (0.1 if s >= 0.8 * steps else 1.0)   # one step decay for the last fifth
        l = np.asarray(dn.train(k, batch=batch, crop=crop, lr=lr_s, seed=seed * 7919 + s))
        losses.extend(l.tolist())
        m = float(np.mean(l))
        log("step %d loss %.5f (%.1f ms / step)" % (s + k, float(np.mean(l[-50:])), dn.last_ms() / k))
        if best_p is not None and m > blowup * best:   # blow-up: back to the best weights, half the step size
            dn.set_params(best_p)
            lr *= 0.5
            rollbacks += 1
            log("step %d: chunk loss %.5f > %.1f x best %.5f; back to the weights of step %d, lr %.3g"
                % (s + k, m, blowup, best, best_step, lr))
            continue
        if m < best:
            best, best_p, best_step = m, dn.params(), s + k
    return (best_p if best_p is not None else dn.params()), losses, best, best_step, rollbacks


def _record(path):
    """The training record stored with a weights file (None when there is none)."""
    if not path:
        return None
    with np.load(path) as z:
        return json.loads(str(z["record"])) if "record" in z else None


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=512, help="Cornell-box scenes (scenes.c4_scene)")
    ap.add_argument("--outdoor", type=int, default=0, help="outdoor sky-lit scenes (scenes.outdoor_scene)")
    ap.add_argument("--first-seed", type=int, default=1000)
    ap.add_argument("--spp-target", type=int, default=2048)
    ap.add_argument("--depth", type=int, default=8, help="max depth of the Cornell-box scenes")
    ap.add_argument("--outdoor-depth", type=int, default=16)
    ap.add_argument("--blob", type=int, default=0, help="blob-instance scenes (scenes.blob_scene)")
    ap.add_argument("--blob-depth", type=int, default=24)
    ap.add_argument("--spp-in", default="2,4,8,16,32", help="input sample counts drawn per scene")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--init", default=None, help="start from these weights (a file written by this trainer)")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "denoiser_mixed.npz"))
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bluetruthengine_b200 as bte
    from bluetruthengine_b200 import scenes
    from bluetruthengine_b200.denoise_data import make_dataset
    from bluetruthengine_b200.denoiser import Denoiser
    log = lambda m: print(m, flush=True)
    r = bte.Renderer()
    paths = [(scenes.c4_scene(args.first_seed + i), args.depth) for i in range(args.scenes)]
    paths += [(scenes.outdoor_scene(args.first_seed + i), args.outdoor_depth) for i in range(args.outdoor)]
    paths += [(scenes.blob_scene(args.first_seed + i), args.blob_depth) for i in range(args.blob)]
    order = np.random.default_rng(args.seed).permutation(len(paths))   # interleave the kinds
    paths = [paths[i] for i in order]
    t0 = time.perf_counter()
    spp_in = tuple(int(x) for x in args.spp_in.split(","))
    noisy, feat, target = make_dataset(r, paths, spp_in_choices=spp_in, spp_target=args.spp_target, depth=args.depth,
                                       seed=args.seed, log=log)
    t_data = time.perf_counter() - t0
    dn = Denoiser()
    dn.init(args.seed)
    if args.init:
        dn.load(args.init)
    dn.set_dataset(noisy, feat, target)
    t1 = time.perf_counter()
    p, losses, best, best_step, rollbacks = train_chunks(dn, args.steps, args.batch, args.crop, args.lr, args.seed, log)
    t_train = time.perf_counter() - t1
    rec = {"scenes": args.scenes, "outdoor": args.outdoor, "outdoor_depth": args.outdoor_depth, "blob": args.blob,
           "blob_depth": args.blob_depth, "spp_in": list(spp_in),
           "first_seed": args.first_seed, "init": os.path.basename(args.init) if args.init else None,
           "init_record": _record(args.init), "spp_target": args.spp_target, "depth": args.depth,
           "steps": args.steps, "batch": args.batch, "crop": args.crop, "lr": args.lr, "seed": args.seed,
           "seconds_data": t_data, "seconds_train": t_train, "loss_first": float(np.mean(losses[:50])),
           "loss_last": float(np.mean(losses[-50:])), "best_chunk_loss": best, "best_step": best_step,
           "rollbacks": rollbacks}
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.savez_compressed(args.out, params=p.astype(np.float16), record=json.dumps(rec))
    log(json.dumps(rec))
    return 0


if __name__ == "__main__":
    sys.exit(main())
