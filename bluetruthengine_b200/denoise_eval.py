"""Time to relMSE <= 2e-3: plain accumulation against denoised low-spp, on one view.

    python -m bluetruthengine_b200.denoise_eval --scene cornell --weights bluetruthengine_b200/weights/denoiser_c4.npz

The reference is the FP64-accumulated 16384-spp image of the same view from sample indices disjoint
from the ones timed.  Times are device times (CUDA events) of the frames and of the denoiser.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time


def evaluate(scene_name="cornell", weights=None, ref_spp=16384, depth=8, bound=2e-3, log=None):
    import bluetruthengine_b200 as bte
    from bluetruthengine_b200 import scenes
    from bluetruthengine_b200.denoise_data import reference, time_to_rel_mse
    from bluetruthengine_b200.denoiser import Denoiser
    path = {"cornell": scenes.cornell}[scene_name]()
    sc = bte.load_scene(path)
    r = bte.Renderer()
    r.cleanup()
    r.upload(sc)
    t0 = time.perf_counter()
    ref = reference(r, sc.width, sc.height, ref_spp, depth)
    t_ref = time.perf_counter() - t0
    dn = Denoiser()
    dn.load(weights)
    res = time_to_rel_mse(r, dn, sc, ref, bound=bound, depth=depth)
    res.update({"scene": scene_name, "width": sc.width, "height": sc.height, "depth": depth, "reference_spp": ref_spp,
                "reference_seconds": t_ref})
    if res["plain"] and res["denoised"]:
        res["speedup"] = res["plain"]["ms"] / res["denoised"]["ms"]
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="cornell")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                                      "denoiser_c4.npz"))
    ap.add_argument("--ref-spp", type=int, default=16384)
    ap.add_argument("--depth", type=int, default=8)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    print(json.dumps(evaluate(args.scene, args.weights, args.ref_spp, args.depth)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
