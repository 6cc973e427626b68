"""Time to relMSE <= 2e-3: plain accumulation against denoised low-spp, on one view.

    python -m bluetruthengine_b200.denoise_eval --scene disney_spheres_1080p
    python -m bluetruthengine_b200.denoise_eval --scene cornell

Views:
  cornell               the Cornell box, 256x256, max depth 8 (no env map)
  disney_spheres_1080p  the 1920x1080 Disney/env-map scene (~1.04M triangles, 2048x1024 sky with a
                        0.5-degree sun of radiance 1e4), max depth 16, alias-table env sampling

The reference is the FP64-accumulated 16384-spp image of the same view from sample indices disjoint
from the ones timed.  Its own error is estimated from its two halves and reported; every image's relMSE
is given as measured against the reference and less that error (the estimate of its relMSE against the
converged image), and the bound applies to the latter.  Times are host wall clock around the renderer
calls and the image readback, with the device time (CUDA events) beside them.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

VIEWS = {
    "cornell": {"depth": 8, "step": 4, "plain_spf": 16, "ref_spf": 256},
    "disney_spheres_1080p": {"depth": 16, "step": 4, "plain_spf": 16, "ref_spf": 16},
}


def scene_for(name):
    from bluetruthengine_b200 import scenes
    if name == "cornell":
        return scenes.cornell()
    if name == "disney_spheres_1080p":
        return scenes.disney_spheres(seed=2, width=1920, height=1080)
    raise ValueError("unknown view %r (known: %s)" % (name, ", ".join(VIEWS)))


def evaluate(scene_name="disney_spheres_1080p", weights=None, ref_spp=16384, bound=2e-3, log=None):
    import bluetruthengine_b200 as bte
    from bluetruthengine_b200.denoise_data import reference, time_to_rel_mse
    from bluetruthengine_b200.denoiser import Denoiser
    v = VIEWS[scene_name]
    sc = bte.load_scene(scene_for(scene_name))
    r = bte.Renderer()
    r.cleanup()
    r.upload(sc)
    t0 = time.perf_counter()
    ref, floor = reference(r, sc.width, sc.height, ref_spp, v["depth"], spf=v["ref_spf"], with_floor=True)
    t_ref = time.perf_counter() - t0
    if log:
        log("%s: reference of %d spp in %.1f s, its own relMSE about %.3g" % (scene_name, ref_spp, t_ref, floor))
    dn = Denoiser()
    dn.load(weights)
    res = time_to_rel_mse(r, dn, sc, ref, bound=bound, depth=v["depth"], step=v["step"], plain_spf=v["plain_spf"],
                          plain_max_spp=ref_spp, floor=floor)
    res.update({"scene": scene_name, "width": sc.width, "height": sc.height, "depth": v["depth"],
                "triangles": int(sc.triangle_count), "reference_spp": ref_spp, "reference_seconds": t_ref})
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="disney_spheres_1080p", choices=sorted(VIEWS))
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                                      "denoiser_mixed.npz"))
    ap.add_argument("--ref-spp", type=int, default=16384)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    res = evaluate(args.scene, args.weights, args.ref_spp, log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
