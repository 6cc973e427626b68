"""The large configuration: 10M triangles (400 instances of eight seeded 25,000-triangle meshes, flattened),
3840x2160, depth 24, mirror / dielectric / microfacet instances under the procedural sky with a soft sun.

    python -m bluetruthengine_b200.large_eval --ref-spp 1024

Reports the BVH build and plain throughput (Msamples/s at 1 spp per frame), then the time to relMSE <= 2e-3
against an FP64 accumulation of `ref-spp` samples from disjoint sample indices, for plain accumulation and for
the denoised low-spp form (the same procedure as the 1080p view: the reference's own error, estimated from its
two halves, is reported and subtracted; plain accumulation that does not cross within `ref-spp` is extrapolated
by the 1/spp law; host wall time around the renderer calls and readback, first call at the size included, with
the device time beside it).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

DENOISE_SPPS = (1, 2, 4, 8, 16, 24, 32, 48, 64, 96, 128)


def run(ref_spp=1024, depth=24, weights=None, log=print, width=3840, height=2160, bound=2e-3):
    import bluetruthengine_b200 as bte
    from bluetruthengine_b200 import ENV_ALIAS, scenes
    from bluetruthengine_b200.denoise_data import reference, time_to_rel_mse
    from bluetruthengine_b200.denoiser import Denoiser
    t0 = time.perf_counter()
    sc = bte.load_scene(scenes.large_instanced(width=width, height=height))
    t_load = time.perf_counter() - t0
    W, H = sc.width, sc.height
    r = bte.Renderer()
    r.cleanup()
    t0 = time.perf_counter()
    r.upload(sc)
    t_upload = time.perf_counter() - t0
    accel = r.accel_info()
    log("loaded %d triangles in %.1fs, upload+build %.1fs, accel %s" % (sc.triangle_count, t_load, t_upload, accel))
    # plain throughput at 1 spp per frame
    r.set_config(samples_per_frame=1, max_depth=depth, rr_start=3, env_sampling=ENV_ALIAS, use_graph=1)
    r.reset_accumulation(W, H)
    for _ in range(2):
        r.render(W, H)
    ms = []
    for _ in range(5):
        r.render(W, H)
        ms.append(r.stats().msTotal)
    st = r.stats()
    t_frame = sorted(ms)[2]
    # the reference and its own error
    t0 = time.perf_counter()
    ref, floor = reference(r, W, H, ref_spp, depth, spf=8, with_floor=True)
    t_ref = time.perf_counter() - t0
    log("reference %d spp: %.1f s wall, its own relMSE about %.3g" % (ref_spp, t_ref, floor))
    dn = Denoiser()
    dn.load(weights)
    res = time_to_rel_mse(r, dn, sc, ref, bound=bound, depth=depth, step=4, plain_spf=8, plain_max_spp=ref_spp,
                          denoise_spps=DENOISE_SPPS, floor=floor, denoise_max_spf=8)
    res.update({"workload": "large_instanced_%dx%d" % (W, H), "triangles": int(sc.triangle_count), "width": W,
                "height": H, "depth": depth, "accel": accel, "seconds_load": t_load, "seconds_upload_build": t_upload,
                "ms_per_frame_1spp": t_frame, "msamples_per_s": W * H / t_frame / 1e3,
                "extends_per_sample": st.extends / st.samples, "shadow_rays_per_sample": st.shadowRays / st.samples,
                "reference_spp": ref_spp, "reference_seconds": t_ref})
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-spp", type=int, default=1024)
    ap.add_argument("--depth", type=int, default=24)
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                                      "denoiser_mixed.npz"))
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    res = run(args.ref_spp, args.depth, weights=args.weights, log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
