"""The large configuration: 10M triangles (400 instances of eight seeded 25,000-triangle meshes, flattened),
3840x2160, depth 24, mirror / dielectric / microfacet instances under the procedural sky.

    python -m bluetruthengine_b200.large_eval --ref-spp 1024

Reports the BVH build, plain throughput (Msamples/s), 1 spp + denoise against the plain FP64 accumulation
of `ref-spp` samples (from disjoint sample indices) with wall and device times for both, and the relMSE of
plain accumulation at a few sample counts against the same reference.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time


def run(ref_spp=1024, depth=24, spf=8, weights=None, log=print):
    import numpy as np
    import bluetruthengine_b200 as bte
    from bluetruthengine_b200 import ENV_ALIAS, scenes
    from bluetruthengine_b200.denoise_data import render_input, reference
    from bluetruthengine_b200.denoiser import Denoiser, rel_mse
    t0 = time.perf_counter()
    sc = bte.load_scene(scenes.large_instanced())
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
    # 1 spp + denoise
    dn = Denoiser()
    dn.load(weights)
    t0 = time.perf_counter()
    noisy, feat, ms_r = render_input(r, W, H, 1, depth)
    out = dn.denoise(noisy, feat)
    wall_den = time.perf_counter() - t0
    ms_d = dn.last_ms()
    # plain accumulation curve from a disjoint sample range, then the reference
    curve = []
    r.reset_accumulation(W, H)
    r.set_frame_index(1 << 20)
    done, t_plain_ms = 0, 0.0
    for target in (4, 16, 64):
        while done < target:
            k = min(spf, target - done)
            r.set_config(samples_per_frame=k, max_depth=depth, rr_start=3, env_sampling=ENV_ALIAS, use_graph=1)
            r.render(W, H)
            t_plain_ms += r.stats().msTotal
            done += k
        curve.append((done, t_plain_ms, r.read_accum_f64(W, H).reshape(H, W, 3) / done))
    t0 = time.perf_counter()
    ref = reference(r, W, H, ref_spp, depth, spf=spf)
    wall_ref = time.perf_counter() - t0
    res = {"workload": "large_instanced_4k", "triangles": int(sc.triangle_count), "width": W, "height": H,
           "depth": depth, "accel": accel, "seconds_load": t_load, "seconds_upload_build": t_upload,
           "ms_per_frame_1spp": t_frame, "msamples_per_s": W * H / t_frame / 1e3,
           "extends_per_sample": st.extends / st.samples, "shadow_rays_per_sample": st.shadowRays / st.samples,
           "reference": {"spp": ref_spp, "wall_s": wall_ref},
           "denoised_1spp": {"ms_render": ms_r, "ms_denoise": ms_d, "wall_s": wall_den, "rel_mse": rel_mse(out, ref),
                             "rel_mse_input": rel_mse(noisy, ref)},
           "plain": [{"spp": n, "ms": t, "rel_mse": rel_mse(img, ref)} for n, t, img in curve]}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-spp", type=int, default=1024)
    ap.add_argument("--depth", type=int, default=24)
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                                      "denoiser_c4.npz"))
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    res = run(args.ref_spp, args.depth, weights=args.weights, log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
