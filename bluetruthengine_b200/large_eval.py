"""The large configuration: 10M triangles (400 instances of eight seeded 25,000-triangle meshes, flattened),
3840x2160, depth 24, mirror / dielectric / microfacet instances under the procedural sky.

    python -m bluetruthengine_b200.large_eval --ref-spp 1024

Reports the BVH build, plain throughput (Msamples/s), then 1 spp + denoise against plain accumulation of
`ref-spp` samples in the FP64 accumulator (from disjoint sample indices): host wall time (renderer calls and
image readback; for the denoised form the first call at the size included, and a warm repeat) with the device
time beside it, and the relMSE of every image against that accumulation -- the denoised 1-spp image, its noisy
input, and plain accumulation at 4, 16, 64 and 256 samples -- as measured and less the accumulation's own
error (estimated from its two halves).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time


def run(ref_spp=1024, depth=24, spf=8, weights=None, log=print, width=3840, height=2160):
    import numpy as np  # noqa: F401
    import bluetruthengine_b200 as bte
    from bluetruthengine_b200 import ENV_ALIAS, scenes
    from bluetruthengine_b200.denoise_data import TARGET_SAMPLE_BASE, _sync, denoised_wall
    from bluetruthengine_b200.denoiser import Denoiser, rel_mse
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
    # plain accumulation of ref_spp samples into the FP64 accumulator: the reference, timed as plain's cost
    r.set_config(samples_per_frame=spf, max_depth=depth, rr_start=3, env_sampling=ENV_ALIAS, use_graph=1)
    _sync()
    t0 = time.perf_counter()
    r.reset_accumulation(W, H)
    r.set_frame_index(TARGET_SAMPLE_BASE)
    done, dev_ref, first, half = 0, 0.0, None, 0
    while done < ref_spp:
        r.render(W, H)
        dev_ref += r.stats().msTotal
        done += spf
        if first is None and done >= ref_spp // 2:   # the first half's sum, for the reference's own error
            first, half = r.read_accum_f64(W, H).reshape(H, W, 3).copy(), done
    total = r.read_accum_f64(W, H).reshape(H, W, 3)
    ref = total / float(done)
    wall_ref = time.perf_counter() - t0
    # the reference's own relMSE against the converged image: a quarter of its halves' relMSE to each other
    floor = rel_mse(first / float(half), (total - first) / float(done - half)) / 4.0 if 0 < half < done else 0.0
    log("reference %d spp: %.1f s wall" % (done, wall_ref))
    # plain accumulation from sample 0, relMSE at a few sample counts
    curve = []
    r.set_config(samples_per_frame=4, max_depth=depth, rr_start=3, env_sampling=ENV_ALIAS, use_graph=1)
    r.reset_accumulation(W, H)
    r.set_frame_index(0)
    n, dev_plain = 0, 0.0
    for target in (4, 16, 64, 256):
        while n < target:
            r.render(W, H)
            dev_plain += r.stats().msTotal
            n += 4
        e = rel_mse(r.read_accum(W, H).reshape(H, W, 3), ref)
        curve.append({"spp": n, "device_ms": dev_plain, "rel_mse": e, "rel_mse_less_floor": e - floor})
    # 1 spp + denoise through the renderer
    dn = Denoiser()
    dn.load(weights)
    if not r.toggle_denoiser():
        raise RuntimeError("denoiser did not turn on")
    try:
        cold = denoised_wall(r, dn, W, H, 1, depth)
        warm = denoised_wall(r, dn, W, H, 1, depth)
    finally:
        r.toggle_denoiser()
    res = {"workload": "large_instanced_%dx%d" % (W, H), "triangles": int(sc.triangle_count), "width": W,
           "height": H, "depth": depth, "accel": accel, "seconds_load": t_load, "seconds_upload_build": t_upload,
           "ms_per_frame_1spp": t_frame, "msamples_per_s": W * H / t_frame / 1e3,
           "extends_per_sample": st.extends / st.samples, "shadow_rays_per_sample": st.shadowRays / st.samples,
           "plain_reference": {"spp": done, "wall_ms": wall_ref * 1e3, "device_ms": dev_ref, "own_rel_mse": floor},
           "denoised_1spp": {"wall_ms_first_call": cold[0] * 1e3, "wall_ms": warm[0] * 1e3,
                             "device_ms_render": warm[1], "device_ms_denoise": warm[2],
                             "rel_mse": rel_mse(warm[3], ref), "rel_mse_less_floor": rel_mse(warm[3], ref) - floor,
                             "rel_mse_input": rel_mse(warm[4], ref)},
           "plain_curve": curve}
    res["wall_ratio_plain_reference_to_denoised"] = res["plain_reference"]["wall_ms"] / res["denoised_1spp"]["wall_ms"]
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
