"""Generate the golden vectors under tests/golden/ from the reference's own code.

The reference has no tests or fixtures; these vectors come from its shading
headers (include/rt_*.cuh, include/wavefront/*.cuh) compiled on the host by
oracle/Makefile into oracle/_ref/libbteref.so, driven through
oracle/ref_harness.cpp.  Run from the repository root with the reference tree
present:  python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
OUT = os.path.dirname(os.path.abspath(__file__))

import bluetruthengine_b200 as bte  # noqa: E402
from bluetruthengine_b200 import scenes  # noqa: E402
import oracle as O  # noqa: E402


def bsdf_params():
    out = {}
    for t in (1, 2, 3, 4, 5):
        b = np.zeros(1, dtype=bte.BSDF_DTYPE)[0]
        b["type"] = t
        b["p0"] = [0.7, 0.4, 0.2, 0.3]
        b["p1"] = {1: [0, 0, 0, 0], 2: [1.5, 1.0, 0, 0], 3: [0, 0, 0, 0], 4: [0.2, 1.5, 1.0, 0.3],
                   5: [0.4, 0.5, 0.3, 0.2]}[t]
        b["p2"] = [0.3, 0.5, 0.2, 0.4]
        b["p3"] = [0.5, 0.6, 1.45, 0.0]
        out[t] = b
    return out


def main():
    O.build(ref=True)
    ref = O.Ref()
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rng = np.random.default_rng(2024)
    # hash + xorshift stream (rt_rng.cuh:8-52)
    xs = rng.integers(0, 2 ** 32, size=4096, dtype=np.uint64).astype(np.uint32)
    hashes = np.array([ref.lib.ref_hash_uint(int(x)) for x in xs], dtype=np.uint32)
    seeds = np.concatenate([[0, 1, 0x9e3779b9], xs[:61]]).astype(np.uint32)
    u32 = np.empty((len(seeds), 64), np.uint32)
    f32 = np.empty((len(seeds), 64), np.float32)
    for i, s in enumerate(seeds):
        a, b = np.empty(64, np.uint32), np.empty(64, np.float32)
        ref.lib.ref_rng_stream(C.c_uint32(int(s)), 64, p(a), p(b))
        u32[i], f32[i] = a, b
    np.savez_compressed(os.path.join(OUT, "rng.npz"), hash_in=xs, hash_out=hashes, seeds=seeds, u32=u32, f32=f32)
    # BSDF tables (rt_bsdf.cuh:42-84 dispatch, every type)
    n = 2000
    wi = rng.normal(size=(n, 3)); wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3)); wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    u = rng.uniform(size=(n, 3))
    wi, wo, u = wi.astype(np.float32), wo.astype(np.float32), u.astype(np.float32)
    tables = {"wi": wi, "wo": wo, "u": u}
    helper = O.Oracle(libm=True)
    for t, b in bsdf_params().items():
        tables["params_%d" % t] = np.frombuffer(b.tobytes(), np.uint8)
        tables["eval_%d" % t] = _ref_call(ref, "eval", b, wi, wo)
        tables["pdf_%d" % t] = _ref_call(ref, "pdf", b, wi, wo)
        owo, ow, opdf, oeta = _ref_sample(ref, b, wi, u)
        tables["swo_%d" % t], tables["sw_%d" % t], tables["spdf_%d" % t], tables["seta_%d" % t] = owo, ow, opdf, oeta
    np.savez_compressed(os.path.join(OUT, "bsdf.npz"), **tables)
    # per-sample radiance on the Cornell box and the all-features scene
    for name, path, depth, W in (("cornell", scenes.cornell(), 8, None), ("random", scenes.random_scene(5), 12, None)):
        sc = bte.load_scene(path)
        W, H = sc.width, sc.height
        view = O.SceneView(sc, env_mode=0, oracle=helper, build_accel=False)
        k = 4096 if name == "cornell" else 3072
        pix = rng.choice(W * H, size=k, replace=False).astype(np.uint32)
        smp = rng.integers(0, 64, size=k).astype(np.uint32)
        rad, hl, st = O.render_samples(ref.lib, view, sc.camera, W, H, depth, pix, smp, hit_log=True, prefix="ref_")
        np.savez_compressed(os.path.join(OUT, "%s_samples.npz" % name), pixels=pix, samples=smp, radiance=rad,
                            hits=hl, depth=depth, stats=np.array(st), generator=scenes.GENERATOR_VERSION)
    print("golden vectors written to", OUT)


def _ref_call(ref, what, b, wi, wo):
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    bb = np.ascontiguousarray(np.asarray(b).reshape(1))
    n = len(wi)
    if what == "eval":
        out = np.empty((n, 3), np.float32)
        ref.lib.ref_bsdf_eval(p(bb), p(wi), p(wo), p(out), n)
    else:
        out = np.empty(n, np.float32)
        ref.lib.ref_bsdf_pdf(p(bb), p(wi), p(wo), p(out), n)
    return out


def _ref_sample(ref, b, wi, u):
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    bb = np.ascontiguousarray(np.asarray(b).reshape(1))
    n = len(wi)
    wo = np.empty((n, 3), np.float32); w = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32); eta = np.empty(n, np.float32)
    ref.lib.ref_bsdf_sample(p(bb), p(wi), p(u), p(wo), p(w), p(pdf), p(eta), n)
    return wo, w, pdf, eta


if __name__ == "__main__":
    main()
