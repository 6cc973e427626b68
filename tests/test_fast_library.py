"""The product library (libbte_b200.so: FP32 shading with CUDA's single-precision functions, fused multiply-adds
allowed) against the reference's own integrator.

The parity library (libbte_b200_parity.so) matches the CPU checker bit for bit (test_gpu_parity.py).  The product
library keeps traversal exact (explicitly rounded arithmetic), so for identical rays its hits equal the checker's
bit for bit; its shading differs from the reference's headers compiled on the host (glibc math) by rounding only.
The north-star bound is 1e-4 relative per sample on identical per-pixel streams: at least 99% of samples must lie
within it, and the fraction beyond it (paths whose branch -- a lobe choice, roulette, a grazing hit -- was decided
differently by a last-bit difference, after which the path is a different path) is printed and bounded.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fast(bte):
    return bte.Renderer(variant="fast")


def _rand_rays(rng, n, lo, hi, towards=False):
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = (rng.uniform(lo, hi, size=(n, 3)) - o) if towards else rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return np.concatenate([o, d], axis=1).astype(np.float32)


def _upload(r, scene, env_mode=1, spp=1, depth=12):
    r.cleanup()
    r.set_tuning()
    r.upload(scene)
    r.set_config(samples_per_frame=spp, max_depth=depth, rr_start=3, env_sampling=env_mode)


@pytest.mark.parametrize("scene_name", ["cornell_scene", "random_scene"])
def test_fast_traversal_equals_oracle(request, fast, oracle_mod, scene_name):
    """Closest hit (triangle, t, u, v) and occlusion for 40k rays, one and eight lanes per ray: the product
    library's traversal equals the checker's brute force bit for bit, as the parity library's does."""
    scene = request.getfixturevalue(scene_name)
    _upload(fast, scene)
    orc = oracle_mod.Oracle(libm=False)
    view = oracle_mod.SceneView(scene, oracle=orc, build_accel=False)
    verts = np.concatenate([scene.triangles["v0"], scene.triangles["v1"], scene.triangles["v2"]])
    lo, hi = verts.min(0), verts.max(0)
    rng = np.random.default_rng(5)
    rays = np.concatenate([_rand_rays(rng, 20000, lo, hi), _rand_rays(rng, 20000, lo, hi, towards=True)])
    ot = np.empty(len(rays), dtype=np.int32)
    otuv = np.empty((len(rays), 3), dtype=np.float32)
    orc.lib.or_trace_closest(view.ptr(), rays.ctypes.data_as(C.c_void_p), len(rays), ot.ctypes.data_as(C.c_void_p),
                             otuv.ctypes.data_as(C.c_void_p))
    for lanes in (1, 8):
        gt, gtuv = fast.trace_closest(rays, lanes=lanes)
        assert np.array_equal(gt, ot), f"{np.sum(gt != ot)} triangle mismatches ({lanes} lanes per ray)"
        hit = gt >= 0
        assert np.array_equal(bits(gtuv[hit]), bits(otuv[hit]))
    tmax = rng.uniform(0.0, float(np.linalg.norm(hi - lo)), size=len(rays)).astype(np.float32)
    oo = np.empty(len(rays), dtype=np.uint8)
    orc.lib.or_trace_occluded(view.ptr(), rays.ctypes.data_as(C.c_void_p), tmax.ctypes.data_as(C.c_void_p), len(rays),
                              oo.ctypes.data_as(C.c_void_p))
    assert np.array_equal(fast.trace_occluded(rays, tmax), oo)


def _vs_reference(oracle_mod, g, ghl, scene, W, H, depth, pix, smp, env_mode, label):
    """Per-sample comparison with the reference's headers compiled on the host (glibc math) -- in alias env
    mode, which the reference does not have, with the checker built on glibc math, which equals those headers
    bit for bit in CDF mode.  Returns (fraction beyond 1e-4, fraction of paths whose hit log differs, fraction
    of primary hits that differ)."""
    orc = oracle_mod.Oracle(libm=True)
    if env_mode == 0:
        if not oracle_mod.Ref.available():
            pytest.skip("reference harness not built")
        lib, prefix = oracle_mod.Ref().lib, "ref_"
    else:
        lib, prefix = orc.lib, "or_"
    view = oracle_mod.SceneView(scene, env_mode=env_mode, oracle=orc, build_accel=True)
    r, rhl, _ = oracle_mod.render_samples(lib, view, scene.camera, W, H, depth, pix, smp, prefix=prefix,
                                          hit_log=True)
    rel = np.abs(g - r) / np.maximum(np.abs(r), 1e-3)
    beyond = float((rel.max(1) > 1e-4).mean())
    path_diff = float(np.any(ghl != rhl, axis=1).mean())
    primary_diff = float((ghl[:, 0] != rhl[:, 0]).mean())
    print(f"{label}: {len(g)} samples, beyond 1e-4: {beyond:.4%}, hit logs differing: {path_diff:.4%}, "
          f"primary hits differing: {primary_diff:.4%}, max rel (agreeing paths): "
          f"{float(rel.max(1)[~np.any(ghl != rhl, axis=1)].max()):.3g}")
    return beyond, path_diff, primary_diff


def test_fast_random_scene_vs_reference_headers(fast, oracle_mod, random_scene):
    """All five BSDFs, area light, spotlight and env map (3 paths per pixel, depth 12)."""
    sc = random_scene
    W, H, spp, depth = sc.width, sc.height, 3, 12
    _upload(fast, sc, env_mode=0, spp=spp, depth=depth)
    fast.set_hit_log(True)
    fast.reset_accumulation(W, H)
    fast.render(W, H)
    n = W * H * spp
    g = fast.read_sample_radiance(n)
    ghl = fast.read_hit_log(n * depth).reshape(n, depth)
    fast.set_hit_log(False)
    ghl = np.where(ghl == -16843010, -2, ghl)
    pix = np.tile(np.arange(W * H, dtype=np.uint32), spp)
    smp = np.repeat(np.arange(spp, dtype=np.uint32), W * H)
    beyond, path_diff, primary_diff = _vs_reference(oracle_mod, g, ghl, sc, W, H, depth, pix, smp, 0, "random scene")
    assert beyond < 0.01 and path_diff < 0.01 and primary_diff < 0.001


@pytest.mark.parametrize("env_mode", [0, 1])
def test_fast_bench_scene_subset_vs_reference_headers(fast, oracle_mod, bte, env_mode):
    """The 1920x1080, ~1.04M-triangle Disney/env-map workload at depth 16: a full frame on the product library,
    6000 random pixels re-rendered on the host: CDF env sampling (the reference's own) by the reference's
    headers, alias-table sampling (this library's) by the checker on glibc math."""
    from bluetruthengine_b200 import scenes
    sc = bte.load_scene(scenes.disney_spheres())
    W, H, depth = sc.width, sc.height, 16
    _upload(fast, sc, env_mode=env_mode, spp=1, depth=depth)
    fast.set_hit_log(True)
    fast.reset_accumulation(W, H)
    fast.render(W, H)
    g = fast.read_sample_radiance(W * H)
    ghl = fast.read_hit_log(W * H * depth).reshape(W * H, depth)
    fast.set_hit_log(False)
    ghl = np.where(ghl == -16843010, -2, ghl)
    rng = np.random.default_rng(21 + env_mode)
    pix = rng.choice(W * H, size=6000, replace=False).astype(np.uint32)
    beyond, path_diff, primary_diff = _vs_reference(oracle_mod, g[pix], ghl[pix], sc, W, H, depth, pix,
                                                    np.zeros(len(pix), np.uint32), env_mode,
                                                    "bench scene env_mode=%d" % env_mode)
    assert beyond < 0.01 and path_diff < 0.01 and primary_diff < 0.001


def test_fast_math_is_single_precision_cuda(fast, oracle_mod):
    """The product library's elementary functions are CUDA's single-precision ones: within a few ulp of the
    correctly rounded result (the parity library's portable functions are exact to the last bit instead)."""
    rng = np.random.default_rng(3)
    n = 1 << 16
    cases = {0: (rng.uniform(-20, 20, n), None, np.sin), 1: (rng.uniform(-20, 20, n), None, np.cos),
             3: (rng.uniform(-80, 80, n), None, np.exp), 4: (np.exp(rng.uniform(-60, 60, n)), None, np.log),
             5: (rng.uniform(0.01, 2, n), rng.uniform(-8, 8, n), np.power),
             6: (rng.normal(size=n), rng.normal(size=n), np.arctan2), 7: (rng.uniform(-1, 1, n), None, np.arccos)}
    for fn, (a, b, ref) in cases.items():
        a = a.astype(np.float32)
        b = None if b is None else b.astype(np.float32)
        got = fast.math_eval(fn, a, b).astype(np.float64)
        exact = ref(a.astype(np.float64)) if b is None else ref(a.astype(np.float64), b.astype(np.float64))
        ulp = np.abs(np.spacing(exact.astype(np.float32)).astype(np.float64))
        err = np.abs(got - exact) / ulp
        print("fn", fn, "max ulp error", float(err.max()))
        assert float(err.max()) <= 8.0, fn
