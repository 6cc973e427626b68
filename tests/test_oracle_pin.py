"""The oracle is pinned to the reference.

Golden vectors (tests/golden/*.npz) were produced by the reference's own
shading headers compiled on the host (tests/golden/make_golden.py).  The
oracle restatement compiled with glibc math must reproduce them bit-for-bit;
compiled with the portable math that the GPU uses it must agree within the
north-star tolerance (1e-4 relative per sample) with identical hit indices.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, bits

GOLD = os.path.join(ROOT, "tests", "golden")


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def test_hash_and_rng_golden(oracle_mod):
    g = np.load(os.path.join(GOLD, "rng.npz"))
    for libm in (True, False):
        orc = oracle_mod.Oracle(libm=libm)
        h = np.array([orc.hash_uint(int(x)) for x in g["hash_in"]], dtype=np.uint32)
        assert np.array_equal(h, g["hash_out"])
        for i, s in enumerate(g["seeds"]):
            u, f = orc.rng_stream(int(s), 64)
            assert np.array_equal(u, g["u32"][i]) and np.array_equal(bits(f), bits(g["f32"][i]))


@pytest.mark.parametrize("btype", [1, 2, 3, 4, 5])
def test_bsdf_golden(oracle_mod, bte, btype):
    g = np.load(os.path.join(GOLD, "bsdf.npz"))
    b = np.frombuffer(g["params_%d" % btype].tobytes(), dtype=bte.BSDF_DTYPE)[0]
    orc = oracle_mod.Oracle(libm=True)
    wi, wo, u = g["wi"], g["wo"], g["u"]
    assert np.array_equal(bits(orc.bsdf_eval(b, wi, wo)), bits(g["eval_%d" % btype]))
    assert np.array_equal(bits(orc.bsdf_pdf(b, wi, wo)), bits(g["pdf_%d" % btype]))
    owo, ow, opdf, oeta = orc.bsdf_sample(b, wi, u)
    assert np.array_equal(bits(owo), bits(g["swo_%d" % btype]))
    assert np.array_equal(bits(ow), bits(g["sw_%d" % btype]))
    assert np.array_equal(bits(opdf), bits(g["spdf_%d" % btype]))
    assert np.array_equal(bits(oeta), bits(g["seta_%d" % btype]))
    # portable math: same values within 1e-5 relative where finite
    porc = oracle_mod.Oracle(libm=False)
    pe = porc.bsdf_eval(b, wi, wo)
    ref = g["eval_%d" % btype]
    fin = np.isfinite(ref)
    assert np.allclose(pe[fin], ref[fin], rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("name,fixture", [("cornell", "cornell_scene"), ("random", "random_scene")])
def test_samples_golden(request, oracle_mod, name, fixture):
    scene = request.getfixturevalue(fixture)
    g = np.load(os.path.join(GOLD, "%s_samples.npz" % name))
    from bluetruthengine_b200 import scenes
    assert int(g["generator"]) == scenes.GENERATOR_VERSION, "fixtures are stale: rerun tests/golden/make_golden.py"
    depth = int(g["depth"])
    W, H = scene.width, scene.height
    orc = oracle_mod.Oracle(libm=True)
    view = oracle_mod.SceneView(scene, env_mode=0, oracle=orc, build_accel=False)
    rad, hl, st = oracle_mod.render_samples(orc.lib, view, scene.camera, W, H, depth, g["pixels"], g["samples"],
                                            hit_log=True)
    assert np.array_equal(hl, g["hits"])
    assert np.array_equal(bits(rad), bits(g["radiance"]))
    assert tuple(st) == tuple(g["stats"])
    # the GPU's arithmetic (portable math): hits identical, radiance within 1e-4 relative
    porc = oracle_mod.Oracle(libm=False)
    pview = oracle_mod.SceneView(scene, env_mode=0, oracle=porc, build_accel=False)
    prad, phl, _ = oracle_mod.render_samples(porc.lib, pview, scene.camera, W, H, depth, g["pixels"], g["samples"],
                                             hit_log=True)
    rel = np.abs(prad - rad) / np.maximum(np.abs(rad), 1e-3)
    assert (rel.max(1) > 1e-4).mean() <= 0.002
    assert (np.all(phl == hl, axis=1)).mean() >= 0.998


def test_oracle_matches_reference_full_frame(oracle_mod, cornell_scene):
    """Whole Cornell frame: oracle (glibc math) == the reference's headers, bit-for-bit."""
    if not oracle_mod.Ref.available():
        pytest.skip("reference harness not built")
    ref = oracle_mod.Ref()
    orc = oracle_mod.Oracle(libm=True)
    sc = cornell_scene
    W, H = sc.width, sc.height
    view = oracle_mod.SceneView(sc, env_mode=0, oracle=orc, build_accel=False)
    pix = np.arange(W * H, dtype=np.uint32)
    smp = np.full(W * H, 3, dtype=np.uint32)
    a, ha, sa = oracle_mod.render_samples(orc.lib, view, sc.camera, W, H, 8, pix, smp, hit_log=True)
    b, hb, sb = oracle_mod.render_samples(ref.lib, view, sc.camera, W, H, 8, pix, smp, hit_log=True, prefix="ref_")
    assert sa == sb and np.array_equal(ha, hb) and np.array_equal(bits(a), bits(b))


def test_oracle_megakernel_matches_reference(oracle_mod, cornell_scene):
    """Megakernel frames (one RNG stream per pixel through 5 paths, the mean of the five): oracle (glibc math) ==
    the reference's headers, bit-for-bit, for frames 0 and 1 of the Cornell box."""
    if not oracle_mod.Ref.available():
        pytest.skip("reference harness not built")
    ref = oracle_mod.Ref()
    orc = oracle_mod.Oracle(libm=True)
    sc = cornell_scene
    W, H = sc.width, sc.height
    view = oracle_mod.SceneView(sc, env_mode=0, oracle=orc, build_accel=False)
    pix = np.arange(0, W * H, 7, dtype=np.uint32)
    for frame in (0, 1):
        a, sa = oracle_mod.render_megakernel(orc.lib, view, sc.camera, W, H, 8, pix, frame)
        b, sb = oracle_mod.render_megakernel(ref.lib, view, sc.camera, W, H, 8, pix, frame, prefix="ref_")
        assert sa == sb and np.array_equal(bits(a), bits(b))
        assert a.mean() > 0


def test_bvh_traversal_equals_brute_force(oracle_mod, random_scene):
    """The oracle's CPU BVH resolves every closest hit exactly as the exhaustive search does."""
    orc = oracle_mod.Oracle(libm=False)
    brute = oracle_mod.SceneView(random_scene, oracle=orc, build_accel=False)
    bvh = oracle_mod.SceneView(random_scene, oracle=orc, build_accel=True)
    rng = np.random.default_rng(4)
    n = 40000
    o = rng.uniform(-15, 15, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    out = []
    for v in (brute, bvh):
        tri = np.empty(n, np.int32)
        tuv = np.empty((n, 3), np.float32)
        orc.lib.or_trace_closest(v.ptr(), _p(rays), n, _p(tri), _p(tuv))
        out.append((tri, tuv))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(bits(out[0][1]), bits(out[1][1]))


def test_present_welford_and_gamma(oracle_mod):
    """rt_path_integrator.cuh:72-105: Welford mean in FP32 and the gamma-2.2 ABGR pack."""
    if not oracle_mod.Ref.available():
        pytest.skip("reference harness not built")
    ref = oracle_mod.Ref()
    rng = np.random.default_rng(9)
    n = 5000
    acc_o = np.zeros((n, 3), np.float32)
    acc_r = np.zeros((n, 3), np.float32)
    orc = oracle_mod.Oracle(libm=True)
    for f in range(5):
        x = rng.exponential(0.5, size=(n, 3)).astype(np.float32)
        acc_o, po = orc.present(acc_o, x, f)
        pr = np.empty(n, np.uint32)
        ref.lib.ref_present(_p(acc_r), _p(x), n, C.c_uint32(f), _p(pr))
        assert np.array_equal(bits(acc_o), bits(acc_r)) and np.array_equal(po, pr)


def test_textured_scene_matches_reference(oracle_mod, random_scene):
    """Albedo + metallic-roughness textures through the reference's loadBsdfForTriangle
    (rt_material.cuh:15-59) with the documented filter: oracle == reference headers."""
    if not oracle_mod.Ref.available():
        pytest.skip("reference harness not built")
    rng = np.random.default_rng(17)
    tex = [rng.integers(0, 256, size=(19, 23, 4), dtype=np.uint8), rng.integers(0, 256, size=(8, 64, 4), dtype=np.uint8),
           None, None, rng.integers(0, 256, size=(33, 7, 4), dtype=np.uint8)]
    mr = [rng.integers(0, 256, size=(16, 16, 4), dtype=np.uint8), None, None, None, None]
    orc = oracle_mod.Oracle(libm=True)
    ref = oracle_mod.Ref()
    sc = random_scene
    v = oracle_mod.SceneView(sc, env_mode=0, oracle=orc, textures=tex, mr_textures=mr)
    W, H = sc.width, sc.height
    pix = np.arange(W * H, dtype=np.uint32)
    smp = np.full(W * H, 5, np.uint32)
    a, ha, _ = oracle_mod.render_samples(orc.lib, v, sc.camera, W, H, 10, pix, smp, hit_log=True)
    b, hb, _ = oracle_mod.render_samples(ref.lib, v, sc.camera, W, H, 10, pix, smp, hit_log=True, prefix="ref_")
    assert np.array_equal(ha, hb) and np.array_equal(bits(a), bits(b))
