"""The LBVH's integer work pinned on its own: the 63-bit Morton codes and the stable radix-sort order the GPU
build produces (bte_debug_lbvh_order, the same kernels as bte_init_accel) equal a numpy computation from the
same triangles (oracle.lbvh_morton_order), bit for bit -- on the 1.04M-triangle 1080p bench scene, on a scene
with many triangles sharing one centroid (ties must keep ascending index), and on a flat scene (one axis of
zero extent)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gpu_order(renderer, tris):
    tris = np.ascontiguousarray(tris)
    keys = np.empty(len(tris), np.uint64)
    order = np.empty(len(tris), np.int32)
    rc = renderer.lib.bte_debug_lbvh_order(tris.ctypes.data_as(C.c_void_p), len(tris), keys.ctypes.data_as(C.c_void_p),
                                           order.ctypes.data_as(C.c_void_p))
    assert rc == 0, renderer.lib.bte_last_error()
    return keys, order


def _triangles(bte, rng, n, spread=10.0, flat_axis=None):
    t = np.zeros(n, bte.TRIANGLE_DTYPE)
    base = rng.uniform(-spread, spread, size=(n, 3)).astype(np.float32)
    for k in ("v0", "v1", "v2"):
        t[k] = base + rng.uniform(-0.5, 0.5, size=(n, 3)).astype(np.float32)
        if flat_axis is not None:
            t[k][:, flat_axis] = np.float32(1.25)
    return t


@pytest.mark.parametrize("case", ["bench_scene", "shared_centroids", "flat", "random_scene"])
def test_lbvh_morton_codes_and_sort_match_numpy(renderer, bte, oracle_mod, case):
    rng = np.random.default_rng(11)
    if case == "bench_scene":
        from bluetruthengine_b200 import scenes
        tris = bte.load_scene(scenes.disney_spheres(seed=2)).triangles
    elif case == "random_scene":
        from bluetruthengine_b200 import scenes
        tris = bte.load_scene(scenes.random_scene(5)).triangles
    elif case == "shared_centroids":
        few = _triangles(bte, rng, 500)
        tris = few[rng.integers(0, len(few), size=60000)]      # 60k triangles over 500 distinct ones
    else:
        tris = _triangles(bte, rng, 20000, flat_axis=2)
    keys, order = _gpu_order(renderer, tris)
    ref_keys, ref_order = oracle_mod.lbvh_morton_order(tris)
    bad = np.where(keys != ref_keys)[0]
    assert len(bad) == 0, f"{len(bad)} Morton codes differ; first {bad[:5]}"
    assert np.array_equal(order, ref_order)
    assert len(np.unique(keys)) > 1
    if case == "shared_centroids":   # many equal codes: the stable order (ascending index per code) is checked above
        assert len(np.unique(keys)) <= 500
