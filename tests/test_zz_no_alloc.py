"""The allocation-free alias-table build (bte_env_build_alias_noalloc).

Some callers cannot allocate device memory when they need new env-map tables
-- a render loop that swaps environment maps between frames, where cudaMalloc
and cudaFree would synchronise the device and stall queued frames, or a host
that has reserved all device memory for its own pool.  This entry point takes
the caller's device buffers and keeps its intermediates in a fixed device
array.  Its tables must equal the ones the allocating path (bte_init_env_map)
builds, on two calls in a row (the array keeps the previous call's contents),
and sizes beyond the array must be refused.  Kept in its own file so a run
that stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _env(h, w):
    from bluetruthengine_b200 import scenes
    rgba = np.ones((h, w, 4), np.float32)
    rgba[..., :3] = scenes.sky_env(w, h, sun_radius_deg=3.0, sun_radiance=500.0)
    return rgba


def test_noalloc_alias_tables_equal_allocating_path(renderer):
    import torch
    lib = renderer.lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    for (h, w) in ((128, 256), (96, 200)):
        rgba = _env(h, w)
        renderer.init_env_map(rgba, 1.0, 0.0)          # the existing (allocating) entry point
        ref = renderer.env_alias_tables(w, h)          # rowProb, rowAlias, colProb, colAlias, pixelPdf
        tex = torch.from_numpy(rgba.reshape(-1).copy()).to(dev)
        outs = [torch.empty(h, dtype=torch.float32, device=dev), torch.empty(h, dtype=torch.int32, device=dev),
                torch.empty(h * w, dtype=torch.float32, device=dev), torch.empty(h * w, dtype=torch.int32, device=dev),
                torch.empty(h * w, dtype=torch.float32, device=dev), torch.empty(1, dtype=torch.float64, device=dev)]
        for call in range(2):
            for o in outs:
                o.fill_(-7)
            torch.cuda.synchronize()
            rc = lib.bte_env_build_alias_noalloc(C.c_void_p(tex.data_ptr()), w, h,
                                                 *[C.c_void_p(o.data_ptr()) for o in outs], C.c_void_p(0))
            assert rc == 0, lib.bte_last_error()
            torch.cuda.synchronize()
            got = [o.cpu().numpy() for o in outs]
            for k in range(5):
                assert np.array_equal(got[k].view(np.uint32), np.asarray(ref[k]).view(np.uint32)), (call, k)
            assert abs(float(got[4].astype(np.float64).sum()) - 1.0) < 1e-4
            assert got[5][0] > 0.0


def test_noalloc_rejects_oversized_maps(renderer):
    import torch
    lib = renderer.lib
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float32, device=dev)
    p = C.c_void_p(buf.data_ptr())
    rc = lib.bte_env_build_alias_noalloc(p, 1024, 512, p, p, p, p, p, p, C.c_void_p(0))
    assert rc < 0 and b"exceeds" in lib.bte_last_error()
    rc = lib.bte_env_build_alias_noalloc(p, 0, 16, p, p, p, p, p, p, C.c_void_p(0))
    assert rc < 0
