"""The allocation-free alias-table build (bte_env_build_alias_noalloc).

Some callers cannot allocate device memory when they need new env-map tables
-- a render loop that swaps environment maps between frames, where cudaMalloc
and cudaFree would synchronise the device and stall queued frames, or a host
that has reserved all device memory for its own pool.  This entry point takes
the caller's device buffers and keeps its intermediates in a fixed device
array.  Its tables must equal the ones the allocating path (bte_init_env_map)
builds, on consecutive calls (the array keeps the previous call's contents),
without the device's free memory changing between calls; its FP64 total must
equal the same sum done on the host; and sizes beyond the array must be
refused.  Kept in its own file so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _env(h, w):
    from bluetruthengine_b200 import scenes
    rgba = np.ones((h, w, 4), np.float32)
    rgba[..., :3] = scenes.sky_env(w, h, sun_radius_deg=3.0, sun_radiance=500.0)
    return rgba


def _host_total(rgba):
    """The FP64 total weight as the build forms it: per row, luminance * sin(theta at the row centre) summed
    left to right, then the row sums top to bottom."""
    h, w = rgba.shape[:2]
    t = rgba.astype(np.float64)
    lum = (0.2126 * t[..., 0] + 0.7152 * t[..., 1]) + 0.0722 * t[..., 2]
    st = np.sin(np.pi * (np.arange(h, dtype=np.float64) + 0.5) / h)
    rows = np.cumsum(lum * st[:, None], axis=1)[:, -1]
    return float(np.cumsum(rows)[-1])


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
        free = []
        for call in range(3):
            for o in outs:
                o.fill_(-7)
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info(0)[0])
            rc = lib.bte_env_build_alias_noalloc(C.c_void_p(tex.data_ptr()), w, h,
                                                 *[C.c_void_p(o.data_ptr()) for o in outs], C.c_void_p(0))
            assert rc == 0, lib.bte_last_error()
            torch.cuda.synchronize()
            got = [o.cpu().numpy() for o in outs]
            for k in range(5):
                assert np.array_equal(got[k].view(np.uint32), np.asarray(ref[k]).view(np.uint32)), (call, k)
            assert abs(float(got[4].astype(np.float64).sum()) - 1.0) < 1e-4
            total = _host_total(rgba)
            assert abs(float(got[5][0]) - total) <= 1e-12 * total, (float(got[5][0]), total)
        free.append(torch.cuda.mem_get_info(0)[0])
        assert free[1] == free[2] == free[3], f"device free memory changed across calls: {free}"


def test_noalloc_rejects_oversized_and_misaligned(renderer):
    import torch
    lib = renderer.lib
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    p = C.c_void_p(buf.data_ptr())
    rc = lib.bte_env_build_alias_noalloc(p, 1024, 512, p, p, p, p, p, p, C.c_void_p(0))
    assert rc < 0 and b"exceeds" in lib.bte_last_error()
    rc = lib.bte_env_build_alias_noalloc(p, 0, 16, p, p, p, p, p, p, C.c_void_p(0))
    assert rc < 0
    odd = C.c_void_p(buf.data_ptr() + 4)       # a 4-byte offset: not 8-byte aligned for the FP64 total
    rc = lib.bte_env_build_alias_noalloc(p, 16, 8, p, p, p, p, p, odd, C.c_void_p(0))
    assert rc < 0 and b"aligned" in lib.bte_last_error()


_FRESH = r"""
import ctypes as C, json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import bluetruthengine_b200 as bte
from bluetruthengine_b200 import scenes
lib = bte.load_library(build_if_missing=False)
torch.cuda.set_device(0)
dev = torch.device("cuda", 0)
h, w = 64, 128
rgba = np.ones((h, w, 4), np.float32)
rgba[..., :3] = scenes.sky_env(w, h, sun_radius_deg=3.0, sun_radiance=500.0)
tex = torch.from_numpy(rgba.reshape(-1).copy()).to(dev)
outs = [torch.empty(h, dtype=torch.float32, device=dev), torch.empty(h, dtype=torch.int32, device=dev),
        torch.empty(h * w, dtype=torch.float32, device=dev), torch.empty(h * w, dtype=torch.int32, device=dev),
        torch.empty(h * w, dtype=torch.float32, device=dev), torch.empty(1, dtype=torch.float64, device=dev)]
torch.cuda.synchronize()
res = {"rc": [], "free": []}
for call in range(3):
    if call:
        res["free"].append(torch.cuda.mem_get_info(0)[0])
    res["rc"].append(lib.bte_env_build_alias_noalloc(C.c_void_p(tex.data_ptr()), w, h,
                     *[C.c_void_p(o.data_ptr()) for o in outs], C.c_void_p(0)))
    torch.cuda.synchronize()
res["free"].append(torch.cuda.mem_get_info(0)[0])
got = [o.cpu().numpy() for o in outs]
r = bte.Renderer()
r.init_env_map(rgba, 1.0, 0.0)
ref = r.env_alias_tables(w, h)
res["equal"] = [bool(np.array_equal(got[k].view(np.uint32), np.asarray(ref[k]).view(np.uint32))) for k in range(5)]
print(json.dumps(res))
"""


def test_noalloc_first_call_in_fresh_process():
    """In a new process whose first library call is this entry point (no renderer set-up before it): the call
    succeeds, later calls leave the device's free memory unchanged, and the tables equal the allocating path's."""
    env = dict(os.environ)
    env.setdefault("CUDA_MODULE_LOADING", "LAZY")
    out = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["rc"] == [0, 0, 0]
    assert res["free"][0] == res["free"][1] == res["free"][2], res["free"]
    assert all(res["equal"]), res["equal"]
