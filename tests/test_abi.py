"""The C-ABI library loads without a GPU and exports every entry point that
include/bte/*.h declares; the launch-parameter layout equals the reference's; a
caller written against the reference's render_kernel.h links, and (on a GPU)
renders the same frames as the C-ABI."""
import os
import re
import subprocess

import pytest

from conftest import ROOT


def _declared():
    d = os.path.join(ROOT, "include", "bte")
    txt = "".join(open(os.path.join(d, f)).read() for f in sorted(os.listdir(d)) if f.endswith(".h"))
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(bte_\w+)\s*\(", txt, re.M)))


@pytest.mark.parametrize("variant", ["fast", "parity"])
def test_library_exports_every_declared_symbol(bte, variant):
    path = bte.library_path(variant)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    decl = _declared()
    assert len(decl) >= 40
    missing = [d for d in decl if d not in exported]
    assert not missing, f"declared but not exported: {missing}"


@pytest.mark.parametrize("variant", ["fast", "parity"])
def test_library_loads_and_reports_errors_without_gpu(bte, variant):
    lib = bte.load_library(variant=variant)
    assert lib.bte_version() == 1
    h = __import__("ctypes").c_void_p()
    assert lib.bte_scene_load(b"/nonexistent/scene.xml", __import__("ctypes").byref(h)) < 0
    assert b"empty or unreadable" in lib.bte_last_error()


def test_pod_layouts_match_reference(bte):
    import numpy as np
    assert bte.TRIANGLE_DTYPE.itemsize == 96     # render_kernel.h:22-26
    assert bte.BSDF_DTYPE.itemsize == 68         # render_kernel.h:88-94
    assert bte.CAMERA_DTYPE.itemsize == 56       # render_kernel.h:33-40
    assert bte.EMITTER_DTYPE.itemsize == 32      # render_kernel.h:44-51
    assert bte.SPOT_DTYPE.itemsize == 48         # render_kernel.h:56-63
    assert np.dtype(bte.RenderConfig).itemsize if hasattr(np, "dtype") else True


def test_launch_params_layout_matches_reference():
    """include/bte/launch_params.h against the reference's own include/optix_launch_params.h and
    include/wavefront/wavefront_buffers.h (compiled on the host with an OptiX-handle shim): the offset and size
    of every field of LaunchParams, WavefrontSoA, WfSceneView and EnvMapData, and the four struct sizes."""
    import ctypes as C
    import numpy as np
    import oracle as O
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libbteref_layout.so")
    if not os.path.exists(lib_path):
        if not O.reference_present():
            import pytest
            pytest.skip("reference tree not present")
        O.build(ref=True)
    lib = C.CDLL(lib_path)
    a, b = np.zeros(512, np.int64), np.zeros(512, np.int64)
    n = lib.ref_layout(a.ctypes.data_as(C.c_void_p), 512)
    m = lib.bte_layout(b.ctypes.data_as(C.c_void_p), 512)
    assert n == m and n > 100
    assert np.array_equal(a[:n], b[:m]), np.where(a[:n] != b[:m])[0]
    assert list(a[n - 4:n]) == [48, 200, 216, 496]


REFERENCE_NAMES = ["cudaInitOptix", "cudaInitScene", "cudaInit", "cudaInitCamera", "cudaInitTriangleEmission",
                   "cudaInitTriangleEmitterFlags", "cudaInitEmitterTable", "cudaInitBsdfs", "cudaInitSpotlights",
                   "cudaInitTextures", "cudaInitMrTextures", "cudaInitEnvMap", "cudaRegisterPBO",
                   "cudaResetAccumulation", "cudaRender", "cudaToggleDenoiser", "cudaSetRenderMode",
                   "cudaGetRenderMode", "cudaCleanup"]


def test_reference_named_cpp_api_links(bte, tmp_path):
    """A caller written against the reference's render_kernel.h (include/render_kernel.h:100-211)
    compiles against bte/render_kernel.h and links with libbte_b200.so."""
    src = tmp_path / "caller.cpp"
    src.write_text('#include "bte/render_kernel.h"\n'
                   'int main(int argc, char**) {\n'
                   '  if (argc > 5) {\n'
                   '    CameraData c{}; cudaInitCamera(c); cudaInitScene(nullptr, 0, nullptr, 0, nullptr, 8, 8);\n'
                   '    cudaInitOptix(); cudaInitEnvMap(nullptr, 0, 0, 0.f, 0.f); cudaSetRenderMode(RenderMode::Wavefront);\n'
                   '    cudaResetAccumulation(8, 8); cudaRender(8, 8); (void)cudaGetRenderMode(); cudaCleanup();\n'
                   '  }\n  return 0;\n}\n')
    lib = bte.library_path("fast")
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(tmp_path / "a.out"),
                        lib, "-Wl,-rpath," + os.path.dirname(lib)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    for name in REFERENCE_NAMES:
        assert name + "(" in out, name


_CALLER = r"""
#include "bte/render_kernel.h"
#include <cstdio>
#include <cstring>
#include <vector>
// A drop-in caller: the scene arrays from the loader, every upload through the reference's function names in
// src/main.cpp's order (:836-930), three cudaRender frames, then the frame and the running mean written out.
int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    BteScene* sc = nullptr;
    if (bte_scene_load(argv[1], &sc) < 0) { std::fprintf(stderr, "%s\n", bte_last_error()); return 3; }
    BteSceneArrays a;
    bte_scene_arrays(sc, &a);
    cudaInitCamera(a.camera);
    cudaInitScene(a.triangles, a.triangleCount, a.materials, a.materialCount, a.triangleMaterialIds, a.width, a.height);
    cudaInitOptix();
    cudaInitTriangleEmission(a.triangleEmission, a.triangleCount);
    cudaInitTriangleEmitterFlags(a.triangleEmitterFlags, a.triangleCount);
    if (a.emitterCount > 0)
        cudaInitEmitterTable(a.emitters, a.emitterCount, a.emitterTriIndices, a.emitterTriIndexCount, a.emitterTriCdf,
                             a.emitterTriCdfCount, a.sceneEmitterCdf);
    else
        cudaInitEmitterTable(nullptr, 0, nullptr, 0, nullptr, 0, nullptr);
    cudaInitBsdfs(a.bsdfs, a.bsdfCount, a.triangleBsdfIds, a.triangleCount);
    cudaInitSpotlights(a.spotlightCount ? a.spotlights : nullptr, a.spotlightCount);
    cudaInitEnvMap(a.envRGBA, a.envWidth, a.envHeight, a.envIntensity, a.envRotationDeg);
    cudaSetRenderMode(RenderMode::Wavefront);
    if (cudaGetRenderMode() != RenderMode::Wavefront) return 4;
    for (int i = 0; i < 3; ++i) cudaRender(a.width, a.height);
    const size_t n = static_cast<size_t>(a.width) * a.height;
    std::vector<uint32_t> fb(n);
    std::vector<float> acc(n * 3);
    if (bte_read_framebuffer(fb.data()) < 0 || bte_read_accum(acc.data()) < 0) return 5;
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 6;
    std::fwrite(fb.data(), 4, n, f);
    std::fwrite(acc.data(), 4, n * 3, f);
    std::fclose(f);
    cudaCleanup();
    bte_scene_free(sc);
    return 0;
}
"""


@pytest.mark.gpu
def test_reference_named_cpp_api_renders(bte, tmp_path):
    """The caller above, compiled against bte/render_kernel.h, linked with the product library and run as its own
    process, renders the Cornell box (three cudaRender frames, the reference's defaults: one path per pixel,
    200 bounces, CDF env sampling); its packed frame and FP32 running mean equal those of the same frames
    through the C-ABI of the same library, bit for bit."""
    import numpy as np
    from bluetruthengine_b200 import scenes
    src = tmp_path / "caller.cpp"
    src.write_text(_CALLER)
    lib = bte.library_path("fast")
    renderer = bte.Renderer(variant="fast")
    exe = tmp_path / "caller"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        lib, "-Wl,-rpath," + os.path.dirname(lib)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    path = scenes.cornell()
    out = tmp_path / "frame.bin"
    run = subprocess.run([str(exe), path, str(out)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, (run.returncode, run.stderr[-2000:])
    sc = bte.load_scene(path)
    W, H = sc.width, sc.height
    data = np.fromfile(str(out), dtype=np.uint32)
    fb_caller, acc_caller = data[:W * H], data[W * H:].view(np.float32).reshape(W * H, 3)
    renderer.cleanup()
    renderer.upload(sc)
    renderer.set_config(samples_per_frame=1, max_depth=200, rr_start=3, env_sampling=bte.ENV_CDF, block_size=128,
                        use_graph=0)
    renderer.reset_accumulation(W, H)
    for _ in range(3):
        renderer.render(W, H)
    fb = renderer.read_framebuffer(W, H).reshape(-1)
    acc = renderer.read_accum(W, H).reshape(-1, 3)
    assert np.array_equal(fb_caller, fb)
    assert np.array_equal(acc_caller.view(np.uint32), acc.view(np.uint32))
    assert float(acc.mean()) > 0.01


@pytest.mark.gpu
def test_launch_params_filled_for_current_frame(bte, renderer, random_scene):
    """bte_get_launch_params after a frame: sizes, counts, camera and frame index as uploaded and rendered, and
    the device arrays it points at hold the uploaded triangles, BSDFs, emission flags and the running mean."""
    import ctypes as C
    import numpy as np
    import torch
    sc = random_scene
    W, H = sc.width, sc.height
    renderer.cleanup()
    renderer.upload(sc)
    renderer.set_config(samples_per_frame=2, max_depth=6, rr_start=3, env_sampling=bte.ENV_CDF)
    renderer.reset_accumulation(W, H)
    renderer.render(W, H)
    renderer.render(W, H)
    buf = (C.c_ubyte * 496)()
    assert renderer.lib.bte_get_launch_params(C.byref(buf)) == 0, renderer.lib.bte_last_error()
    raw = bytes(buf)
    i32 = lambda off: int(np.frombuffer(raw, np.int32, 1, off)[0])  # noqa: E731
    u64 = lambda off: int(np.frombuffer(raw, np.uint64, 1, off)[0])  # noqa: E731
    assert (i32(16), i32(20), i32(24), i32(28)) == (W, H, 0, 4)
    assert raw[32:88] == np.asarray(sc.camera, dtype=bte.CAMERA_DTYPE).tobytes()
    assert u64(88) != 0
    assert i32(104) == sc.triangle_count and i32(120) == len(sc.bsdfs)
    assert i32(168) == len(sc.emitters) and i32(208) == len(sc.spotlights)
    assert raw[288] == (1 if sc.env_rgba is not None else 0)
    if sc.env_rgba is not None:
        assert (i32(248), i32(252)) == (sc.env_rgba.shape[1], sc.env_rgba.shape[0])
    assert i32(296 + 192) == W * H * 2        # wf.maxPaths: paths of the last frame

    def dev(ptr, nbytes):
        class A:
            __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}
        return torch.as_tensor(A(), device="cuda").cpu().numpy().tobytes()

    assert dev(u64(96), sc.triangle_count * 96) == np.ascontiguousarray(sc.triangles).tobytes()
    assert dev(u64(112), len(sc.bsdfs) * 68) == np.ascontiguousarray(sc.bsdfs).tobytes()
    assert dev(u64(144), sc.triangle_count) == np.ascontiguousarray(sc.triangle_emitter_flags, np.uint8).tobytes()
    assert dev(u64(8), W * H * 12) == renderer.read_accum(W, H).astype(np.float32).tobytes()
