"""The C-ABI library loads without a GPU and exports every entry point that
include/bte/render_api.h declares."""
import os
import re
import subprocess

from conftest import ROOT


def _declared():
    txt = open(os.path.join(ROOT, "include", "bte", "render_api.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(bte_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol(bte):
    path = bte.library_path()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    decl = _declared()
    assert len(decl) >= 40
    missing = [d for d in decl if d not in exported]
    assert not missing, f"declared but not exported: {missing}"


def test_library_loads_and_reports_errors_without_gpu(bte):
    lib = bte.load_library()
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
    lib = bte.library_path()
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(tmp_path / "a.out"),
                        lib, "-Wl,-rpath," + os.path.dirname(lib)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    for name in REFERENCE_NAMES:
        assert name + "(" in out, name
