"""Build the path tracer's two C-ABI libraries in-tree with nvcc for sm_100a.

Both are plain C-ABI shared libraries (no torch types): CUDA kernels, the C++
host runtime and the scene loader, built from the same sources.

libbte_b200.so         the product.  Shading runs in FP32 with CUDA's own
                       single-precision functions and fused multiply-adds
                       allowed (-fmad=true, IEEE division and square root, no
                       flush-to-zero: nvcc's defaults, the reference's own
                       arithmetic model).  Traversal arithmetic is written with
                       explicitly rounded operations, so hits do not depend on
                       contraction.
libbte_b200_parity.so  the parity build: the stage kernels compiled with
                       -fmad=false and the portable double-evaluated elementary
                       functions, so per-sample results match the CPU checker
                       bit for bit.

Only the translation unit holding the path-tracing kernels (bte_kernels.cu)
differs between them; every other object is compiled once (-fmad=false) and
linked into both.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "libbte_b200.so")
OUT_PARITY = os.path.join(HERE, "libbte_b200_parity.so")
OBJ_DIR = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-std=c++17", "-lineinfo", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
        "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", INCLUDE]
EXACT = BASE + ["-fmad=false"]
FAST = BASE + ["-fmad=true", "-DBTE_FAST_MATH"]
SHARED = ["bte_bvh.cu", "bte_env.cu", "bte_renderer.cu", "bte_scene.cpp", "bte_scene_api.cpp",
          "bte_image.cpp", "bte_output.cpp", "bte_gltf.cpp",
          "bte_compat.cpp", "bte_denoise_kernels.cu", "bte_denoise_tc.cu", "bte_denoise.cu"]
VARIANT = "bte_kernels.cu"
# (object name, source, flags)
UNITS = [(os.path.splitext(s)[0] + ".o", s, EXACT) for s in SHARED] + \
        [("bte_kernels_parity.o", VARIANT, EXACT), ("bte_kernels_fast.o", VARIANT, FAST)]
LIBS = {OUT: "bte_kernels_fast.o", OUT_PARITY: "bte_kernels_parity.o"}


def _compile(unit, verbose: bool) -> str:
    name, src, flags = unit
    obj = os.path.join(OBJ_DIR, name)
    cmd = [NVCC] + ARCH + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + cmd[1:]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}\n{r.stdout}")
    if verbose:
        sys.stderr.write(f"== {name}\n" + r.stderr)
    return obj


def _stale() -> bool:
    for out in LIBS:
        if not os.path.exists(out):
            return True
    t = min(os.path.getmtime(out) for out in LIBS)
    for d in (CSRC, os.path.join(INCLUDE, "bte")):
        for f in os.listdir(d):
            if os.path.getmtime(os.path.join(d, f)) > t:
                return True
    return os.path.getmtime(os.path.abspath(__file__)) > t


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    os.makedirs(OBJ_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = dict(zip([u[0] for u in UNITS], ex.map(lambda u: _compile(u, verbose), UNITS)))
    shared = [objs[os.path.splitext(s)[0] + ".o"] for s in SHARED]
    for out, kernels in LIBS.items():
        tmp = out + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + shared + [objs[kernels]] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}\n{r.stdout}")
        os.replace(tmp, out)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
