"""Build libbte_b200.so in-tree with nvcc for sm_100a.

The product is a plain C-ABI shared library (no torch types): CUDA kernels,
the C++ host runtime and the scene loader.  Kernels are compiled with
-fmad=false (no implicit multiply-add contraction) because per-sample results
must match the CPU checker bit-for-bit; fused multiply-adds that the
traversal wants are written explicitly.
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
OBJ_DIR = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
          "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", INCLUDE]
SOURCES = ["bte_kernels.cu", "bte_bvh.cu", "bte_env.cu", "bte_renderer.cu", "bte_scene.cpp", "bte_scene_api.cpp",
           "bte_image.cpp", "bte_output.cpp", "bte_gltf.cpp",
           "bte_compat.cpp", "bte_denoise_kernels.cu", "bte_denoise_tc.cu", "bte_denoise.cu"]


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC] + ARCH + COMMON + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + cmd[1:]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}\n{r.stdout}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    for d in (CSRC, os.path.join(INCLUDE, "bte")):
        for f in os.listdir(d):
            if os.path.getmtime(os.path.join(d, f)) > t:
                return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    os.makedirs(OBJ_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    tmp = OUT + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}\n{r.stdout}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
