"""ORACLE binding (test infrastructure only).

ctypes access to the CPU checker:
  liboracle.so        restatement of the reference's path tracer, portable math
                      (bit-compatible with the GPU kernels)
  liboracle_libm.so   the same restatement with glibc math (bit-compatible with
                      the reference's own headers)
  _ref/libbteref.so   the reference's shading headers compiled on the host
                      (needs the reference tree at build time; the built .so
                      travels with the repository snapshot)
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


# The reference source tree the checker compiles from (read-only); override with BTE_REFERENCE_ROOT.
REFERENCE_ROOT = os.environ.get("BTE_REFERENCE_ROOT", "/root/reference")


def reference_present() -> bool:
    return os.path.isdir(os.path.join(REFERENCE_ROOT, "include"))


def build(ref: bool = True) -> None:
    """Build the oracle libraries (and the reference harness when the reference tree is present)."""
    targets = ["liboracle.so", "liboracle_libm.so"]
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True, env=env)
    if ref and reference_present():
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + REFERENCE_ROOT], check=True, env=env)


class OCamera(C.Structure):
    _fields_ = [("v", C.c_float * 14)]


class OConfig(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("maxDepth", C.c_int), ("rrStart", C.c_int)]


class OStats(C.Structure):
    _fields_ = [("extends", C.c_int64), ("shadowRays", C.c_int64)]


class OScene(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("triangleCount", C.c_int), ("emitterFlags", C.c_void_p),
                ("emission", C.c_void_p), ("bsdfs", C.c_void_p), ("bsdfCount", C.c_int), ("triBsdfIds", C.c_void_p),
                ("triMaterialIds", C.c_void_p), ("emitters", C.c_void_p), ("emitterCount", C.c_int),
                ("emitterTriIndices", C.c_void_p), ("emitterTriCdf", C.c_void_p), ("sceneEmitterCdf", C.c_void_p),
                ("spots", C.c_void_p), ("spotCount", C.c_int),
                ("texPixels", C.c_void_p), ("texW", C.c_void_p), ("texH", C.c_void_p), ("textureCount", C.c_int),
                ("mrPixels", C.c_void_p), ("mrW", C.c_void_p), ("mrH", C.c_void_p),
                ("hasEnv", C.c_int), ("envTexels", C.c_void_p), ("envW", C.c_int), ("envH", C.c_int),
                ("envIntensity", C.c_float), ("envRotation", C.c_float), ("envMarginal", C.c_void_p),
                ("envConditional", C.c_void_p), ("envTotalPower", C.c_float), ("envSampling", C.c_int),
                ("aliasRowProb", C.c_void_p), ("aliasRowIdx", C.c_void_p), ("aliasColProb", C.c_void_p),
                ("aliasColIdx", C.c_void_p), ("envPixelPdf", C.c_void_p), ("accel", C.c_void_p)]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _Lib:
    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.p = prefix

    def f(self, name):
        return getattr(self.lib, self.p + name)


class Oracle:
    """The C restatement (liboracle*.so)."""

    def __init__(self, libm: bool = False):
        path = os.path.join(HERE, "liboracle_libm.so" if libm else "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        self._l = _Lib(path, "or_")
        self.lib = self._l.lib
        self.lib.or_hash_uint.restype = C.c_uint32
        self.lib.or_pack_gamma.restype = C.c_uint32
        self.lib.or_hash_uint.argtypes = [C.c_uint32]
        self.lib.or_pack_gamma.argtypes = [C.c_float, C.c_float, C.c_float]

    def hash_uint(self, x: int) -> int:
        return int(self.lib.or_hash_uint(C.c_uint32(x)))

    def rng_stream(self, seed: int, n: int):
        u = np.empty(n, dtype=np.uint32)
        f = np.empty(n, dtype=np.float32)
        self.lib.or_rng_stream(C.c_uint32(seed), n, _p(u), _p(f))
        return u, f

    def math_eval(self, fn: int, a, b=None):
        a = np.ascontiguousarray(a, dtype=np.float32)
        b = np.zeros_like(a) if b is None else np.ascontiguousarray(b, dtype=np.float32)
        out = np.empty_like(a)
        self.lib.or_math_eval(fn, _p(a), _p(b), _p(out), len(a))
        return out

    def bsdf_eval(self, bsdf, wi, wo, fn="or_bsdf_eval"):
        b = np.ascontiguousarray(np.asarray(bsdf).reshape(1))
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        wo = np.ascontiguousarray(wo, dtype=np.float32)
        out = np.empty((len(wi), 3), dtype=np.float32)
        getattr(self.lib, fn)(_p(b), _p(wi), _p(wo), _p(out), len(wi))
        return out

    def bsdf_pdf(self, bsdf, wi, wo, fn="or_bsdf_pdf"):
        b = np.ascontiguousarray(np.asarray(bsdf).reshape(1))
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        wo = np.ascontiguousarray(wo, dtype=np.float32)
        out = np.empty(len(wi), dtype=np.float32)
        getattr(self.lib, fn)(_p(b), _p(wi), _p(wo), _p(out), len(wi))
        return out

    def bsdf_sample(self, bsdf, wi, u, fn="or_bsdf_sample"):
        b = np.ascontiguousarray(np.asarray(bsdf).reshape(1))
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        u = np.ascontiguousarray(u, dtype=np.float32)
        n = len(wi)
        wo = np.empty((n, 3), dtype=np.float32)
        w = np.empty((n, 3), dtype=np.float32)
        pdf = np.empty(n, dtype=np.float32)
        eta = np.empty(n, dtype=np.float32)
        getattr(self.lib, fn)(_p(b), _p(wi), _p(u), _p(wo), _p(w), _p(pdf), _p(eta), n)
        return wo, w, pdf, eta

    def env_build_cdf(self, rgba):
        rgba = np.ascontiguousarray(rgba, dtype=np.float32)
        h, w = rgba.shape[:2]
        marg = np.empty(h + 1, dtype=np.float32)
        cond = np.empty(h * (w + 1), dtype=np.float32)
        tp = C.c_float()
        self.lib.or_env_build_cdf(_p(rgba), w, h, _p(marg), _p(cond), C.byref(tp))
        return marg, cond, float(tp.value)

    def env_build_alias(self, rgba):
        rgba = np.ascontiguousarray(rgba, dtype=np.float32)
        h, w = rgba.shape[:2]
        rp = np.empty(h, dtype=np.float32)
        ri = np.empty(h, dtype=np.int32)
        cp = np.empty(h * w, dtype=np.float32)
        ci = np.empty(h * w, dtype=np.int32)
        pp = np.empty(h * w, dtype=np.float32)
        tot = C.c_double()
        self.lib.or_env_build_alias(_p(rgba), w, h, _p(rp), _p(ri), _p(cp), _p(ci), _p(pp), C.byref(tot))
        return rp, ri, cp, ci, pp, float(tot.value)

    def tex_float4(self, texels, wrap_v, uv):
        t = np.ascontiguousarray(texels, dtype=np.float32)
        h, w = t.shape[:2]
        uv = np.ascontiguousarray(uv, dtype=np.float32)
        out = np.empty((len(uv), 4), dtype=np.float32)
        self.lib.or_tex_float4(_p(t), w, h, 1 if wrap_v else 0, _p(uv), _p(out), len(uv))
        return out

    def pack_gamma(self, r, g, b) -> int:
        return int(self.lib.or_pack_gamma(C.c_float(r), C.c_float(g), C.c_float(b)))

    def present(self, accum, radiance, frame_index):
        accum = np.ascontiguousarray(accum, dtype=np.float32)
        radiance = np.ascontiguousarray(radiance, dtype=np.float32)
        out = np.empty(len(radiance), dtype=np.uint32)
        self.lib.or_present(_p(accum), _p(radiance), len(radiance), C.c_uint32(frame_index), _p(out))
        return accum, out


class SceneView:
    """An OScene over a bluetruthengine_b200.Scene (keeps the arrays alive)."""

    def __init__(self, scene, env_mode: int = 0, oracle: Optional[Oracle] = None, build_accel: Optional[bool] = None,
                 env_tables=None, textures=None, mr_textures=None):
        self.scene = scene
        self.keep = []
        s = OScene()
        T = scene.triangle_count

        def keep(a):
            self.keep.append(a)
            return _p(a)

        s.triangles = keep(np.ascontiguousarray(scene.triangles))
        s.triangleCount = T
        s.emitterFlags = keep(np.ascontiguousarray(scene.triangle_emitter_flags))
        s.emission = keep(np.ascontiguousarray(scene.triangle_emission, dtype=np.float32))
        s.bsdfs = keep(np.ascontiguousarray(scene.bsdfs))
        s.bsdfCount = len(scene.bsdfs)
        s.triBsdfIds = keep(np.ascontiguousarray(scene.triangle_bsdf_ids, dtype=np.int32))
        s.triMaterialIds = keep(np.ascontiguousarray(scene.triangle_material_ids, dtype=np.int32))
        E = len(scene.emitters)
        s.emitterCount = E
        if E > 0:
            s.emitters = keep(np.ascontiguousarray(scene.emitters))
            s.emitterTriIndices = keep(np.ascontiguousarray(scene.emitter_tri_indices, dtype=np.int32))
            s.emitterTriCdf = keep(np.ascontiguousarray(scene.emitter_tri_cdf, dtype=np.float32))
            s.sceneEmitterCdf = keep(np.ascontiguousarray(scene.scene_emitter_cdf, dtype=np.float32))
        s.spotCount = len(scene.spotlights)
        if s.spotCount:
            s.spots = keep(np.ascontiguousarray(scene.spotlights))
        s.textureCount = 0
        if textures:
            def table(imgs):
                arrs = [None if im is None else np.ascontiguousarray(im, dtype=np.uint8) for im in imgs]
                self.keep.extend(a for a in arrs if a is not None)
                ptrs = (C.c_void_p * len(arrs))(*[None if a is None else a.ctypes.data for a in arrs])
                ws = np.array([0 if a is None else a.shape[1] for a in arrs], dtype=np.int32)
                hs = np.array([0 if a is None else a.shape[0] for a in arrs], dtype=np.int32)
                self.keep.extend([ptrs, ws, hs])
                return C.cast(ptrs, C.c_void_p), _p(ws), _p(hs)
            s.texPixels, s.texW, s.texH = table(textures)
            s.textureCount = len(textures)
            if mr_textures:
                s.mrPixels, s.mrW, s.mrH = table(mr_textures)
        if scene.env_rgba is not None:
            env = np.ascontiguousarray(scene.env_rgba, dtype=np.float32)
            h, w = env.shape[:2]
            s.hasEnv = 1
            s.envTexels = keep(env)
            s.envW, s.envH = w, h
            s.envIntensity = scene.env_intensity
            pi = np.float32(3.14159265358979323846)
            s.envRotation = float(np.float32(scene.env_rotation_deg) * (pi / np.float32(180.0)))
            s.envSampling = env_mode
            orc = oracle or Oracle()
            if env_tables is not None:
                marg, cond, tp, rp, ri, cp, ci, pp, tpd = env_tables
            else:
                marg, cond, tp = orc.env_build_cdf(env)
                rp, ri, cp, ci, pp, tpd = orc.env_build_alias(env)
            s.envMarginal = keep(marg)
            s.envConditional = keep(cond)
            s.envTotalPower = float(np.float32(tpd)) if env_mode == 1 else tp
            s.aliasRowProb = keep(rp)
            s.aliasRowIdx = keep(ri)
            s.aliasColProb = keep(cp)
            s.aliasColIdx = keep(ci)
            s.envPixelPdf = keep(pp)
        self.s = s
        self._accel_lib = None
        if build_accel is None:
            build_accel = T > 64
        if build_accel:
            orc = oracle or Oracle()
            orc.lib.or_build_accel(C.byref(self.s))
            self._accel_lib = orc.lib

    def __del__(self):
        try:
            if self._accel_lib is not None and self.s.accel:
                self._accel_lib.or_free_accel(C.byref(self.s))
        except Exception:
            pass

    def ptr(self):
        return C.byref(self.s)


def camera_struct(cam) -> OCamera:
    c = OCamera()
    flat = np.frombuffer(np.asarray(cam).tobytes(), dtype=np.float32)
    for i in range(14):
        c.v[i] = float(flat[i])
    return c


def render_samples(lib_or, view: SceneView, cam, width, height, max_depth, pixels, samples, rr_start=3, hit_log=False,
                   threads=0, prefix="or_"):
    """Per-sample radiance [n,3] (+ per-bounce hit triangles, stats)."""
    pixels = np.ascontiguousarray(pixels, dtype=np.uint32)
    samples = np.ascontiguousarray(samples, dtype=np.uint32)
    n = len(pixels)
    out = np.empty((n, 3), dtype=np.float32)
    hl = np.empty((n, max_depth), dtype=np.int32) if hit_log else None
    st = OStats()
    cfg = OConfig(width, height, max_depth, rr_start)
    camc = camera_struct(cam)
    getattr(lib_or, prefix + "render_samples")(view.ptr(), C.byref(camc), C.byref(cfg), _p(pixels), _p(samples), n,
                                               _p(out), _p(hl), C.byref(st), threads)
    return out, hl, (int(st.extends), int(st.shadowRays))


def render_megakernel(lib_or, view: SceneView, cam, width, height, max_depth, pixels, frame_index, spp=5, rr_start=3,
                      threads=0, prefix="or_"):
    """One megakernel frame (src/optix_programs.cu:54-108): per pixel one RNG stream through spp paths; the
    frame's mean radiance [n,3] and stats."""
    pixels = np.ascontiguousarray(pixels, dtype=np.uint32)
    n = len(pixels)
    out = np.empty((n, 3), dtype=np.float32)
    st = OStats()
    cfg = OConfig(width, height, max_depth, rr_start)
    camc = camera_struct(cam)
    getattr(lib_or, prefix + "render_megakernel")(view.ptr(), C.byref(camc), C.byref(cfg), _p(pixels), n,
                                                  C.c_uint32(int(frame_index)), int(spp), _p(out), C.byref(st), threads)
    return out, (int(st.extends), int(st.shadowRays))


class Ref:
    """The reference's own shading headers compiled on the host (oracle/_ref)."""

    def __init__(self, fast: bool = False):
        path = os.path.join(REF_DIR, "libbteref_fast.so" if fast else "libbteref.so")
        if not os.path.exists(path):
            build(ref=True)
        self.lib = C.CDLL(path)
        self.lib.ref_hash_uint.restype = C.c_uint32
        self.lib.ref_hash_uint.argtypes = [C.c_uint32]

    @staticmethod
    def available(fast: bool = False) -> bool:
        return os.path.exists(os.path.join(REF_DIR, "libbteref_fast.so" if fast else "libbteref.so")) or \
            reference_present()


# POD layouts of the reference's include/render_kernel.h:9-94 (the arrays the loader hands to the cudaInit* calls)
_F3 = ("<f4", 3)
REF_TRIANGLE_DTYPE = np.dtype([("v0",) + _F3, ("v1",) + _F3, ("v2",) + _F3, ("n0",) + _F3, ("n1",) + _F3,
                               ("n2",) + _F3, ("uv0", "<f4", 2), ("uv1", "<f4", 2), ("uv2", "<f4", 2)])
REF_BSDF_DTYPE = np.dtype([("type", "<i4"), ("p0", "<f4", 4), ("p1", "<f4", 4), ("p2", "<f4", 4), ("p3", "<f4", 4)])
REF_EMITTER_DTYPE = np.dtype([("triIndexOffset", "<i4"), ("triCount", "<i4"), ("cdfOffset", "<i4"),
                              ("radiance",) + _F3, ("areaSum", "<f4"), ("powerWeight", "<f4")])
REF_SPOT_DTYPE = np.dtype([("position",) + _F3, ("direction",) + _F3, ("radiance",) + _F3, ("intensity", "<f4"),
                           ("innerConeCosine", "<f4"), ("outerConeCosine", "<f4")])
REF_CAMERA_DTYPE = np.dtype([("origin",) + _F3, ("forward",) + _F3, ("right",) + _F3, ("up",) + _F3,
                             ("fovYRadians", "<f4"), ("aspect", "<f4")])


class RefScene:
    """A scene flattened by the reference's own loader (src/scene.cpp, tinyobjloader, mesh_transform.h,
    gltf_loader.cpp and stb_image compiled from the reference tree: oracle/_ref/libbteref_loader.so) with the
    glue of src/main.cpp:533-930.  Carries the attributes SceneView reads; no product library is involved."""

    def __init__(self, path: str):
        lib_path = os.path.join(REF_DIR, "libbteref_loader.so")
        if not os.path.exists(lib_path):
            build(ref=True)
        lib = C.CDLL(lib_path)
        if lib.refl_load(str(path).encode()) < 0:
            raise RuntimeError("reference loader failed on %s" % path)
        cnt = np.zeros(6, np.int32)
        lib.refl_counts(_p(cnt))
        T, B, E, EC, SC, NC = (int(x) for x in cnt)
        self.triangles = np.empty(T, REF_TRIANGLE_DTYPE)
        self.bsdfs = np.empty(B, REF_BSDF_DTYPE)
        self.triangle_bsdf_ids, self.triangle_material_ids = np.empty(T, np.int32), np.empty(T, np.int32)
        self.triangle_emitter_flags = np.empty(T, np.uint8)
        self.emitter_tri_indices = np.empty(E, np.int32)
        self.emitter_tri_cdf = np.empty(EC, np.float32)
        self.scene_emitter_cdf = np.empty(SC, np.float32)
        cam = np.empty(NC, np.float32)
        lib.refl_copy(_p(self.triangles), _p(self.bsdfs), _p(self.triangle_bsdf_ids), _p(self.triangle_material_ids),
                      _p(self.triangle_emitter_flags), _p(self.emitter_tri_indices), _p(self.emitter_tri_cdf),
                      _p(self.scene_emitter_cdf), _p(cam))
        ex = np.zeros(5, np.int32)
        lib.refl_extras_counts(_p(ex))
        NE, NT, NS, EW, EH = (int(x) for x in ex)
        self.emitters = np.zeros(NE, REF_EMITTER_DTYPE)
        self.triangle_emission = np.zeros((NT, 3), np.float32)
        self.spotlights = np.zeros(NS, REF_SPOT_DTYPE)
        env = np.zeros((EH, EW, 4), np.float32) if EW > 0 else np.zeros(4, np.float32)
        self.camera = np.zeros(1, REF_CAMERA_DTYPE)
        lib.refl_extras_copy(_p(self.emitters), _p(self.triangle_emission), _p(self.spotlights), _p(env),
                             _p(self.camera))
        self.camera = self.camera[0]
        self.env_rgba = env if EW > 0 else None
        self.width, self.height = int(cam[10]), int(cam[11])
        self.env_intensity, self.env_rotation_deg = float(cam[12]), float(cam[13])
        self.triangle_count = T


def lbvh_morton_order(triangles):
    """CPU restatement of the LBVH's integer steps (the product's acceleration-structure build; the reference
    builds an OptiX GAS instead, src/host/optix_setup.cu:215-292, whose internals are closed): per triangle the
    centroid 0.5*(min+max) of its vertex bounds in float32, the centroid bounds, per axis
    q = min(trunc((c - lo) / (hi - lo) * 2^21), 2^21 - 1) (0 on a flat axis), the 63-bit code interleaving
    qx, qy, qz (x highest), and the stable ascending order of the codes.  Returns (codes uint64, order int32)."""
    v0, v1, v2 = (np.asarray(triangles[k], np.float32) for k in ("v0", "v1", "v2"))
    lo = np.minimum(v0, np.minimum(v1, v2))
    hi = np.maximum(v0, np.maximum(v1, v2))
    c = (np.float32(0.5) * (lo + hi)).astype(np.float32)
    clo, chi = c.min(axis=0), c.max(axis=0)
    q = np.zeros_like(c, dtype=np.uint32)
    for k in range(3):
        ext = np.float32(chi[k] - clo[k])
        if ext > 0:
            f = ((c[:, k] - clo[k]) / ext).astype(np.float32)
        else:
            f = np.zeros(len(c), np.float32)
        f = np.clip(f, np.float32(0.0), np.float32(1.0))
        q[:, k] = np.minimum((f * np.float32(2097152.0)).astype(np.uint32), np.uint32(2097151))

    def spread(x):
        x = x.astype(np.uint64) & np.uint64(0x1fffff)
        for shift, mask in ((32, 0x1f00000000ffff), (16, 0x1f0000ff0000ff), (8, 0x100f00f00f00f00f),
                            (4, 0x10c30c30c30c30c3), (2, 0x1249249249249249)):
            x = (x | (x << np.uint64(shift))) & np.uint64(mask)
        return x

    codes = (spread(q[:, 0]) << np.uint64(2)) | (spread(q[:, 1]) << np.uint64(1)) | spread(q[:, 2])
    return codes, np.argsort(codes, kind="stable").astype(np.int32)
