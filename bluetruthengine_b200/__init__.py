"""bluetruthengine_b200 -- B200-native wavefront path tracer behind Blue Truth
Engine's renderer API.

Python host mirror of the reference's include/render_kernel.h over the C-ABI
library libbte_b200.so (include/bte/render_api.h).  Function names follow the
reference (init_scene <- cudaInitScene, render <- cudaRender, ...).  Errors
raise BteError with the library's message; the reference exits the process
instead (src/host/cuda_check.h:14-32).  There is no CPU fallback: without the
library or without a CUDA device, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

__all__ = ["BteError", "Renderer", "Scene", "load_scene", "library_path", "load_library", "default_variant",
           "LIBRARIES", "RenderConfig",
           "ENV_CDF", "ENV_ALIAS", "TRIANGLE_DTYPE", "BSDF_DTYPE", "EMITTER_DTYPE", "SPOT_DTYPE", "CAMERA_DTYPE"]

HERE = os.path.dirname(os.path.abspath(__file__))
ENV_CDF = 0
ENV_ALIAS = 1


class BteError(RuntimeError):
    pass


# ---- POD layouts, byte-identical to render_kernel.h:9-94 ----
TRIANGLE_DTYPE = np.dtype([("v0", "<f4", 3), ("v1", "<f4", 3), ("v2", "<f4", 3), ("n0", "<f4", 3), ("n1", "<f4", 3),
                           ("n2", "<f4", 3), ("uv0", "<f4", 2), ("uv1", "<f4", 2), ("uv2", "<f4", 2)])
BSDF_DTYPE = np.dtype([("type", "<i4"), ("p0", "<f4", 4), ("p1", "<f4", 4), ("p2", "<f4", 4), ("p3", "<f4", 4)])
EMITTER_DTYPE = np.dtype([("triIndexOffset", "<i4"), ("triCount", "<i4"), ("cdfOffset", "<i4"), ("radiance", "<f4", 3),
                          ("areaSum", "<f4"), ("powerWeight", "<f4")])
SPOT_DTYPE = np.dtype([("position", "<f4", 3), ("direction", "<f4", 3), ("radiance", "<f4", 3), ("intensity", "<f4"),
                       ("innerConeCosine", "<f4"), ("outerConeCosine", "<f4")])
CAMERA_DTYPE = np.dtype([("origin", "<f4", 3), ("forward", "<f4", 3), ("right", "<f4", 3), ("up", "<f4", 3),
                         ("fovYRadians", "<f4"), ("aspect", "<f4")])
assert TRIANGLE_DTYPE.itemsize == 96 and BSDF_DTYPE.itemsize == 68 and CAMERA_DTYPE.itemsize == 56
VIEW_DTYPE = np.dtype([("camera", CAMERA_DTYPE), ("width", "<i4"), ("height", "<i4"), ("samplesPerFrame", "<i4")])


class Tuning(C.Structure):
    """BteTuning (include/bte/render_api.h)."""
    _fields_ = [("bvhWidth", C.c_int), ("maxLeafTriangles", C.c_int), ("shadeMinBlocks", C.c_int),
                ("postponePercent", C.c_int), ("sortShading", C.c_int), ("tailPaths", C.c_int),
                ("bvhBuilder", C.c_int), ("plocRadius", C.c_int), ("overlapConnect", C.c_int),
                ("wideCollapse", C.c_int), ("raySortBits", C.c_int), ("raySortBounces", C.c_int),
                ("leafTestsPerStep", C.c_int), ("orderBounces", C.c_int)]


class RenderConfig(C.Structure):
    _fields_ = [("samplesPerFrame", C.c_int), ("maxDepth", C.c_int), ("rrStart", C.c_int), ("envSampling", C.c_int),
                ("blockSize", C.c_int), ("useGraph", C.c_int)]


class FrameStats(C.Structure):
    _fields_ = [("samples", C.c_int64), ("extends", C.c_int64), ("shadowRays", C.c_int64),
                ("maxBounceReached", C.c_int), ("msTotal", C.c_float), ("msGenerate", C.c_float),
                ("msExtend", C.c_float), ("msShade", C.c_float), ("msConnect", C.c_float), ("msPresent", C.c_float),
                ("msTail", C.c_float), ("tailBounce", C.c_int), ("tailExtends", C.c_int64),
                ("tailShadowRays", C.c_int64)]


class _SceneArrays(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("triangleCount", C.c_int), ("materials", C.c_void_p),
                ("materialCount", C.c_int), ("triangleMaterialIds", C.c_void_p), ("triangleBsdfIds", C.c_void_p),
                ("bsdfs", C.c_void_p), ("bsdfCount", C.c_int), ("triangleEmission", C.c_void_p),
                ("triangleEmitterFlags", C.c_void_p), ("emitters", C.c_void_p), ("emitterCount", C.c_int),
                ("emitterTriIndices", C.c_void_p), ("emitterTriIndexCount", C.c_int), ("emitterTriCdf", C.c_void_p),
                ("emitterTriCdfCount", C.c_int), ("sceneEmitterCdf", C.c_void_p), ("spotlights", C.c_void_p),
                ("spotlightCount", C.c_int), ("envRGBA", C.c_void_p), ("envWidth", C.c_int), ("envHeight", C.c_int),
                ("envIntensity", C.c_float), ("envRotationDeg", C.c_float), ("camera", C.c_ubyte * 56),
                ("width", C.c_int), ("height", C.c_int),
                ("albedoPixels", C.POINTER(C.c_void_p)), ("albedoWidths", C.POINTER(C.c_int)),
                ("albedoHeights", C.POINTER(C.c_int)), ("mrPixels", C.POINTER(C.c_void_p)),
                ("mrWidths", C.POINTER(C.c_int)), ("mrHeights", C.POINTER(C.c_int))]


# The two builds of the library (bluetruthengine_b200/build.py): "fast" is the product (FP32 shading with
# CUDA's single-precision functions), "parity" matches the CPU checker bit for bit.  BTE_LIBRARY selects the
# default for this process.
LIBRARIES = {"fast": "libbte_b200.so", "parity": "libbte_b200_parity.so"}


def default_variant() -> str:
    v = os.environ.get("BTE_LIBRARY", "fast")
    if v not in LIBRARIES:
        raise BteError(f"BTE_LIBRARY must be one of {sorted(LIBRARIES)}, not {v!r}")
    return v


def library_path(variant: Optional[str] = None) -> str:
    return os.path.join(HERE, LIBRARIES[variant or default_variant()])


_LIBS: dict = {}


def load_library(build_if_missing: bool = True, variant: Optional[str] = None) -> C.CDLL:
    """Load one build of the library (default: BTE_LIBRARY, else the product), building both with nvcc when
    they are absent or older than their sources."""
    variant = variant or default_variant()
    if variant in _LIBS:
        return _LIBS[variant]
    path = library_path(variant)
    if build_if_missing:
        from . import build as _build
        _build.build()
    if not os.path.exists(path):
        raise BteError(f"{os.path.basename(path)} not found at {path}; run bluetruthengine_b200/build.py")
    lib = C.CDLL(path)
    lib.bte_last_error.restype = C.c_char_p
    lib.bte_get_render_mode.restype = C.c_int
    _LIBS[variant] = lib
    return lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc: int, lib: Optional[C.CDLL] = None):
    if rc < 0:
        lib = lib or load_library(False)
        raise BteError(lib.bte_last_error().decode("utf-8", "replace"))
    return rc


def _view(ptr: int, dtype, count: int) -> np.ndarray:
    if count <= 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    dt = np.dtype(dtype)
    buf = (C.c_char * (dt.itemsize * count)).from_address(ptr)
    return np.frombuffer(buf, dtype=dt, count=count).copy()


@dataclass
class Scene:
    """Flattened scene: the arrays src/main.cpp:600-930 passes to the cudaInit* calls."""
    triangles: np.ndarray           # TRIANGLE_DTYPE [T]
    materials: np.ndarray           # float32 [M,3]
    triangle_material_ids: np.ndarray
    triangle_bsdf_ids: np.ndarray
    bsdfs: np.ndarray               # BSDF_DTYPE [B]
    triangle_emission: np.ndarray   # float32 [T,3]
    triangle_emitter_flags: np.ndarray  # uint8 [T]
    emitters: np.ndarray            # EMITTER_DTYPE [E]
    emitter_tri_indices: np.ndarray
    emitter_tri_cdf: np.ndarray
    scene_emitter_cdf: np.ndarray   # float32 [E+1]
    spotlights: np.ndarray          # SPOT_DTYPE [S]
    env_rgba: Optional[np.ndarray]  # float32 [H,W,4]
    env_intensity: float
    env_rotation_deg: float
    camera: np.ndarray              # CAMERA_DTYPE scalar
    width: int
    height: int
    albedo_textures: list = None    # per material: uint8 [H,W,4] or None
    mr_textures: list = None        # per material: uint8 [H,W,4] or None (metallic-roughness maps)

    @property
    def triangle_count(self) -> int:
        return int(self.triangles.shape[0])


def decode_image(data: bytes) -> np.ndarray:
    """PNG / JPEG bytes -> uint8 [H,W,4] (the library's texture decoder; no GPU needed)."""
    lib = load_library()
    buf = np.frombuffer(data, dtype=np.uint8)
    w, h, c = C.c_int(), C.c_int(), C.c_int()
    _check(lib.bte_image_decode(_ptr(buf), C.c_longlong(len(buf)), None, C.c_longlong(0), C.byref(w), C.byref(h),
                                C.byref(c)))
    out = np.empty((h.value, w.value, 4), dtype=np.uint8)
    _check(lib.bte_image_decode(_ptr(buf), C.c_longlong(len(buf)), _ptr(out), C.c_longlong(out.size), C.byref(w),
                                C.byref(h), C.byref(c)))
    return out


def encode_png(rgba: np.ndarray) -> bytes:
    """uint8 [H,W,4] (first row first) -> PNG bytes (the library's encoder; no GPU needed)."""
    lib = load_library()
    a = np.ascontiguousarray(rgba, dtype=np.uint8)
    h, w = a.shape[:2]
    n = C.c_longlong()
    _check(lib.bte_encode_png(_ptr(a), w, h, None, C.c_longlong(0), C.byref(n)))
    out = np.empty(n.value, dtype=np.uint8)
    _check(lib.bte_encode_png(_ptr(a), w, h, _ptr(out), C.c_longlong(n.value), C.byref(n)))
    return out.tobytes()


def load_gltf(path: str, transform=None) -> dict:
    """A glTF / GLB model flattened as the reference's loadGltfModel does (no GPU needed).  transform: posX/Y/Z,
    rotX/Y/Z (degrees), scaleX/Y/Z.  Returns triangles, material_ids and per material bsdf, emission,
    is_emitter, albedo / mr images (uint8 [H,W,4] or None), and the number of outlier primitives skipped."""
    lib = load_library()
    h = C.c_void_p()
    xf = None if transform is None else np.ascontiguousarray(transform, dtype=np.float32)
    _check(lib.bte_gltf_load(str(path).encode(), _ptr(xf), C.byref(h)))
    try:
        t, m, sk = C.c_int(), C.c_int(), C.c_int()
        _check(lib.bte_gltf_counts(h, C.byref(t), C.byref(m), C.byref(sk)))
        tris = np.empty(t.value, TRIANGLE_DTYPE)
        ids = np.empty(t.value, np.int32)
        _check(lib.bte_gltf_triangles(h, _ptr(tris), _ptr(ids)))
        mats = []
        for i in range(m.value):
            b = np.zeros(1, BSDF_DTYPE)
            em = np.zeros(3, np.float32)
            ie = C.c_int()
            awh, mwh = np.zeros(2, np.int32), np.zeros(2, np.int32)
            _check(lib.bte_gltf_material(h, i, _ptr(b), _ptr(em), C.byref(ie), _ptr(awh), _ptr(mwh), None, None))
            alb = np.empty((awh[1], awh[0], 4), np.uint8) if awh[0] else None
            mr = np.empty((mwh[1], mwh[0], 4), np.uint8) if mwh[0] else None
            _check(lib.bte_gltf_material(h, i, None, None, None, None, None, _ptr(alb), _ptr(mr)))
            mats.append({"bsdf": b[0], "emission": em, "is_emitter": bool(ie.value), "albedo": alb, "mr": mr})
        return {"triangles": tris, "material_ids": ids, "materials": mats, "skipped_outliers": sk.value}
    finally:
        lib.bte_gltf_free(h)


def load_scene(path: str) -> Scene:
    """Parse scene.xml + OBJ (+ .hdr) with the library's loader (no GPU needed)."""
    lib = load_library()
    h = C.c_void_p()
    _check(lib.bte_scene_load(path.encode(), C.byref(h)))
    try:
        a = _SceneArrays()
        _check(lib.bte_scene_arrays(h, C.byref(a)))
        T = a.triangleCount
        env = None
        if a.envRGBA and a.envWidth > 0:
            env = _view(a.envRGBA, np.float32, a.envWidth * a.envHeight * 4).reshape(a.envHeight, a.envWidth, 4)
        cam = np.frombuffer(bytes(a.camera), dtype=CAMERA_DTYPE, count=1)[0].copy()
        E = a.emitterCount

        def images(px, ws, hs):
            out = []
            for i in range(a.materialCount):
                if not px or not px[i]:
                    out.append(None)
                else:
                    out.append(_view(px[i], np.uint8, ws[i] * hs[i] * 4).reshape(hs[i], ws[i], 4))
            return out

        albedo = images(a.albedoPixels, a.albedoWidths, a.albedoHeights)
        mr = images(a.mrPixels, a.mrWidths, a.mrHeights)
        return Scene(
            triangles=_view(a.triangles, TRIANGLE_DTYPE, T),
            materials=_view(a.materials, np.float32, 3 * a.materialCount).reshape(-1, 3),
            triangle_material_ids=_view(a.triangleMaterialIds, np.int32, T),
            triangle_bsdf_ids=_view(a.triangleBsdfIds, np.int32, T),
            bsdfs=_view(a.bsdfs, BSDF_DTYPE, a.bsdfCount),
            triangle_emission=_view(a.triangleEmission, np.float32, 3 * T).reshape(-1, 3),
            triangle_emitter_flags=_view(a.triangleEmitterFlags, np.uint8, T),
            emitters=_view(a.emitters, EMITTER_DTYPE, E),
            emitter_tri_indices=_view(a.emitterTriIndices, np.int32, a.emitterTriIndexCount),
            emitter_tri_cdf=_view(a.emitterTriCdf, np.float32, a.emitterTriCdfCount),
            scene_emitter_cdf=_view(a.sceneEmitterCdf, np.float32, E + 1 if E > 0 else 1),
            spotlights=_view(a.spotlights, SPOT_DTYPE, a.spotlightCount),
            env_rgba=env, env_intensity=float(a.envIntensity), env_rotation_deg=float(a.envRotationDeg),
            camera=cam, width=int(a.width), height=int(a.height), albedo_textures=albedo, mr_textures=mr)
    finally:
        lib.bte_scene_free(h)


class Renderer:
    """The reference's renderer API (render_kernel.h:100-211) over libbte_b200.

    One renderer state per process, like the reference's globals.
    """

    def __init__(self, variant: Optional[str] = None):
        self.variant = variant or default_variant()
        self.lib = load_library(variant=self.variant)
        self._keep = []

    def _ck(self, rc: int) -> int:
        return _check(rc, self.lib)

    # ---- uploads ----
    def init_scene(self, triangles, materials, triangle_material_ids, width, height):
        t = np.ascontiguousarray(triangles, dtype=TRIANGLE_DTYPE)
        m = np.ascontiguousarray(materials, dtype=np.float32)
        ids = None if triangle_material_ids is None else np.ascontiguousarray(triangle_material_ids, dtype=np.int32)
        self._ck(self.lib.bte_init_scene(_ptr(t), len(t), _ptr(m), len(m), _ptr(ids), int(width), int(height)))

    def init_accel(self):
        self._ck(self.lib.bte_init_accel())

    init_optix = init_accel   # the reference name (cudaInitOptix) builds the acceleration structure

    def init_camera(self, camera):
        c = np.ascontiguousarray(np.asarray(camera, dtype=CAMERA_DTYPE).reshape(1))
        self._ck(self.lib.bte_init_camera(_ptr(c)))

    def init_triangle_emission(self, emission):
        e = None if emission is None else np.ascontiguousarray(emission, dtype=np.float32)
        self._ck(self.lib.bte_init_triangle_emission(_ptr(e), 0 if e is None else len(e)))

    def init_triangle_emitter_flags(self, flags):
        f = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
        self._ck(self.lib.bte_init_triangle_emitter_flags(_ptr(f), 0 if f is None else len(f)))

    def init_emitter_table(self, emitters, tri_indices, tri_cdf, scene_cdf):
        if emitters is None or len(emitters) == 0:
            self._ck(self.lib.bte_init_emitter_table(None, 0, None, 0, None, 0, None))
            return
        e = np.ascontiguousarray(emitters, dtype=EMITTER_DTYPE)
        ti = np.ascontiguousarray(tri_indices, dtype=np.int32)
        tc = np.ascontiguousarray(tri_cdf, dtype=np.float32)
        sc = np.ascontiguousarray(scene_cdf, dtype=np.float32)
        self._ck(self.lib.bte_init_emitter_table(_ptr(e), len(e), _ptr(ti), len(ti), _ptr(tc), len(tc), _ptr(sc)))

    def init_bsdfs(self, bsdfs, triangle_bsdf_ids):
        b = np.ascontiguousarray(bsdfs, dtype=BSDF_DTYPE)
        ids = np.ascontiguousarray(triangle_bsdf_ids, dtype=np.int32)
        self._ck(self.lib.bte_init_bsdfs(_ptr(b), len(b), _ptr(ids), len(ids)))

    def init_spotlights(self, spots):
        if spots is None or len(spots) == 0:
            self._ck(self.lib.bte_init_spotlights(None, 0))
            return
        s = np.ascontiguousarray(spots, dtype=SPOT_DTYPE)
        self._ck(self.lib.bte_init_spotlights(_ptr(s), len(s)))

    def init_env_map(self, rgba, intensity=1.0, rotation_deg=0.0):
        if rgba is None:
            self._ck(self.lib.bte_init_env_map(None, 0, 0, C.c_float(0.0), C.c_float(0.0)))
            return
        e = np.ascontiguousarray(rgba, dtype=np.float32)
        h, w = e.shape[0], e.shape[1]
        self._ck(self.lib.bte_init_env_map(_ptr(e), w, h, C.c_float(intensity), C.c_float(rotation_deg)))

    def init_textures(self, images):
        self._init_tex(self.lib.bte_init_textures, images)

    def init_mr_textures(self, images):
        self._init_tex(self.lib.bte_init_mr_textures, images)

    def _init_tex(self, fn, images):
        if not images:
            self._ck(fn(None, None, None, 0))
            return
        arrs = [None if im is None else np.ascontiguousarray(im, dtype=np.uint8) for im in images]
        ptrs = (C.c_void_p * len(arrs))(*[None if a is None else a.ctypes.data for a in arrs])
        ws = np.array([0 if a is None else a.shape[1] for a in arrs], dtype=np.int32)
        hs = np.array([0 if a is None else a.shape[0] for a in arrs], dtype=np.int32)
        self._ck(fn(ptrs, _ptr(ws), _ptr(hs), len(arrs)))

    def upload(self, scene: Scene):
        """All uploads in the order of src/main.cpp:819-930."""
        self.init_camera(scene.camera)
        any_tex = lambda ims: ims is not None and any(im is not None for im in ims)
        self.init_textures(scene.albedo_textures if any_tex(scene.albedo_textures) else None)
        self.init_mr_textures(scene.mr_textures if any_tex(scene.mr_textures) else None)
        self.init_scene(scene.triangles, scene.materials, scene.triangle_material_ids, scene.width, scene.height)
        self.init_accel()
        self.init_triangle_emission(scene.triangle_emission)
        self.init_triangle_emitter_flags(scene.triangle_emitter_flags)
        self.init_emitter_table(scene.emitters, scene.emitter_tri_indices, scene.emitter_tri_cdf,
                                scene.scene_emitter_cdf)
        self.init_bsdfs(scene.bsdfs, scene.triangle_bsdf_ids)
        self.init_spotlights(scene.spotlights)
        self.init_env_map(scene.env_rgba, scene.env_intensity, scene.env_rotation_deg)

    # ---- frame API ----
    def set_config(self, samples_per_frame=1, max_depth=200, rr_start=3, env_sampling=ENV_CDF, block_size=0,
                   use_graph=0):
        cfg = RenderConfig(samples_per_frame, max_depth, rr_start, env_sampling, block_size, use_graph)
        self._ck(self.lib.bte_set_render_config(C.byref(cfg)))

    def reset_accumulation(self, width, height):
        self._ck(self.lib.bte_reset_accumulation(int(width), int(height)))

    def render(self, width, height):
        self._ck(self.lib.bte_render(int(width), int(height)))

    def set_output_buffer(self, device_ptr: int):
        self._ck(self.lib.bte_set_output_buffer(C.c_void_p(device_ptr)))

    def set_render_mode(self, mode: int):
        self._ck(self.lib.bte_set_render_mode(int(mode)))

    def get_render_mode(self) -> int:
        return int(self.lib.bte_get_render_mode())

    def cleanup(self):
        self._ck(self.lib.bte_cleanup())

    def stats(self) -> FrameStats:
        s = FrameStats()
        self._ck(self.lib.bte_get_frame_stats(C.byref(s)))
        return s

    def set_stage_timing(self, on: bool):
        self._ck(self.lib.bte_set_stage_timing(1 if on else 0))

    def toggle_denoiser(self) -> bool:
        """cudaToggleDenoiser: returns the new state; needs denoiser weights loaded."""
        return bool(self._ck(self.lib.bte_toggle_denoiser()))

    def read_denoised(self, width: int, height: int) -> np.ndarray:
        out = np.empty((height, width, 3), dtype=np.float32)
        self._ck(self.lib.bte_read_denoised(out.ctypes.data_as(C.c_void_p)))
        return out

    def render_views(self, views):
        """One frame of several camera views (sequence of (camera, width, height, samples_per_frame)) in one launch
        sequence; view slot i accumulates across calls."""
        arr = np.zeros(len(views), dtype=VIEW_DTYPE)
        for i, (cam, w, h, spp) in enumerate(views):
            arr[i]["camera"] = np.asarray(cam, dtype=CAMERA_DTYPE)
            arr[i]["width"], arr[i]["height"], arr[i]["samplesPerFrame"] = w, h, spp
        self._ck(self.lib.bte_render_views(_ptr(arr), len(views)))

    def read_view_accum(self, view: int, width: int, height: int):
        """(FP32 running mean [W*H, 3], FP64 running sum [W*H, 3]) of a batched view."""
        mean = np.empty((width * height, 3), dtype=np.float32)
        total = np.empty((width * height, 3), dtype=np.float64)
        self._ck(self.lib.bte_read_view_accum(int(view), _ptr(mean), _ptr(total)))
        return mean, total

    def reset_views(self):
        self._ck(self.lib.bte_reset_views())

    def select_scene(self, scene: int):
        """Make scene slot 0..7 the one every upload, configuration and render call acts on."""
        self._ck(self.lib.bte_select_scene(int(scene)))

    def selected_scene(self) -> int:
        out = C.c_int(0)
        self._ck(self.lib.bte_get_selected_scene(C.byref(out)))
        return out.value

    def set_batch_mode(self, mode: int):
        """1: a scene batch renders in one launch sequence over every scene's paths (default); 0: per scene."""
        self._ck(self.lib.bte_set_batch_mode(int(mode)))

    def batch_mode(self) -> int:
        out = C.c_int(0)
        self._ck(self.lib.bte_get_batch_mode(C.byref(out)))
        return out.value

    def render_scene_batch(self, batch):
        """One frame of several scene slots' views (sequence of (slot, views), views as for render_views): every
        scene's launch sequence is enqueued on its own streams before any wait, so the scenes run side by side."""
        slots = np.array([int(k) for k, _ in batch], dtype=np.int32)
        counts = np.array([len(v) for _, v in batch], dtype=np.int32)
        flat = [view for _, v in batch for view in v]
        arr = np.zeros(len(flat), dtype=VIEW_DTYPE)
        for i, (cam, w, h, spp) in enumerate(flat):
            arr[i]["camera"] = np.asarray(cam, dtype=CAMERA_DTYPE)
            arr[i]["width"], arr[i]["height"], arr[i]["samplesPerFrame"] = w, h, spp
        self._ck(self.lib.bte_render_scene_batch(_ptr(slots), _ptr(counts), _ptr(arr), len(batch)))

    def set_aov(self, enabled: bool):
        """Accumulate the denoiser features per pixel: albedo and shading normal at each path's first hit that is not a
        mirror or dielectric, seen through the ones in front of it (include/bte/render_api.h, bte_set_aov)."""
        self._ck(self.lib.bte_set_aov(1 if enabled else 0))

    def read_aov(self, width: int, height: int):
        """(albedo [H, W, 3], normal [H, W, 3]) running means, float32."""
        out = np.empty((height, width, 6), dtype=np.float32)
        self._ck(self.lib.bte_read_aov(out.ctypes.data_as(C.c_void_p)))
        return out[..., :3].copy(), out[..., 3:].copy()

    def set_tuning(self, max_leaf: int = 2, shade_min_blocks: int = 3, bvh_width: int = 8,
                   postpone_percent: int = 0, sort_shading: int = 1, tail_paths: int = 4096, bvh_builder: int = 1,
                   ploc_radius: int = 4, overlap_connect: int = 1, wide_collapse: int = 1, ray_sort_bits: int = 0,
                   ray_sort_bounces: int = 4, leaf_tests_per_step: int = 0, order_bounces: int = 3):
        t = Tuning(int(bvh_width), int(max_leaf), int(shade_min_blocks), int(postpone_percent), int(sort_shading),
                   int(tail_paths), int(bvh_builder), int(ploc_radius),
                   int(overlap_connect), int(wide_collapse), int(ray_sort_bits), int(ray_sort_bounces),
                   int(leaf_tests_per_step), int(order_bounces))
        self._ck(self.lib.bte_set_tuning(C.byref(t)))

    def tuning(self) -> dict:
        t = Tuning()
        self._ck(self.lib.bte_get_tuning(C.byref(t)))
        return {f: getattr(t, f) for f, _ in Tuning._fields_}

    def accel_info(self) -> dict:
        w, n, d, ms = C.c_int(), C.c_int(), C.c_int(), C.c_float()
        self._ck(self.lib.bte_get_accel_info(C.byref(w), C.byref(n), C.byref(d), C.byref(ms)))
        b = C.c_int()
        self._ck(self.lib.bte_get_accel_builder(C.byref(b)))
        return {"width": w.value, "nodes": n.value, "depth": d.value, "ms_build": ms.value, "builder": b.value}

    def set_hit_log(self, on: bool):
        self._ck(self.lib.bte_set_hit_log(1 if on else 0))

    def frame_index(self) -> int:
        v = C.c_uint32()
        self._ck(self.lib.bte_get_frame_index(C.byref(v)))
        return int(v.value)

    def set_frame_index(self, i: int):
        self._ck(self.lib.bte_set_frame_index(C.c_uint32(i)))

    # ---- headless output ----
    def write_png(self, path: str):
        self._ck(self.lib.bte_write_png(str(path).encode()))

    def capture_screenshot(self) -> str:
        buf = C.create_string_buffer(64)
        self._ck(self.lib.bte_capture_screenshot(buf, 64))
        return buf.value.decode()

    def record_start(self, raw_path: Optional[str] = None, fps: int = 30):
        self._ck(self.lib.bte_record_start(None if raw_path is None else str(raw_path).encode(), int(fps)))

    def record_frame(self):
        self._ck(self.lib.bte_record_frame())

    def record_stop(self):
        self._ck(self.lib.bte_record_stop())

    def mark_scene_changed(self):
        self._ck(self.lib.bte_mark_scene_changed())

    def framebuffer_size(self):
        w, h = C.c_int(), C.c_int()
        self._ck(self.lib.bte_get_framebuffer_size(C.byref(w), C.byref(h)))
        return w.value, h.value

    def read_framebuffer(self, width, height) -> np.ndarray:
        out = np.empty(width * height, dtype=np.uint32)
        self._ck(self.lib.bte_read_framebuffer(_ptr(out)))
        return out

    def read_accum(self, width, height) -> np.ndarray:
        out = np.empty((width * height, 3), dtype=np.float32)
        self._ck(self.lib.bte_read_accum(_ptr(out)))
        return out

    def read_accum_f64(self, width, height) -> np.ndarray:
        out = np.empty((width * height, 3), dtype=np.float64)
        self._ck(self.lib.bte_read_accum_f64(_ptr(out)))
        return out

    def read_sample_radiance(self, count: int) -> np.ndarray:
        out = np.empty((count, 3), dtype=np.float32)
        self._ck(self.lib.bte_read_sample_radiance(_ptr(out), int(count)))
        return out

    def read_hit_log(self, count: int) -> np.ndarray:
        out = np.empty(count, dtype=np.int32)
        self._ck(self.lib.bte_read_hit_log(_ptr(out), int(count)))
        return out

    # ---- parity probes ----
    def trace_closest(self, rays: np.ndarray, lanes: int = 1):
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = len(r)
        tri = np.empty(n, dtype=np.int32)
        tuv = np.empty((n, 3), dtype=np.float32)
        self._ck(self.lib.bte_trace_closest_lanes(_ptr(r), n, int(lanes), _ptr(tri), _ptr(tuv)))
        return tri, tuv

    def trace_occluded(self, rays: np.ndarray, tmax: np.ndarray, lanes: int = 1):
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        t = np.ascontiguousarray(tmax, dtype=np.float32)
        out = np.empty(len(r), dtype=np.uint8)
        self._ck(self.lib.bte_trace_occluded_lanes(_ptr(r), _ptr(t), len(r), int(lanes), _ptr(out)))
        return out

    def env_query(self, op: int, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = len(x)
        width = {0: 3, 1: 1, 2: 7}[op]
        out = np.empty((n, width), dtype=np.float32)
        self._ck(self.lib.bte_env_query(int(op), _ptr(x), n, _ptr(out)))
        return out

    def env_tables(self, w, h):
        marg = np.empty(h + 1, dtype=np.float32)
        cond = np.empty(h * (w + 1), dtype=np.float32)
        tp = C.c_float()
        self._ck(self.lib.bte_env_tables(_ptr(marg), _ptr(cond), C.byref(tp)))
        return marg, cond, float(tp.value)

    def env_alias_tables(self, w, h):
        rp = np.empty(h, dtype=np.float32)
        ri = np.empty(h, dtype=np.int32)
        cp = np.empty(h * w, dtype=np.float32)
        ci = np.empty(h * w, dtype=np.int32)
        pp = np.empty(h * w, dtype=np.float32)
        self._ck(self.lib.bte_env_alias_tables(_ptr(rp), _ptr(ri), _ptr(cp), _ptr(ci), _ptr(pp)))
        return rp, ri, cp, ci, pp

    def math_eval(self, fn: int, a: np.ndarray, b: Optional[np.ndarray] = None) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float32)
        bb = None if b is None else np.ascontiguousarray(b, dtype=np.float32)
        out = np.empty_like(a)
        self._ck(self.lib.bte_math_eval(int(fn), _ptr(a), _ptr(bb), _ptr(out), len(a)))
        return out

    def bsdf_query(self, bsdf, op: int, wi: np.ndarray, x: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(np.asarray(bsdf, dtype=BSDF_DTYPE).reshape(1))
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = len(wi)
        width = {0: 3, 1: 1, 2: 8}[op]
        out = np.empty((n, width), dtype=np.float32)
        self._ck(self.lib.bte_bsdf_query(_ptr(b), int(op), _ptr(wi), _ptr(x), n, _ptr(out)))
        return out

    def tex_hw_vs_sw(self, texels: np.ndarray, wrap_v: bool, uv: np.ndarray):
        t = np.ascontiguousarray(texels, dtype=np.float32)
        h, w = t.shape[0], t.shape[1]
        uv = np.ascontiguousarray(uv, dtype=np.float32)
        n = len(uv)
        hw = np.empty((n, 4), dtype=np.float32)
        sw = np.empty((n, 4), dtype=np.float32)
        self._ck(self.lib.bte_tex_hw_vs_sw(_ptr(t), w, h, 1 if wrap_v else 0, _ptr(uv), n, _ptr(hw), _ptr(sw)))
        return hw, sw
