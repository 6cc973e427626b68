"""Seeded synthetic scenes, written as scene.xml + OBJ (+ Radiance .hdr).

The reference ships no benchmark scenes (its shipped scene.xml references
.glb files that are not in its repository), so every workload here is
generated from a fixed seed with the shapes, sizes and value distributions of
the workload it stands in for, and goes through the same scene.xml/OBJ loader
a user's scene would.

  cornell(seed)          Cornell box in a 555-unit cube: 5 axis-aligned quad walls
                         (white 0.73, red 0.65/0.05/0.05, green 0.12/0.45/0.15),
                         a 130x105 ceiling quad light with radiance (17,12,4), two
                         Lambertian boxes (165^3 and 165x330x165, rotated -18/+18
                         degrees), 36 triangles, 256x256, no environment map.
  disney_spheres(seed)   64 seed-placed icospheres (subdivision 3-6, radius U[0.2,2])
                         on a 200x200 tessellated ground plane (~1.0M triangles),
                         per-object Disney parameters (baseColor U[0,1]^3, roughness
                         U[0.05,1], metallic Bernoulli(0.3), specular 0.5, clearcoat
                         U[0,1]), procedural 2048x1024 HDR sky with a 0.5-degree sun
                         of radiance 1e4, 1920x1080.
"""
from __future__ import annotations

import math
import os
import struct

import numpy as np

GENERATOR_VERSION = 4
CACHE_ROOT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), ".scene_cache")


def _fmt(x: float) -> str:
    return "%.9g" % float(np.float32(x))


# ---------------------------------------------------------------- writers
def write_obj(path: str, verts: np.ndarray, faces: np.ndarray, normals: np.ndarray | None = None):
    """Triangles only; faces are 0-based (written 1-based)."""
    verts = np.asarray(verts, dtype=np.float32)
    faces = np.asarray(faces, dtype=np.int64) + 1
    with open(path, "w") as f:
        f.write("# generated by bluetruthengine_b200.scenes\n")
        f.write("".join("v %s %s %s\n" % (_fmt(a), _fmt(b), _fmt(c)) for a, b, c in verts))
        if normals is not None:
            normals = np.asarray(normals, dtype=np.float32)
            f.write("".join("vn %s %s %s\n" % (_fmt(a), _fmt(b), _fmt(c)) for a, b, c in normals))
            f.write("".join("f %d//%d %d//%d %d//%d\n" % (a, a, b, b, c, c) for a, b, c in faces))
        else:
            f.write("".join("f %d %d %d\n" % (a, b, c) for a, b, c in faces))


def rgbe_encode(rgb: np.ndarray) -> np.ndarray:
    """float RGB [H,W,3] -> RGBE bytes [H,W,4] (Radiance shared-exponent format)."""
    rgb = np.asarray(rgb, dtype=np.float64)
    v = rgb.max(axis=-1)
    out = np.zeros(rgb.shape[:-1] + (4,), dtype=np.uint8)
    ok = v >= 1e-32
    m, e = np.frexp(v[ok])
    scale = m * 256.0 / v[ok]
    out[ok, 0:3] = np.clip(np.floor(rgb[ok] * scale[:, None]), 0, 255).astype(np.uint8)
    out[ok, 3] = (e + 128).astype(np.uint8)
    return out


def rgbe_decode(rgbe: np.ndarray) -> np.ndarray:
    """RGBE bytes -> RGBA float32 as the loader decodes them (value * 2^(e-136), alpha 1)."""
    rgbe = np.asarray(rgbe)
    out = np.zeros(rgbe.shape[:-1] + (4,), dtype=np.float32)
    e = rgbe[..., 3].astype(np.int32)
    f1 = np.where(e != 0, np.ldexp(np.float32(1.0), e - 136).astype(np.float32), np.float32(0.0)).astype(np.float32)
    for c in range(3):
        out[..., c] = (rgbe[..., c].astype(np.float32) * f1).astype(np.float32)
    out[..., 3] = 1.0
    return out


def write_hdr(path: str, rgb: np.ndarray):
    """Radiance .hdr with run-length-format scanlines (literal runs only)."""
    rgbe = rgbe_encode(rgb)
    h, w = rgbe.shape[:2]
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
        f.write(("-Y %d +X %d\n" % (h, w)).encode())
        for y in range(h):
            f.write(bytes([2, 2, (w >> 8) & 0xFF, w & 0xFF]))
            for c in range(4):
                row = rgbe[y, :, c]
                for s in range(0, w, 128):
                    chunk = row[s:s + 128]
                    f.write(bytes([len(chunk)]))
                    f.write(chunk.tobytes())


# ---------------------------------------------------------------- geometry
def quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3); geometric normal = (p1-p0) x (p2-p0)."""
    v = np.array([p0, p1, p2, p3], dtype=np.float64)
    f = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int64)
    return v, f


def unit_cube():
    """[-0.5,0.5]^3 with outward-facing windings, 12 triangles."""
    v = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)], dtype=np.float64)
    idx = {tuple(p): i for i, p in enumerate(v.tolist())}

    def q(a, b, c, d):
        return [[idx[a], idx[b], idx[c]], [idx[a], idx[c], idx[d]]]

    h = 0.5
    faces = []
    faces += q((h, -h, -h), (h, h, -h), (h, h, h), (h, -h, h))          # +x
    faces += q((-h, -h, -h), (-h, -h, h), (-h, h, h), (-h, h, -h))      # -x
    faces += q((-h, h, -h), (-h, h, h), (h, h, h), (h, h, -h))          # +y
    faces += q((-h, -h, -h), (h, -h, -h), (h, -h, h), (-h, -h, h))      # -y
    faces += q((-h, -h, h), (h, -h, h), (h, h, h), (-h, h, h))          # +z
    faces += q((-h, -h, -h), (-h, h, -h), (h, h, -h), (h, -h, -h))      # -z
    return v, np.array(faces, dtype=np.int64)


def icosphere(level: int):
    """Unit icosphere by midpoint subdivision; returns (verts, faces) with outward windings."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
                  [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        ab, bc, ca = inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    # make windings outward
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    flip = (n * v[f[:, 0]]).sum(1) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


def grid_plane(n: int, half: float):
    """n x n quads on y=0 spanning [-half, half]^2, normal +y (2*n*n triangles)."""
    xs = np.linspace(-half, half, n + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    v = np.stack([X.ravel(), np.zeros(X.size), Z.ravel()], 1)
    i = np.arange(n)[:, None] * (n + 1) + np.arange(n)[None, :]
    i = i.ravel()
    a, b, c, d = i, i + 1, i + (n + 1) + 1, i + (n + 1)
    # (a, b, c): b-a = +z, c-a = +x+z -> (+z) x (+x) = +y
    f = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    return v, f


# ---------------------------------------------------------------- scenes
def _scene_dir(name: str, seed: int) -> str:
    d = os.path.join(CACHE_ROOT, "%s_s%d_v%d" % (name, seed, GENERATOR_VERSION))
    os.makedirs(d, exist_ok=True)
    return d


def _done(d: str) -> bool:
    return os.path.exists(os.path.join(d, ".complete"))


def _mark(d: str):
    with open(os.path.join(d, ".complete"), "w") as f:
        f.write("ok\n")


def cornell(seed: int = 1, width: int = 256, height: int = 256) -> str:
    """Config-1 Cornell box; returns the scene.xml path."""
    d = _scene_dir("cornell_%dx%d" % (width, height), seed)
    path = os.path.join(d, "scene.xml")
    if _done(d):
        return path
    L = 555.0
    walls = {
        "floor": quad((0, 0, 0), (0, 0, L), (L, 0, L), (L, 0, 0)),          # normal +y
        "ceiling": quad((0, L, 0), (L, L, 0), (L, L, L), (0, L, L)),        # normal -y
        "back": quad((0, 0, L), (0, L, L), (L, L, L), (L, 0, L)),           # normal -z
        "left": quad((L, 0, 0), (L, 0, L), (L, L, L), (L, L, 0)),           # x = 555, normal -x
        "right": quad((0, 0, 0), (0, L, 0), (0, L, L), (0, 0, L)),          # x = 0, normal +x
    }
    cx, cz, y = L / 2, L / 2, L - 0.5
    lw, ld = 130.0 / 2, 105.0 / 2
    walls["light"] = quad((cx - lw, y, cz - ld), (cx + lw, y, cz - ld), (cx + lw, y, cz + ld), (cx - lw, y, cz + ld))
    for name, (v, f) in walls.items():
        write_obj(os.path.join(d, name + ".obj"), v, f)
    cv, cf = unit_cube()
    write_obj(os.path.join(d, "cube.obj"), cv, cf)
    xml = f"""<scene>
    <bsdf name="white" type="diffuse" albedoR="0.73" albedoG="0.73" albedoB="0.73" />
    <bsdf name="red" type="diffuse" albedoR="0.65" albedoG="0.05" albedoB="0.05" />
    <bsdf name="green" type="diffuse" albedoR="0.12" albedoG="0.45" albedoB="0.15" />
    <bsdf name="lightb" type="diffuse" albedoR="0.78" albedoG="0.78" albedoB="0.78" />
    <material name="whiteMat" bsdf="white" />
    <material name="redMat" bsdf="red" />
    <material name="greenMat" bsdf="green" />
    <material name="lightMat" bsdf="lightb" />
    <mesh filename="floor.obj" material="whiteMat" />
    <mesh filename="ceiling.obj" material="whiteMat" />
    <mesh filename="back.obj" material="whiteMat" />
    <mesh filename="left.obj" material="redMat" />
    <mesh filename="right.obj" material="greenMat" />
    <mesh filename="light.obj" material="lightMat" isEmitter="true" radianceR="17" radianceG="12" radianceB="4" />
    <mesh filename="cube.obj" material="whiteMat" scaleX="165" scaleY="165" scaleZ="165" rotY="-18" posX="185" posY="82.5" posZ="169" />
    <mesh filename="cube.obj" material="whiteMat" scaleX="165" scaleY="330" scaleZ="165" rotY="18" posX="368" posY="165" posZ="351" />
    <window width="{width}" height="{height}" />
    <camera eyeX="277.5" eyeY="277.5" eyeZ="-790" lookAtX="277.5" lookAtY="277.5" lookAtZ="277.5" upX="0" upY="1" upZ="0" fovY="39.5" />
</scene>
"""
    with open(path, "w") as f:
        f.write(xml)
    _mark(d)
    return path


def sky_env(width: int = 2048, height: int = 1024, sun_elev_deg: float = 35.0, sun_azim: float = 0.8,
            sun_radius_deg: float = 0.5, sun_radiance: float = 1.0e4) -> np.ndarray:
    """Procedural sky (gradient) plus a sun disc; RGB float [H,W,3] in equirectangular layout
    (row 0 = +Y pole, phi = u*2pi - pi, direction = (sin t cos p, cos t, sin t sin p))."""
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    phi = u * 2 * np.pi - np.pi
    th = v * np.pi
    P, T = np.meshgrid(phi, th)
    dx, dy, dz = np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)
    horizon = np.array([0.90, 0.95, 1.00])
    zenith = np.array([0.20, 0.38, 0.85])
    ground = np.array([0.33, 0.30, 0.26]) * 0.35
    up = np.clip(dy, 0.0, 1.0)[..., None]
    s = np.sqrt(up)
    sky = horizon * (1 - s) + zenith * s
    rgb = np.where((dy > 0)[..., None], sky, ground)
    el, az = math.radians(sun_elev_deg), sun_azim
    sd = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    cosang = dx * sd[0] + dy * sd[1] + dz * sd[2]
    sun = cosang >= math.cos(math.radians(sun_radius_deg))
    rgb[sun] = np.array([1.0, 0.96, 0.88]) * sun_radiance
    return rgb.astype(np.float32)


def disney_spheres(seed: int = 2, width: int = 1920, height: int = 1080, n_spheres: int = 64,
                   grid: int = 200, env_w: int = 2048, env_h: int = 1024) -> str:
    """Config-2 scene; returns the scene.xml path."""
    d = _scene_dir("disney_%dx%d_n%d_g%d_e%d" % (width, height, n_spheres, grid, env_w), seed)
    path = os.path.join(d, "scene.xml")
    if _done(d):
        return path
    rng = np.random.default_rng(seed)
    for lvl in (3, 4, 5, 6):
        v, f = icosphere(lvl)
        write_obj(os.path.join(d, "ico%d.obj" % lvl), v, f, normals=v)
    gv, gf = grid_plane(grid, 25.0)
    write_obj(os.path.join(d, "ground.obj"), gv, gf)
    write_hdr(os.path.join(d, "sky.hdr"), sky_env(env_w, env_h))
    lines = ["<scene>", '    <environment map="sky.hdr" intensity="1.0" rotation="0.0" />',
             '    <bsdf name="groundB" type="disney" base_colorR="0.5" base_colorG="0.5" base_colorB="0.5" '
             'roughness="0.6" metallic="0" specular="0.5" clearcoat="0" />',
             '    <material name="groundM" bsdf="groundB" />',
             '    <mesh filename="ground.obj" material="groundM" />']
    # subdivision levels: a fixed mix (32 x L3, 15 x L4, 9 x L5, 8 x L6 for 64 spheres) that puts the
    # scene at ~1.04M triangles with the ground, assigned to spheres in seeded order
    mix = np.array([3] * 32 + [4] * 15 + [5] * 9 + [6] * 8)
    if n_spheres != 64:
        mix = np.resize(mix, n_spheres)
    levels = rng.permutation(mix)
    for i in range(n_spheres):
        r = rng.uniform(0.2, 2.0)
        x, z = rng.uniform(-20.0, 20.0, size=2)
        bc = rng.uniform(0.0, 1.0, size=3)
        rough = rng.uniform(0.05, 1.0)
        metal = 1.0 if rng.uniform() < 0.3 else 0.0
        cc = rng.uniform(0.0, 1.0)
        lines.append('    <bsdf name="s%dB" type="disney" base_colorR="%s" base_colorG="%s" base_colorB="%s" '
                     'roughness="%s" metallic="%s" specular="0.5" clearcoat="%s" />'
                     % (i, _fmt(bc[0]), _fmt(bc[1]), _fmt(bc[2]), _fmt(rough), _fmt(metal), _fmt(cc)))
        lines.append('    <material name="s%dM" bsdf="s%dB" />' % (i, i))
        lines.append('    <mesh filename="ico%d.obj" material="s%dM" scaleX="%s" scaleY="%s" scaleZ="%s" '
                     'posX="%s" posY="%s" posZ="%s" />' % (levels[i], i, _fmt(r), _fmt(r), _fmt(r), _fmt(x), _fmt(r),
                                                          _fmt(z)))
    lines.append('    <window width="%d" height="%d" />' % (width, height))
    lines.append('    <camera eyeX="0" eyeY="11" eyeZ="-36" lookAtX="0" lookAtY="1" lookAtZ="0" '
                 'upX="0" upY="1" upZ="0" fovY="42" />')
    lines.append("</scene>")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    _mark(d)
    return path


def random_scene(seed: int, n_tris: int = 200, extent: float = 10.0) -> str:
    """Small random triangle soup with mixed BSDFs, an area light and a spotlight,
    plus a small env map: exercises every shading branch in parity tests."""
    d = _scene_dir("random_t%d" % n_tris, seed)
    path = os.path.join(d, "scene.xml")
    if _done(d):
        return path
    rng = np.random.default_rng(seed)
    c = rng.uniform(-extent, extent, size=(n_tris, 1, 3))
    v = (c + rng.normal(0, extent * 0.15, size=(n_tris, 3, 3))).reshape(-1, 3)
    f = np.arange(3 * n_tris).reshape(-1, 3)
    half = n_tris // 2
    write_obj(os.path.join(d, "soupA.obj"), v[:3 * half], f[:half])
    nrm = rng.normal(size=(3 * (n_tris - half), 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    write_obj(os.path.join(d, "soupB.obj"), v[3 * half:], f[:n_tris - half], normals=nrm)
    lv, lf = quad((-2, extent * 1.6, -2), (2, extent * 1.6, -2), (2, extent * 1.6, 2), (-2, extent * 1.6, 2))
    write_obj(os.path.join(d, "lamp.obj"), lv, lf)   # normal -y: emits downwards
    write_hdr(os.path.join(d, "env.hdr"), sky_env(64, 32, sun_radius_deg=6.0, sun_radiance=50.0))
    xml = """<scene>
    <environment map="env.hdr" intensity="0.7" rotation="25" />
    <bsdf name="dis" type="disney" base_colorR="0.8" base_colorG="0.5" base_colorB="0.3" roughness="0.35" metallic="0.3"
          specular="0.6" specular_transmission="0.3" specular_tint="0.2" sheen="0.4" sheen_tint="0.5" subsurface="0.3"
          anisotropic="0.4" clearcoat="0.6" clearcoat_gloss="0.7" eta="1.45" />
    <bsdf name="mf" type="microfacet" albedoR="0.3" albedoG="0.35" albedoB="0.4" alpha="0.25" intIOR="1.6" extIOR="1.0" />
    <bsdf name="glass" type="dielectric" intIOR="1.5" extIOR="1.0" />
    <bsdf name="mir" type="mirror" albedoR="0.9" albedoG="0.9" albedoB="0.85" />
    <bsdf name="lam" type="diffuse" albedoR="0.6" albedoG="0.6" albedoB="0.6" />
    <material name="mDis" bsdf="dis" />
    <material name="mMf" bsdf="mf" />
    <material name="mGlass" bsdf="glass" />
    <material name="mMir" bsdf="mir" />
    <material name="mLam" bsdf="lam" />
    <mesh filename="soupA.obj" material="mDis" />
    <mesh filename="soupB.obj" material="mMf" />
    <mesh filename="soupA.obj" material="mGlass" posX="3" rotY="40" />
    <mesh filename="soupB.obj" material="mMir" posZ="-4" rotX="15" scaleX="0.7" scaleY="0.7" scaleZ="0.7" />
    <mesh filename="soupA.obj" material="mLam" posY="-6" rotZ="70" />
    <mesh filename="lamp.obj" material="mLam" isEmitter="true" radianceR="30" radianceG="25" radianceB="20" />
    <spotlight posX="0" posY="14" posZ="-12" dirX="0" dirY="-0.7" dirZ="0.7" radianceR="1" radianceG="0.9"
               radianceB="0.8" intensity="400" innerConeAngle="20" outerConeAngle="40" />
    <window width="64" height="48" />
    <camera eyeX="0" eyeY="4" eyeZ="-30" lookAtX="0" lookAtY="0" lookAtZ="0" upX="0" upY="1" upZ="0" fovY="50" />
</scene>
"""
    with open(path, "w") as f:
        f.write(xml)
    _mark(d)
    return path


def _c4_assets() -> str:
    """Shared meshes of the denoiser training scenes (one directory, one XML per scene)."""
    d = os.path.join(CACHE_ROOT, "c4_assets_v%d" % GENERATOR_VERSION)
    os.makedirs(d, exist_ok=True)
    if _done(d):
        return d
    L = 555.0
    walls = {
        "floor": quad((0, 0, 0), (0, 0, L), (L, 0, L), (L, 0, 0)),
        "ceiling": quad((0, L, 0), (L, L, 0), (L, L, L), (0, L, L)),
        "back": quad((0, 0, L), (0, L, L), (L, L, L), (L, 0, L)),
        "left": quad((L, 0, 0), (L, 0, L), (L, L, L), (L, L, 0)),
        "right": quad((0, 0, 0), (0, L, 0), (0, L, L), (0, 0, L)),
        # unit light quad in the xz plane facing -y (scaled and placed per scene)
        "lightq": quad((-0.5, 0, -0.5), (0.5, 0, -0.5), (0.5, 0, 0.5), (-0.5, 0, 0.5)),
    }
    for name, (v, f) in walls.items():
        write_obj(os.path.join(d, name + ".obj"), v, f)
    cv, cf = unit_cube()
    write_obj(os.path.join(d, "cube.obj"), cv, cf)
    sv, sf = icosphere(3)
    write_obj(os.path.join(d, "sphere.obj"), sv, sf, normals=sv)
    _mark(d)
    return d


def c4_scene(seed: int, width: int = 256, height: int = 256) -> str:
    """Denoiser training scene: a Cornell box (the 555-unit box of the plain-method scene) with seeded
    wall colours, light size/colour, 0-2 diffuse boxes, 1-3 dielectric spheres (IOR U[1.3, 1.8]) and,
    sometimes, a mirror or rough-conductor-like microfacet object; camera jittered.  Returns the XML path."""
    d = _c4_assets()
    path = os.path.join(d, "c4_%d_%dx%d.xml" % (seed, width, height))
    if os.path.exists(path):
        return path
    rng = np.random.default_rng(1_000_003 * seed + 17)
    L = 555.0
    col = lambda lo, hi: rng.uniform(lo, hi, 3)
    white = rng.uniform(0.55, 0.85)
    left = col(0.03, 0.8)
    right = col(0.03, 0.8)
    le = np.array([17.0, 12.0, 4.0]) * rng.uniform(0.5, 2.0) * rng.uniform(0.7, 1.3, 3)
    lw, ld = 130.0 * rng.uniform(0.6, 1.6), 105.0 * rng.uniform(0.6, 1.6)
    f3 = lambda v: "R=\"%.5f\" {0}G=\"%.5f\" {0}B=\"%.5f\"" % tuple(v)
    bs = [f'<bsdf name="white" type="diffuse" albedoR="{white:.5f}" albedoG="{white:.5f}" albedoB="{white:.5f}" />',
          '<bsdf name="left" type="diffuse" albedo%s />' % (f3(left).format("albedo")),
          '<bsdf name="right" type="diffuse" albedo%s />' % (f3(right).format("albedo")),
          '<bsdf name="lightb" type="diffuse" albedoR="0.78" albedoG="0.78" albedoB="0.78" />']
    meshes = ['<mesh filename="floor.obj" material="mWhite" />', '<mesh filename="ceiling.obj" material="mWhite" />',
              '<mesh filename="back.obj" material="mWhite" />', '<mesh filename="left.obj" material="mLeft" />',
              '<mesh filename="right.obj" material="mRight" />',
              '<mesh filename="lightq.obj" material="mLight" isEmitter="true" radianceR="%.4f" radianceG="%.4f" '
              'radianceB="%.4f" scaleX="%.3f" scaleY="1" scaleZ="%.3f" posX="277.5" posY="554.5" posZ="277.5" />'
              % (le[0], le[1], le[2], lw, ld)]
    mats = ['<material name="mWhite" bsdf="white" />', '<material name="mLeft" bsdf="left" />',
            '<material name="mRight" bsdf="right" />', '<material name="mLight" bsdf="lightb" />']
    for k in range(int(rng.integers(0, 3))):
        sx, sy, sz = rng.uniform(80, 200), rng.uniform(80, 350), rng.uniform(80, 200)
        c = col(0.2, 0.85)
        bs.append('<bsdf name="box%d" type="diffuse" albedo%s />' % (k, f3(c).format("albedo")))
        mats.append('<material name="mBox%d" bsdf="box%d" />' % (k, k))
        meshes.append('<mesh filename="cube.obj" material="mBox%d" scaleX="%.3f" scaleY="%.3f" scaleZ="%.3f" rotY="%.3f" '
                      'posX="%.3f" posY="%.3f" posZ="%.3f" />'
                      % (k, sx, sy, sz, rng.uniform(-45, 45), rng.uniform(110, 445), sy / 2, rng.uniform(110, 445)))
    for k in range(int(rng.integers(1, 4))):
        r = rng.uniform(40, 100)
        ior = rng.uniform(1.3, 1.8)
        bs.append('<bsdf name="glass%d" type="dielectric" intIOR="%.4f" extIOR="1.0" />' % (k, ior))
        mats.append('<material name="mGlass%d" bsdf="glass%d" />' % (k, k))
        y = r if rng.uniform() < 0.7 else rng.uniform(r, L - 150 - r)
        meshes.append('<mesh filename="sphere.obj" material="mGlass%d" scaleX="%.3f" scaleY="%.3f" scaleZ="%.3f" '
                      'posX="%.3f" posY="%.3f" posZ="%.3f" />'
                      % (k, r, r, r, rng.uniform(r, L - r), y, rng.uniform(r, L - r)))
    if rng.uniform() < 0.35:
        r = rng.uniform(40, 90)
        if rng.uniform() < 0.5:
            bs.append('<bsdf name="extra" type="mirror" albedo%s />' % (f3(col(0.7, 0.95)).format("albedo")))
        else:
            bs.append('<bsdf name="extra" type="microfacet" albedo%s alpha="%.3f" intIOR="1.6" extIOR="1.0" />'
                      % (f3(col(0.1, 0.7)).format("albedo"), rng.uniform(0.05, 0.5)))
        mats.append('<material name="mExtra" bsdf="extra" />')
        meshes.append('<mesh filename="sphere.obj" material="mExtra" scaleX="%.3f" scaleY="%.3f" scaleZ="%.3f" '
                      'posX="%.3f" posY="%.3f" posZ="%.3f" />' % (r, r, r, rng.uniform(r, L - r), r, rng.uniform(r, L - r)))
    eye = np.array([277.5, 277.5, -790.0]) + rng.uniform(-40, 40, 3)
    fov = 39.5 + rng.uniform(-5, 5)
    xml = "<scene>\n    " + "\n    ".join(bs + mats + meshes) + "\n"
    xml += '    <window width="%d" height="%d" />\n' % (width, height)
    xml += ('    <camera eyeX="%.3f" eyeY="%.3f" eyeZ="%.3f" lookAtX="277.5" lookAtY="277.5" lookAtZ="277.5" '
            'upX="0" upY="1" upZ="0" fovY="%.3f" />\n</scene>\n' % (eye[0], eye[1], eye[2], fov))
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(xml)
    os.replace(tmp, path)
    return path


def _outdoor_assets() -> str:
    """Shared assets of the outdoor denoiser training scenes: icospheres, a ground plane and four skies
    (sun elevations 12, 30, 50 and 70 degrees, sun radius 0.5-1.5 degrees, 1024x512)."""
    d = os.path.join(CACHE_ROOT, "outdoor_assets_v%d" % GENERATOR_VERSION)
    os.makedirs(d, exist_ok=True)
    if _done(d):
        return d
    for lvl in (2, 3, 4):
        v, f = icosphere(lvl)
        write_obj(os.path.join(d, "ico%d.obj" % lvl), v, f, normals=v)
    gv, gf = grid_plane(24, 25.0)
    write_obj(os.path.join(d, "ground.obj"), gv, gf)
    for k, (el, rad) in enumerate([(12.0, 1.5), (30.0, 1.0), (50.0, 0.5), (70.0, 0.75)]):
        write_hdr(os.path.join(d, "sky%d.hdr" % k), sky_env(1024, 512, sun_elev_deg=el, sun_radius_deg=rad))
    _mark(d)
    return d


def outdoor_scene(seed: int, width: int = 256, height: int = 256) -> str:
    """Denoiser training scene of the outdoor kind (the 1080p Disney/env-map view and the large scene's
    materials): 6-20 spheres on a Disney ground under one of four procedural skies (random rotation and
    intensity), each sphere Disney (baseColor U[0,1]^3, roughness U[0.05,1], metallic Bernoulli(0.3),
    specular 0.5, clearcoat U[0,1]; 55%), microfacet (alpha U[0.01,0.5]; 15%), mirror (15%) or dielectric
    (IOR U[1.3,1.8]; 15%); camera at a random azimuth, distance and height looking into the group.
    Returns the XML path."""
    d = _outdoor_assets()
    path = os.path.join(d, "outdoor_%d_%dx%d.xml" % (seed, width, height))
    if os.path.exists(path):
        return path
    rng = np.random.default_rng(2_000_029 * seed + 5)
    g = rng.uniform(0.3, 0.7)
    bs = ['<bsdf name="groundB" type="disney" base_colorR="%s" base_colorG="%s" base_colorB="%s" roughness="%s" '
          'metallic="0" specular="0.5" clearcoat="0" />' % (_fmt(g), _fmt(g * rng.uniform(0.9, 1.1)),
                                                            _fmt(g * rng.uniform(0.8, 1.1)), _fmt(rng.uniform(0.3, 0.9)))]
    mats = ['<material name="groundM" bsdf="groundB" />']
    meshes = ['<mesh filename="ground.obj" material="groundM" />']
    for i in range(int(rng.integers(6, 21))):
        r = rng.uniform(0.3, 2.5)
        x, z = rng.uniform(-12.0, 12.0, size=2)
        kind = rng.uniform()
        if kind < 0.55:
            bc = rng.uniform(0.0, 1.0, size=3)
            bs.append('<bsdf name="s%dB" type="disney" base_colorR="%s" base_colorG="%s" base_colorB="%s" '
                      'roughness="%s" metallic="%s" specular="0.5" clearcoat="%s" />'
                      % (i, _fmt(bc[0]), _fmt(bc[1]), _fmt(bc[2]), _fmt(rng.uniform(0.05, 1.0)),
                         _fmt(1.0 if rng.uniform() < 0.3 else 0.0), _fmt(rng.uniform(0.0, 1.0))))
        elif kind < 0.70:
            c = rng.uniform(0.05, 0.8, 3)
            bs.append('<bsdf name="s%dB" type="microfacet" albedoR="%s" albedoG="%s" albedoB="%s" alpha="%s" '
                      'intIOR="1.5" extIOR="1.0" />' % (i, _fmt(c[0]), _fmt(c[1]), _fmt(c[2]),
                                                        _fmt(rng.uniform(0.01, 0.5))))
        elif kind < 0.85:
            c = rng.uniform(0.6, 0.95, 3)
            bs.append('<bsdf name="s%dB" type="mirror" albedoR="%s" albedoG="%s" albedoB="%s" />'
                      % (i, _fmt(c[0]), _fmt(c[1]), _fmt(c[2])))
        else:
            bs.append('<bsdf name="s%dB" type="dielectric" intIOR="%s" extIOR="1.0" />' % (i, _fmt(rng.uniform(1.3, 1.8))))
        mats.append('<material name="s%dM" bsdf="s%dB" />' % (i, i))
        meshes.append('<mesh filename="ico%d.obj" material="s%dM" scaleX="%s" scaleY="%s" scaleZ="%s" posX="%s" '
                      'posY="%s" posZ="%s" />' % (int(rng.integers(2, 5)), i, _fmt(r), _fmt(r), _fmt(r), _fmt(x), _fmt(r),
                                                  _fmt(z)))
    az = rng.uniform(0, 2 * np.pi)
    dist = rng.uniform(14.0, 34.0)
    eye = (dist * np.cos(az), rng.uniform(1.5, 14.0), dist * np.sin(az))
    tgt = (rng.uniform(-4, 4), rng.uniform(0.0, 2.0), rng.uniform(-4, 4))
    xml = "<scene>\n    " + "\n    ".join(bs + mats + meshes) + "\n"
    xml += '    <environment map="sky%d.hdr" intensity="%s" rotation="%s" />\n' % (
        int(rng.integers(0, 4)), _fmt(rng.uniform(0.5, 2.0)), _fmt(rng.uniform(0.0, 360.0)))
    xml += '    <window width="%d" height="%d" />\n' % (width, height)
    xml += ('    <camera eyeX="%s" eyeY="%s" eyeZ="%s" lookAtX="%s" lookAtY="%s" lookAtZ="%s" upX="0" upY="1" upZ="0" '
            'fovY="%s" />\n</scene>\n' % (_fmt(eye[0]), _fmt(eye[1]), _fmt(eye[2]), _fmt(tgt[0]), _fmt(tgt[1]),
                                            _fmt(tgt[2]), _fmt(rng.uniform(30.0, 60.0))))
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(xml)
    os.replace(tmp, path)
    return path


def _blob_assets() -> str:
    """Shared assets of the blob denoiser training scenes: eight seeded 25,000-triangle blob meshes (seeds other
    than the large scene's), a ground plane and four soft-sun skies (sun elevations 20, 35, 50 and 65 degrees,
    radius 4-8 degrees, radiance 10-40; 1024x512)."""
    d = os.path.join(CACHE_ROOT, "blob_assets_v%d" % GENERATOR_VERSION)
    os.makedirs(d, exist_ok=True)
    if _done(d):
        return d
    for m in range(8):
        v, f, n = blob_mesh(9000 + m)
        write_obj(os.path.join(d, "blob%d.obj" % m), v, f, normals=n)
    gv, gf = quad((-60, 0, -60), (-60, 0, 60), (60, 0, 60), (60, 0, -60))
    write_obj(os.path.join(d, "ground.obj"), gv, gf)
    for k, (el, rad, lum) in enumerate([(20.0, 8.0, 10.0), (35.0, 6.0, 20.0), (50.0, 5.0, 30.0), (65.0, 4.0, 40.0)]):
        write_hdr(os.path.join(d, "sky%d.hdr" % k),
                  sky_env(1024, 512, sun_elev_deg=el, sun_radius_deg=rad, sun_radiance=lum))
    _mark(d)
    return d


def blob_scene(seed: int, width: int = 256, height: int = 256) -> str:
    """Denoiser training scene of the large configuration's kind: 6-16 instances of the blob meshes (scale
    U[0.6, 1.4], rotations as in `large_instanced`), each mirror (tint U[0.6, 0.95]^3), dielectric (IOR
    U[1.3, 1.8]) or microfacet (albedo U[0.05, 0.8]^3, alpha U[0.01, 0.5]) with equal odds, on a diffuse
    ground under one of four soft-sun skies (random rotation and intensity); camera at a random azimuth,
    distance and height looking into the group.  Returns the XML path."""
    d = _blob_assets()
    path = os.path.join(d, "blob_%d_%dx%d.xml" % (seed, width, height))
    if os.path.exists(path):
        return path
    rng = np.random.default_rng(3_000_017 * seed + 11)
    g = rng.uniform(0.3, 0.6)
    bs = ['<bsdf name="groundB" type="diffuse" albedoR="%s" albedoG="%s" albedoB="%s" />'
          % (_fmt(g), _fmt(g * rng.uniform(0.9, 1.05)), _fmt(g * rng.uniform(0.8, 1.0)))]
    mats = ['<material name="groundM" bsdf="groundB" />']
    meshes = ['<mesh filename="ground.obj" material="groundM" />']
    for i in range(int(rng.integers(6, 17))):
        kind = int(rng.integers(0, 3))
        if kind == 0:
            c = rng.uniform(0.6, 0.95, 3)
            bs.append('<bsdf name="b%dB" type="mirror" albedoR="%s" albedoG="%s" albedoB="%s" />'
                      % (i, _fmt(c[0]), _fmt(c[1]), _fmt(c[2])))
        elif kind == 1:
            bs.append('<bsdf name="b%dB" type="dielectric" intIOR="%s" extIOR="1.0" />' % (i, _fmt(rng.uniform(1.3, 1.8))))
        else:
            c = rng.uniform(0.05, 0.8, 3)
            bs.append('<bsdf name="b%dB" type="microfacet" albedoR="%s" albedoG="%s" albedoB="%s" alpha="%s" '
                      'intIOR="1.5" extIOR="1.0" />' % (i, _fmt(c[0]), _fmt(c[1]), _fmt(c[2]),
                                                        _fmt(rng.uniform(0.01, 0.5))))
        mats.append('<material name="b%dM" bsdf="b%dB" />' % (i, i))
        s = rng.uniform(0.6, 1.4)
        x, z = rng.uniform(-7.0, 7.0, size=2)
        meshes.append('<mesh filename="blob%d.obj" material="b%dM" scaleX="%s" scaleY="%s" scaleZ="%s" rotY="%s" '
                      'rotX="%s" posX="%s" posY="%s" posZ="%s" />'
                      % (int(rng.integers(0, 8)), i, _fmt(s), _fmt(s), _fmt(s), _fmt(rng.uniform(0, 360)),
                         _fmt(rng.uniform(-30, 30)), _fmt(x), _fmt(s * 0.9), _fmt(z)))
    az = rng.uniform(0, 2 * np.pi)
    dist = rng.uniform(8.0, 22.0)
    eye = (dist * np.cos(az), rng.uniform(2.0, 12.0), dist * np.sin(az))
    tgt = (rng.uniform(-3, 3), rng.uniform(0.0, 1.5), rng.uniform(-3, 3))
    xml = "<scene>\n    " + "\n    ".join(bs + mats + meshes) + "\n"
    xml += '    <environment map="sky%d.hdr" intensity="%s" rotation="%s" />\n' % (
        int(rng.integers(0, 4)), _fmt(rng.uniform(0.5, 2.0)), _fmt(rng.uniform(0.0, 360.0)))
    xml += '    <window width="%d" height="%d" />\n' % (width, height)
    xml += ('    <camera eyeX="%s" eyeY="%s" eyeZ="%s" lookAtX="%s" lookAtY="%s" lookAtZ="%s" upX="0" upY="1" upZ="0" '
            'fovY="%s" />\n</scene>\n' % (_fmt(eye[0]), _fmt(eye[1]), _fmt(eye[2]), _fmt(tgt[0]), _fmt(tgt[1]),
                                            _fmt(tgt[2]), _fmt(rng.uniform(30.0, 60.0))))
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(xml)
    os.replace(tmp, path)
    return path


def blob_mesh(seed: int, nu: int = 125, nv: int = 100):
    """Seeded closed mesh of exactly 2*nu*nv triangles: a torus of random proportions whose surface is
    displaced along its normal by a few random low-frequency harmonics.  Returns (verts, faces, normals)."""
    rng = np.random.default_rng(seed)
    R, r = 1.0, rng.uniform(0.25, 0.6)
    u = np.arange(nu) * (2 * np.pi / nu)
    v = np.arange(nv) * (2 * np.pi / nv)
    U, V = np.meshgrid(u, v, indexing="ij")
    disp = np.zeros_like(U)
    for _ in range(4):
        a, b = rng.integers(1, 6), rng.integers(1, 5)
        disp += rng.uniform(0.03, 0.12) * r * np.sin(a * U + rng.uniform(0, 2 * np.pi)) * np.cos(b * V + rng.uniform(0, 2 * np.pi))
    rr = r + disp
    x = (R + rr * np.cos(V)) * np.cos(U)
    y = rr * np.sin(V) * rng.uniform(0.6, 1.4)
    z = (R + rr * np.cos(V)) * np.sin(U)
    verts = np.stack([x, y, z], -1).reshape(-1, 3)
    i = np.arange(nu)[:, None] * nv + np.arange(nv)[None, :]
    i1 = ((np.arange(nu)[:, None] + 1) % nu) * nv + np.arange(nv)[None, :]
    i2 = np.arange(nu)[:, None] * nv + (np.arange(nv)[None, :] + 1) % nv
    i3 = ((np.arange(nu)[:, None] + 1) % nu) * nv + (np.arange(nv)[None, :] + 1) % nv
    faces = np.concatenate([np.stack([i.ravel(), i2.ravel(), i3.ravel()], 1), np.stack([i.ravel(), i3.ravel(), i1.ravel()], 1)])
    # area-weighted vertex normals, oriented outward from the torus core
    fn = np.cross(verts[faces[:, 1]] - verts[faces[:, 0]], verts[faces[:, 2]] - verts[faces[:, 0]])
    core = np.stack([R * np.cos(U), np.zeros_like(U), R * np.sin(U)], -1).reshape(-1, 3)
    if np.sum(fn * (verts[faces[:, 0]] - core[faces[:, 0]])) < 0:
        faces = faces[:, [0, 2, 1]]
        fn = -fn
    n = np.zeros_like(verts)
    for k in range(3):
        np.add.at(n, faces[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-12)
    return verts, faces, n


def large_instanced(seed: int = 5, width: int = 3840, height: int = 2160, n_instances: int = 400, n_meshes: int = 8,
                    env_w: int = 2048, env_h: int = 1024, sun_radius_deg: float = 6.0, sun_radiance: float = 20.0) -> str:
    """The large configuration: n_instances placements of n_meshes seed-generated 25,000-triangle meshes
    (10M triangles flattened), each instance mirror, dielectric or microfacet (alpha U[0.01, 0.5]), on a
    diffuse ground under the procedural sky with a soft sun (a 6-degree disc of radiance 20: caustics through
    the glass and mirror instances are found only by BSDF sampling, and under a 0.5-degree sun of radiance 1e4
    their variance keeps even a 1024-spp accumulation at relMSE ~0.9 against the converged image); returns the
    scene.xml path."""
    d = _scene_dir("large_%dx%d_n%d_m%d_sun%g_%g" % (width, height, n_instances, n_meshes, sun_radius_deg,
                                                     sun_radiance), seed)
    path = os.path.join(d, "scene.xml")
    if _done(d):
        return path
    rng = np.random.default_rng(seed)
    for m in range(n_meshes):
        v, f, n = blob_mesh(seed * 100 + m)
        write_obj(os.path.join(d, "blob%d.obj" % m), v, f, normals=n)
    gv, gf = quad((-200, 0, -200), (-200, 0, 200), (200, 0, 200), (200, 0, -200))
    write_obj(os.path.join(d, "ground.obj"), gv, gf)
    write_hdr(os.path.join(d, "sky.hdr"), sky_env(env_w, env_h, sun_radius_deg=sun_radius_deg, sun_radiance=sun_radiance))
    bs = ['<bsdf name="ground" type="diffuse" albedoR="0.45" albedoG="0.42" albedoB="0.38" />']
    mats = ['<material name="mGround" bsdf="ground" />']
    meshes = ['<mesh filename="ground.obj" material="mGround" />']
    side = int(np.ceil(np.sqrt(n_instances)))
    for k in range(n_instances):
        kind = int(rng.integers(0, 3))
        if kind == 0:
            c = rng.uniform(0.6, 0.95, 3)
            bs.append('<bsdf name="b%d" type="mirror" albedoR="%.4f" albedoG="%.4f" albedoB="%.4f" />' % (k, *c))
        elif kind == 1:
            bs.append('<bsdf name="b%d" type="dielectric" intIOR="%.4f" extIOR="1.0" />' % (k, rng.uniform(1.3, 1.8)))
        else:
            c = rng.uniform(0.05, 0.8, 3)
            bs.append('<bsdf name="b%d" type="microfacet" albedoR="%.4f" albedoG="%.4f" albedoB="%.4f" alpha="%.4f" '
                      'intIOR="1.5" extIOR="1.0" />' % (k, *c, rng.uniform(0.01, 0.5)))
        mats.append('<material name="m%d" bsdf="b%d" />' % (k, k))
        gx, gz = k % side, k // side
        s = rng.uniform(0.6, 1.4)
        meshes.append('<mesh filename="blob%d.obj" material="m%d" scaleX="%.3f" scaleY="%.3f" scaleZ="%.3f" rotY="%.2f" '
                      'rotX="%.2f" posX="%.3f" posY="%.3f" posZ="%.3f" />'
                      % (int(rng.integers(0, n_meshes)), k, s, s, s, rng.uniform(0, 360), rng.uniform(-30, 30),
                         (gx - side / 2 + rng.uniform(-0.25, 0.25)) * 3.2, s * 0.9, (gz - side / 2 + rng.uniform(-0.25, 0.25)) * 3.2))
    xml = "<scene>\n    " + "\n    ".join(bs + mats + meshes) + "\n"
    xml += '    <environment map="sky.hdr" intensity="1.0" rotation="0.0" />\n'
    xml += '    <window width="%d" height="%d" />\n' % (width, height)
    xml += ('    <camera eyeX="0" eyeY="22" eyeZ="-48" lookAtX="0" lookAtY="0" lookAtZ="4" upX="0" upY="1" upZ="0" '
            'fovY="50" />\n</scene>\n')
    with open(path, "w") as f:
        f.write(xml)
    _mark(d)
    return path
