"""Synthetic glTF 2.0 / GLB models for the glTF reader tests (written at test time, deterministic).

write_models(dir) writes:
  rich.glb        node hierarchy (quaternion TRS, matrix, scale), interleaved POSITION/NORMAL in one strided
                  buffer view, u8 / u16 / u32 / no indices, triangles / strip / fan / lines, float and
                  normalized u8 / u16 texture coordinates, PNG + JPEG textures in buffer views, every KHR
                  material extension the reference maps, an emissive material, a primitive without material
  external.gltf   JSON with an external .bin, a base64 data-URI buffer, an external PNG, an unlit material,
                  a "Background" node, an "Outline" material primitive, a 16-bit PNG texture
  outliers.glb    six primitives of which one is far too large and one far away (culled), NORMAL missing
  noscene.gltf    no "scenes": every node is a root (children are visited again as roots)
Texture images come from tests/golden/images/fixtures.npz.
"""
from __future__ import annotations

import base64
import json
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FLOAT, U8, U16, U32, I8, I16 = 5126, 5121, 5123, 5125, 5120, 5122


class Builder:
    def __init__(self):
        self.j = {"asset": {"version": "2.0", "generator": "tests"}, "buffers": [], "bufferViews": [], "accessors": [],
                  "meshes": [], "nodes": [], "materials": [], "textures": [], "images": []}
        self.bin = bytearray()

    def _align(self):
        while len(self.bin) % 4:
            self.bin.append(0)

    def view(self, data: bytes, stride: int = 0) -> int:
        self._align()
        v = {"buffer": 0, "byteOffset": len(self.bin), "byteLength": len(data)}
        if stride:
            v["byteStride"] = stride
        self.bin += data
        self.j["bufferViews"].append(v)
        return len(self.j["bufferViews"]) - 1

    def accessor(self, view: int, ctype: int, count: int, type_: str, offset: int = 0, normalized=False,
                 mn=None, mx=None) -> int:
        a = {"bufferView": view, "componentType": ctype, "count": count, "type": type_}
        if offset:
            a["byteOffset"] = offset
        if normalized:
            a["normalized"] = True
        if mn is not None:
            a["min"], a["max"] = [float(v) for v in mn], [float(v) for v in mx]
        self.j["accessors"].append(a)
        return len(self.j["accessors"]) - 1

    def data(self, arr: np.ndarray, ctype: int, type_: str, normalized=False, bounds=False) -> int:
        arr = np.ascontiguousarray(arr)
        v = self.view(arr.tobytes())
        n = arr.shape[0]
        mn = arr.min(0) if bounds else None
        mx = arr.max(0) if bounds else None
        return self.accessor(v, ctype, n, type_, normalized=normalized, mn=mn, mx=mx)

    def image_view(self, data: bytes, mime: str) -> int:
        v = self.view(data)
        self.j["images"].append({"bufferView": v, "mimeType": mime})
        self.j["textures"].append({"source": len(self.j["images"]) - 1})
        return len(self.j["textures"]) - 1

    def image_uri(self, uri: str) -> int:
        self.j["images"].append({"uri": uri})
        self.j["textures"].append({"source": len(self.j["images"]) - 1})
        return len(self.j["textures"]) - 1

    def material(self, m: dict) -> int:
        self.j["materials"].append(m)
        return len(self.j["materials"]) - 1

    def mesh(self, prims) -> int:
        self.j["meshes"].append({"primitives": prims})
        return len(self.j["meshes"]) - 1

    def node(self, **kw) -> int:
        self.j["nodes"].append(kw)
        return len(self.j["nodes"]) - 1

    def glb(self) -> bytes:
        self.j["buffers"] = [{"byteLength": len(self.bin)}]
        js = json.dumps(self.j).encode()
        js += b" " * ((4 - len(js) % 4) % 4)
        self._align()
        body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(self.bin), 0x004E4942) + bytes(self.bin)
        return struct.pack("<4sII", b"glTF", 2, 12 + len(body)) + body


def grid(nx, ny, size=1.0, z=0.0, seed=0):
    """A bumpy nx*ny vertex grid: positions, normals, uvs, triangle indices."""
    rng = np.random.default_rng(seed)
    u, v = np.meshgrid(np.linspace(0, 1, nx), np.linspace(0, 1, ny))
    h = 0.1 * np.sin(6 * u) * np.cos(4 * v) + 0.02 * rng.standard_normal(u.shape)
    pos = np.stack([(u - 0.5) * size, (v - 0.5) * size, z + h * size], -1).reshape(-1, 3).astype(np.float32)
    nrm = np.stack([-0.6 * np.cos(6 * u) * np.cos(4 * v), 0.4 * np.sin(6 * u) * np.sin(4 * v), np.ones_like(u)], -1)
    nrm = (nrm / np.linalg.norm(nrm, axis=-1, keepdims=True)).reshape(-1, 3).astype(np.float32)
    uv = np.stack([u, v], -1).reshape(-1, 2).astype(np.float32)
    idx = []
    for j in range(ny - 1):
        for i in range(nx - 1):
            a = j * nx + i
            idx += [a, a + 1, a + nx, a + 1, a + nx + 1, a + nx]
    return pos, nrm, uv, np.array(idx)


def _fixture(name):
    z = np.load(os.path.join(HERE, "images", "fixtures.npz"))
    return z["file_" + name].tobytes()


def rich():
    b = Builder()
    tex_png = b.image_view(_fixture("rgba8_31x33"), "image/png")
    tex_jpg = b.image_view(_fixture("jstb_q90_64x48"), "image/jpeg")
    m0 = b.material({"name": "painted", "pbrMetallicRoughness": {
        "baseColorFactor": [0.8, 0.6, 1.0, 0.9], "metallicFactor": 0.25, "roughnessFactor": 0.4,
        "baseColorTexture": {"index": tex_png}, "metallicRoughnessTexture": {"index": tex_jpg}}})
    m1 = b.material({"name": "glassish", "pbrMetallicRoughness": {"baseColorFactor": [0.2, 0.7, 0.3, 1.0]},
                     "extensions": {"KHR_materials_ior": {"ior": 1.33}, "KHR_materials_transmission": {"transmissionFactor": 0.7},
                                    "KHR_materials_clearcoat": {"clearcoatFactor": 0.5, "clearcoatRoughnessFactor": 0.2},
                                    "KHR_materials_sheen": {"sheenColorFactor": [0.3, 0.5, 0.1]}}})
    m2 = b.material({"name": "lamp", "emissiveFactor": [1.0, 0.8, 0.5],
                     "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 12.0}}})
    m3 = b.material({"name": "jpgtinted", "pbrMetallicRoughness": {"baseColorTexture": {"index": tex_jpg, "texCoord": 0},
                                                                    "metallicFactor": 0.0}})
    pos, nrm, uv, idx = grid(9, 7, 2.0, seed=1)
    inter = np.concatenate([pos, nrm], 1).astype(np.float32)   # interleaved, stride 24
    iv = b.view(inter.tobytes(), stride=24)
    a_pos = b.accessor(iv, FLOAT, len(pos), "VEC3", 0, mn=pos.min(0), mx=pos.max(0))
    a_nrm = b.accessor(iv, FLOAT, len(pos), "VEC3", 12)
    a_uv = b.data(uv, FLOAT, "VEC2")
    a_uv8 = b.data(np.round(uv * 255).astype(np.uint8), U8, "VEC2", normalized=True)
    a_uv16 = b.data(np.round(uv * 65535).astype(np.uint16), U16, "VEC2", normalized=True)
    p0 = {"attributes": {"POSITION": a_pos, "NORMAL": a_nrm, "TEXCOORD_0": a_uv}, "indices": b.data(idx.astype(np.uint16), U16, "SCALAR"),
          "material": m0}
    p1 = {"attributes": {"POSITION": a_pos, "TEXCOORD_0": a_uv8}, "indices": b.data(idx[:60].astype(np.uint8), U8, "SCALAR"),
          "material": m1, "mode": 5}
    p2 = {"attributes": {"POSITION": a_pos, "NORMAL": a_nrm, "TEXCOORD_0": a_uv16}, "material": m3, "mode": 6}
    p3 = {"attributes": {"POSITION": a_pos}, "indices": b.data(idx[:30].astype(np.uint32), U32, "SCALAR"), "mode": 4}
    p4 = {"attributes": {"POSITION": a_pos}, "indices": b.data(idx[:12].astype(np.uint16), U16, "SCALAR"), "mode": 1,
          "material": m1}
    mesh_a = b.mesh([p0, p1, p2, p3, p4])
    lpos, lnrm, luv, lidx = grid(3, 3, 0.5, z=1.5, seed=2)
    mesh_l = b.mesh([{"attributes": {"POSITION": b.data(lpos, FLOAT, "VEC3", bounds=True), "TEXCOORD_0": b.data(luv, FLOAT, "VEC2")},
                      "indices": b.data(lidx.astype(np.uint32), U32, "SCALAR"), "material": m2}])
    q = np.array([0.2, -0.3, 0.1, 0.9])
    q = q / np.linalg.norm(q)
    child = b.node(name="child", mesh=mesh_a, matrix=[1.1, 0.1, 0, 0, -0.1, 0.9, 0.2, 0, 0, -0.2, 1.2, 0, 0.3, -0.4, 0.5, 1])
    lamp = b.node(name="lamp", mesh=mesh_l, scale=[1.5, 1.5, 1.0], translation=[0.0, 0.2, 0.0])
    b.node(name="root", children=[child, lamp], translation=[0.5, 1.0, -0.25], rotation=q.tolist(), scale=[2.0, 2.0, 2.0])
    b.node(name="second", mesh=mesh_a, rotation=[0.0, 0.7071068, 0.0, 0.7071068])
    b.j["scenes"] = [{"nodes": [2, 3]}, {"nodes": [3]}]
    b.j["scene"] = 0
    return b.glb()


def external(directory):
    b = Builder()
    t16 = b.image_uri("tex16.png")
    tpng = b.image_uri("tex%20b.png")
    m0 = b.material({"name": "flat", "pbrMetallicRoughness": {"baseColorFactor": [0.9, 0.2, 0.2, 1.0],
                                                             "baseColorTexture": {"index": tpng}},
                     "extensions": {"KHR_materials_unlit": {}}})
    m1 = b.material({"name": "Toon_Outline", "pbrMetallicRoughness": {"baseColorFactor": [0, 0, 0, 1]}})
    m2 = b.material({"name": "deep", "pbrMetallicRoughness": {"baseColorTexture": {"index": t16}, "roughnessFactor": 0.3}})
    pos, nrm, uv, idx = grid(6, 5, 1.0, seed=3)
    a_pos = b.data(pos, FLOAT, "VEC3", bounds=True)
    a_uv = b.data(uv, FLOAT, "VEC2")
    a_idx = b.data(idx.astype(np.uint16), U16, "SCALAR")
    mesh = b.mesh([{"attributes": {"POSITION": a_pos, "TEXCOORD_0": a_uv}, "indices": a_idx, "material": m0},
                   {"attributes": {"POSITION": a_pos}, "indices": a_idx, "material": m1},
                   {"attributes": {"POSITION": a_pos, "TEXCOORD_0": a_uv}, "indices": a_idx, "material": m2}])
    bpos, _, _, bidx = grid(3, 3, 50.0, seed=4)
    bmesh = b.mesh([{"attributes": {"POSITION": b.data(bpos, FLOAT, "VEC3", bounds=True)},
                     "indices": b.data(bidx.astype(np.uint8), U8, "SCALAR")}])
    n0 = b.node(name="thing", mesh=mesh, translation=[0.0, 0.0, 1.0])
    n1 = b.node(name="Background", mesh=bmesh)
    b.j["scenes"] = [{"nodes": [n0, n1]}]
    # second buffer as a data URI holding extra normals for the first primitive
    extra = nrm.astype(np.float32).tobytes()
    b.j["buffers"] = [{"uri": "external.bin", "byteLength": len(b.bin)},
                      {"uri": "data:application/octet-stream;base64," + base64.b64encode(extra).decode(), "byteLength": len(extra)}]
    b.j["bufferViews"].append({"buffer": 1, "byteOffset": 0, "byteLength": len(extra)})
    b.j["accessors"].append({"bufferView": len(b.j["bufferViews"]) - 1, "componentType": FLOAT, "count": len(nrm), "type": "VEC3"})
    b.j["meshes"][mesh]["primitives"][0]["attributes"]["NORMAL"] = len(b.j["accessors"]) - 1
    with open(os.path.join(directory, "external.bin"), "wb") as f:
        f.write(bytes(b.bin))
    with open(os.path.join(directory, "tex16.png"), "wb") as f:
        f.write(_fixture("rgba16_31x33"))
    with open(os.path.join(directory, "tex b.png"), "wb") as f:
        f.write(_fixture("p4t_9x17"))
    return json.dumps(b.j, indent=1).encode()


def outliers():
    b = Builder()
    m = b.material({"name": "plain", "pbrMetallicRoughness": {"baseColorFactor": [0.5, 0.5, 0.5, 1.0]}})
    prims = []
    for k, (size, off) in enumerate([(1.0, 0.0), (1.2, 0.5), (0.9, -0.4), (1.1, 0.2), (40.0, 0.0), (1.0, 60.0)]):
        pos, _, _, idx = grid(4, 4, size, seed=10 + k)
        pos = pos + np.array([off, 0.0, 0.0], np.float32)
        prims.append({"attributes": {"POSITION": b.data(pos, FLOAT, "VEC3", bounds=True)},
                      "indices": b.data(idx.astype(np.uint16), U16, "SCALAR"), "material": m})
    b.node(name="all", mesh=b.mesh(prims))
    b.j["scenes"] = [{"nodes": [0]}]
    return b.glb()


def noscene():
    b = Builder()
    pos, nrm, uv, idx = grid(4, 3, 1.0, seed=20)
    mesh = b.mesh([{"attributes": {"POSITION": b.data(pos, FLOAT, "VEC3", bounds=True), "NORMAL": b.data(nrm, FLOAT, "VEC3")},
                    "indices": b.data(idx.astype(np.uint16), U16, "SCALAR")}])
    c = b.node(name="leaf", mesh=mesh, translation=[0.0, 1.0, 0.0])
    b.node(name="top", mesh=mesh, children=[c], scale=[0.5, 0.5, 0.5])
    b.j["buffers"] = [{"uri": "data:application/gltf-buffer;base64," + base64.b64encode(bytes(b.bin)).decode(),
                       "byteLength": len(b.bin)}]
    return json.dumps(b.j).encode()


def write_models(directory: str) -> dict:
    os.makedirs(directory, exist_ok=True)
    files = {"rich.glb": rich(), "external.gltf": external(directory), "outliers.glb": outliers(), "noscene.gltf": noscene()}
    for name, data in files.items():
        with open(os.path.join(directory, name), "wb") as f:
            f.write(data)
    return {name: os.path.join(directory, name) for name in files}
