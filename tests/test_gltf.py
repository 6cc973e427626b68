"""glTF 2.0 / GLB models (bte_gltf.cpp) against the reference's own loader.

The reference flattens <model> drop-ins with src/gltf_loader.cpp (tinygltf + stb_image + GLM).  That file is
compiled on the host unmodified (oracle/_ref/libbteref_gltf.so, with its vendored tinygltf and stb_image and
a GLM shim, GLM being absent) and its output is compared with the library's reader bit for bit: triangles
(positions, shading normals, uvs), material slots, Disney BSDFs, emission and RGBA8 images.  The models
(tests/golden/gltf_models.py) cover the GLB container, external and data-URI buffers, strided and
normalized accessors, every index type, strips / fans / lines, node hierarchies, every KHR material
extension the reference maps, the skipped backdrop / outline primitives, the outlier culling, a 16-bit
texture and a file without scenes.  No GPU is needed."""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, bits

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import gltf_models  # noqa: E402

REF_GLTF = os.path.join(ROOT, "oracle", "_ref", "libbteref_gltf.so")
REF_LOADER = os.path.join(ROOT, "oracle", "_ref", "libbteref_loader.so")
TRANSFORMS = [[0, 0, 0, 0, 0, 0, 1, 1, 1], [1.5, -2, 0.25, 30, -45, 10, 2, 0.5, 1.5]]


def _need(path):
    if not os.path.exists(path):
        import oracle as O
        if not O.reference_present():
            pytest.skip("reference harness not built")
        O.build(ref=True)


@pytest.fixture(scope="module")
def models(tmp_path_factory):
    return gltf_models.write_models(str(tmp_path_factory.mktemp("gltf")))


_REF_SCRIPT = r"""
import ctypes as C, sys, numpy as np
sys.path.insert(0, ROOT)
import bluetruthengine_b200 as bte
lib = C.CDLL(LIB)
xf = np.array(XF, np.float32)
n = lib.refg_load(PATH.encode(), xf.ctypes.data_as(C.c_void_p))
tris = np.empty(n, bte.TRIANGLE_DTYPE)
ids = np.empty(n, np.int32)
lib.refg_triangles(tris.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p))
out = dict(tris=tris.view(np.uint8), ids=ids)
p = lambda a: a.ctypes.data_as(C.c_void_p)
for i in range(lib.refg_material_count()):
    b, em, ie = np.zeros(1, bte.BSDF_DTYPE), np.zeros(3, np.float32), C.c_int()
    a, m = np.zeros(2, np.int32), np.zeros(2, np.int32)
    lib.refg_material(i, p(b), p(em), C.byref(ie), p(a), p(m), None, None)
    alb = np.zeros((max(a[1], 1), max(a[0], 1), 4), np.uint8)
    mr = np.zeros((max(m[1], 1), max(m[0], 1), 4), np.uint8)
    lib.refg_material(i, p(b), p(em), C.byref(ie), p(a), p(m), p(alb), p(mr))
    out["b%d" % i] = b.view(np.uint8)
    out["e%d" % i] = em
    out["ie%d" % i] = np.array([ie.value])
    out["a%d" % i] = alb if a[0] else np.zeros(0, np.uint8)
    out["m%d" % i] = mr if m[0] else np.zeros(0, np.uint8)
np.savez(OUT, **out)
"""


def _reference_model(path, xf, out):
    """The reference's loadGltfModel in a child process (it exits the process on a load failure)."""
    code = (f"ROOT={ROOT!r}\nLIB={REF_GLTF!r}\nXF={list(xf)!r}\nPATH={path!r}\nOUT={out!r}\n") + _REF_SCRIPT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


@pytest.mark.parametrize("name", ["rich.glb", "external.gltf", "outliers.glb", "noscene.gltf"])
@pytest.mark.parametrize("xf", [0, 1])
def test_model_matches_reference_loader(bte, models, tmp_path, name, xf):
    _need(REF_GLTF)
    path = models[name]
    ours = bte.load_gltf(path, TRANSFORMS[xf])
    ref = _reference_model(path, TRANSFORMS[xf], str(tmp_path / "ref.npz"))
    assert len(ours["triangles"]) == len(ref["ids"]) > 0
    assert np.array_equal(ours["triangles"].view(np.uint8), ref["tris"])
    assert np.array_equal(ours["material_ids"], ref["ids"])
    assert len(ours["materials"]) == sum(1 for k in ref.files if k.startswith("b"))
    for i, m in enumerate(ours["materials"]):
        assert np.array_equal(np.frombuffer(m["bsdf"].tobytes(), np.uint8), ref["b%d" % i].reshape(-1)), i
        assert np.array_equal(bits(m["emission"]), bits(ref["e%d" % i])) and m["is_emitter"] == bool(ref["ie%d" % i][0])
        for key, rk in (("albedo", "a"), ("mr", "m")):
            r = ref["%s%d" % (rk, i)]
            if m[key] is None:
                assert r.size == 0, (i, key)
            else:
                assert r.shape == m[key].shape and np.array_equal(r, m[key]), (i, key)


def test_model_features_are_exercised(bte, models):
    """The fixtures reach the paths they are meant to: skipped primitives, culled outliers, textures,
    emission, the default material, a 16-bit texture read four bytes per pixel."""
    rich = bte.load_gltf(models["rich.glb"])
    mats = rich["materials"]
    assert any(m["is_emitter"] for m in mats)
    assert mats[0]["albedo"] is not None and mats[0]["mr"] is not None
    assert len(mats) == 5   # four file materials + the default one (a primitive without material)
    ext = bte.load_gltf(models["external.gltf"])
    assert len(ext["triangles"]) == 80   # the outline primitive and the Background node are skipped
    assert np.asarray(ext["materials"][0]["bsdf"]["p0"]).reshape(-1)[3] == 1.0   # unlit: roughness 1
    assert bte.load_gltf(models["outliers.glb"])["skipped_outliers"] == 2
    ns = bte.load_gltf(models["noscene.gltf"])
    assert len(ns["triangles"]) == 3 * 12   # the child node is walked as a root and as a child


def _scene_with_models(tmp_path, models):
    from bluetruthengine_b200 import scenes
    import re
    src = scenes.cornell()
    d = os.path.dirname(src)
    xml = open(src).read()
    xml = re.sub(r'filename="([^"]+)"', lambda m: f'filename="{os.path.join(d, m.group(1))}"', xml)
    add = (f'<model filename="{models["rich.glb"]}" posX="270" posY="150" posZ="300" rotY="25" scaleX="60" scaleY="60" '
           f'scaleZ="60" />\n<model filename="{models["external.gltf"]}" posX="120" posY="300" posZ="200" scaleX="80" '
           f'scaleY="80" scaleZ="80" rotX="-30" />\n')
    xml = xml.replace("<window", add + "<window")
    p = tmp_path / "scene_models.xml"
    p.write_text(xml)
    return str(p)


def test_scene_with_models_matches_reference(bte, models, tmp_path):
    """A scene.xml with OBJ meshes and two <model> drop-ins against the reference's flattening
    (src/main.cpp:760-817 over its loadGltfModel): triangles, BSDFs, per-triangle ids and emitter flags,
    emitter tables (the emissive glTF material becomes an area emitter), material images."""
    _need(REF_LOADER)
    path = _scene_with_models(tmp_path, models)
    sc = bte.load_scene(path)
    from test_loader import _ref_flatten
    r = _ref_flatten(bte, path)
    assert sc.triangle_count == len(r["tris"])
    assert np.array_equal(sc.triangles.view(np.uint8), r["tris"].view(np.uint8))
    assert np.array_equal(sc.bsdfs.view(np.uint8), r["bsdfs"].view(np.uint8))
    assert np.array_equal(sc.triangle_bsdf_ids, r["tb"]) and np.array_equal(sc.triangle_material_ids, r["tm"])
    assert np.array_equal(sc.triangle_emitter_flags, r["flags"])
    assert np.array_equal(sc.emitter_tri_indices, r["emTri"])
    assert np.array_equal(bits(sc.emitter_tri_cdf), bits(r["emCdf"]))
    assert np.array_equal(bits(sc.scene_emitter_cdf), bits(r["sceneCdf"]))
    lib = C.CDLL(REF_LOADER)
    lib.refl_load(path.encode())
    assert lib.refl_emitter_count() == len(sc.emitters) >= 2
    n = lib.refl_material_count()
    assert n == len(sc.materials) == len(sc.albedo_textures) == len(sc.mr_textures)
    for i in range(n):
        col = np.zeros(3, np.float32)
        w, h = C.c_int(), C.c_int()
        has = lib.refl_material(i, col.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(h), None)
        assert np.array_equal(bits(sc.materials[i]), bits(col))
        if has:
            img = np.empty((h.value, w.value, 4), np.uint8)
            lib.refl_material(i, col.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(h), img.ctypes.data_as(C.c_void_p))
            assert np.array_equal(sc.albedo_textures[i], img)
        else:
            assert sc.albedo_textures[i] is None
        has = lib.refl_material_mr(i, C.byref(w), C.byref(h), None)
        if has:
            img = np.empty((h.value, w.value, 4), np.uint8)
            lib.refl_material_mr(i, C.byref(w), C.byref(h), img.ctypes.data_as(C.c_void_p))
            assert np.array_equal(sc.mr_textures[i], img)
        else:
            assert sc.mr_textures[i] is None


def test_bad_models_fail_with_a_message(bte, models, tmp_path):
    """Unreadable models are reported through the status code (the reference exits the process)."""
    cases = {}
    glb = open(models["rich.glb"], "rb").read()
    cases["truncated.glb"] = glb[:len(glb) // 2]
    cases["badjson.gltf"] = b'{"asset": {"version": "2.0"}, "nodes": [ {"mesh": 0 ]}'
    j = json.loads(open(models["external.gltf"]).read())
    j["buffers"][0]["uri"] = "missing.bin"
    cases["missing.gltf"] = json.dumps(j).encode()
    cases["empty.gltf"] = b'{"asset": {"version": "2.0"}}'
    for name, data in cases.items():
        p = tmp_path / name
        p.write_bytes(data)
        with pytest.raises(bte.BteError):
            bte.load_gltf(str(p))
    with pytest.raises(bte.BteError, match="cannot open"):
        bte.load_gltf(str(tmp_path / "nope.glb"))
