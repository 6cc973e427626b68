"""scene.xml / OBJ / .hdr loader (bte_scene.cpp) against the reference's own
parser, OBJ reader and transforms (oracle/ref_loader.cpp), plus its error
behaviour (status codes instead of process exit)."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, bits

REF_LOADER = os.path.join(ROOT, "oracle", "_ref", "libbteref_loader.so")


def _ref_flatten(bte, path):
    if not os.path.exists(REF_LOADER):
        import oracle as O
        if O.reference_present():
            O.build(ref=True)
        else:
            pytest.skip("reference loader harness not built")
    lib = C.CDLL(REF_LOADER)
    lib.refl_load(path.encode())
    cnt = np.zeros(6, np.int32)
    lib.refl_counts(cnt.ctypes.data_as(C.c_void_p))
    T, B, E, EC, SC, NC = (int(x) for x in cnt)
    tris = np.empty(T, bte.TRIANGLE_DTYPE)
    bsdfs = np.empty(B, bte.BSDF_DTYPE)
    tb, tm = np.empty(T, np.int32), np.empty(T, np.int32)
    fl = np.empty(T, np.uint8)
    et, ec, sc, cam = np.empty(E, np.int32), np.empty(EC, np.float32), np.empty(SC, np.float32), np.empty(NC, np.float32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    lib.refl_copy(p(tris), p(bsdfs), p(tb), p(tm), p(fl), p(et), p(ec), p(sc), p(cam))
    return dict(tris=tris, bsdfs=bsdfs, tb=tb, tm=tm, flags=fl, emTri=et, emCdf=ec, sceneCdf=sc, cam=cam)


@pytest.mark.parametrize("which", ["cornell", "random", "disney"])
def test_loader_matches_reference_parser(bte, which):
    from bluetruthengine_b200 import scenes
    path = {"cornell": scenes.cornell, "random": lambda: scenes.random_scene(5), "disney": scenes.disney_spheres}[which]()
    sc = bte.load_scene(path)
    r = _ref_flatten(bte, path)
    assert sc.triangle_count == len(r["tris"])
    assert np.array_equal(sc.triangles.view(np.uint32).reshape(-1), r["tris"].view(np.uint32).reshape(-1))
    assert np.array_equal(sc.bsdfs.view(np.uint8), r["bsdfs"].view(np.uint8))
    assert np.array_equal(sc.triangle_bsdf_ids, r["tb"]) and np.array_equal(sc.triangle_material_ids, r["tm"])
    assert np.array_equal(sc.triangle_emitter_flags, r["flags"])
    assert np.array_equal(sc.emitter_tri_indices, r["emTri"])
    assert np.array_equal(bits(sc.emitter_tri_cdf), bits(r["emCdf"]))
    assert np.array_equal(bits(sc.scene_emitter_cdf), bits(r["sceneCdf"]))
    cam = r["cam"]
    assert sc.width == int(cam[10]) and sc.height == int(cam[11])
    assert np.float32(sc.env_intensity) == cam[12] and np.float32(sc.env_rotation_deg) == cam[13]
    assert len(sc.spotlights) == int(cam[14])
    assert np.array_equal(bits(sc.camera["origin"]), bits(cam[0:3]))


@pytest.mark.parametrize("which", ["cornell", "random", "disney"])
def test_reference_scene_matches_loader(bte, which):
    """The whole upload set flattened by the reference's loader alone (oracle.RefScene: emitter table,
    per-triangle emission, spotlights, the .hdr env map through the reference's stb_image, camera basis)
    equals the product loader's, byte for byte.  The reference arm of the bench renders RefScene."""
    import oracle as O
    from bluetruthengine_b200 import scenes
    if not (os.path.exists(REF_LOADER) or O.reference_present()):
        pytest.skip("reference loader harness not built")
    path = {"cornell": scenes.cornell, "random": lambda: scenes.random_scene(5), "disney": scenes.disney_spheres}[which]()
    r = O.RefScene(path)
    s = bte.load_scene(path)
    same = lambda a, b: np.ascontiguousarray(a).tobytes() == np.ascontiguousarray(b).tobytes()  # noqa: E731
    assert same(r.triangles, s.triangles) and same(r.bsdfs, s.bsdfs)
    assert same(r.emitters, s.emitters) and same(r.spotlights, s.spotlights)
    assert same(np.asarray(r.triangle_emission, np.float32), np.asarray(s.triangle_emission, np.float32))
    assert (r.env_rgba is None) == (s.env_rgba is None)
    if r.env_rgba is not None:
        assert same(r.env_rgba, s.env_rgba)
    assert same(r.camera, s.camera)
    assert (r.width, r.height, r.env_intensity, r.env_rotation_deg) == \
        (s.width, s.height, np.float32(s.env_intensity), np.float32(s.env_rotation_deg))


def test_cornell_contents(cornell_scene):
    sc = cornell_scene
    assert sc.triangle_count == 36 and sc.width == 256 and sc.height == 256
    assert len(sc.emitters) == 1
    e = sc.emitters[0]
    assert e["triCount"] == 2 and e["areaSum"] == np.float32(130 * 105)
    assert np.array_equal(e["radiance"], np.array([17, 12, 4], np.float32))
    assert int(sc.triangle_emitter_flags.sum()) == 2
    cam = sc.camera
    f, r, u = cam["forward"], cam["right"], cam["up"]
    assert abs(np.dot(f, r)) < 1e-6 and abs(np.dot(f, u)) < 1e-6 and abs(np.linalg.norm(u) - 1) < 1e-6
    # every wall faces into the box; the light faces down
    light = sc.triangles[sc.triangle_emitter_flags == 1]
    assert np.all(light["n0"][:, 1] < -0.99)


def test_hdr_roundtrip(bte, random_scene):
    from bluetruthengine_b200 import scenes
    expect = scenes.rgbe_decode(scenes.rgbe_encode(scenes.sky_env(64, 32, sun_radius_deg=6.0, sun_radiance=50.0)))
    assert np.array_equal(bits(random_scene.env_rgba), bits(expect))


def _write(tmp_path, xml, objs=None):
    for name, txt in (objs or {}).items():
        (tmp_path / name).write_text(txt)
    p = tmp_path / "scene.xml"
    p.write_text(xml)
    return str(p)


TRI = "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n"
OK_TAIL = '<window width="8" height="8" /><camera eyeX="0" eyeY="0" eyeZ="-5" lookAtX="0" lookAtY="0" lookAtZ="0" upX="0" upY="1" upZ="0" fovY="40" />'


@pytest.mark.parametrize("xml,msg", [
    ('<bsdf name="a" type="velvet" /><material name="m" bsdf="a" /><mesh filename="t.obj" material="m" />' + OK_TAIL,
     "unsupported type"),
    ('<bsdf name="a" type="diffuse" albedoR="x1" /><material name="m" bsdf="a" /><mesh filename="t.obj" material="m" />'
     + OK_TAIL, "invalid float"),
    ('<bsdf name="a" type="diffuse" /><material name="m" bsdf="a" /><mesh filename="t.obj" material="m" />'
     '<window width="8" height="8" />', "camera"),
    ('<bsdf name="a" type="diffuse" /><material name="m" bsdf="zz" /><mesh filename="t.obj" material="m" />' + OK_TAIL,
     "not found"),
    ('<bsdf name="a" type="diffuse" /><material name="m" bsdf="a" /><mesh filename="missing.obj" material="m" />'
     + OK_TAIL, "failed to load OBJ"),
])
def test_loader_errors_are_status_codes(bte, tmp_path, xml, msg):
    path = _write(tmp_path, "<scene>" + xml + "</scene>", {"t.obj": TRI})
    with pytest.raises(bte.BteError, match=msg):
        bte.load_scene(path)


def test_obj_forms_and_negative_indices(bte, tmp_path):
    obj = ("v 0 0 0\nv 2 0 0\nv 0 2 0\nv 2 2 0\nvn 0 0 1\nvt 0 0\nvt 1 0\nvt 0 1\n"
           "f 1/1/1 2/2/1 3/3/1\nf -3//-1 -1//-1 -2//-1\nf 1 2 4 3\n")
    path = _write(tmp_path, '<scene><bsdf name="a" type="diffuse" /><material name="m" bsdf="a" />'
                  '<mesh filename="q.obj" material="m" scaleX="2" rotZ="90" posX="1" />' + OK_TAIL + "</scene>",
                  {"q.obj": obj})
    sc = bte.load_scene(path)
    assert sc.triangle_count == 4   # 1 + 1 + quad fan (2)
    assert np.allclose(sc.triangles["n0"][0], [0, 0, 1], atol=1e-6)
