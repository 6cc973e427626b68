"""Texture decoding (bte_image.cpp) against the reference's decoder, and textured materials in the loader.

The reference loads albedo textures with its vendored stb_image (stbi_load(..., 4), src/main.cpp:407-470).
tests/golden/images/fixtures.npz holds 160 PNG / JPEG files (every PNG colour type and bit depth, filters,
Adam7, tRNS; baseline JPEG 4:4:4 / 4:2:2 / 4:2:0 / 4:4:0 / grey, restart intervals, files written by the
reference's own encoder) with the RGBA8 bytes stb_image decodes from each (tests/golden/make_image_golden.py).
The library's decoder must give the same bytes.  No GPU is needed."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, bits
import oracle as _O  # the checker's reference-tree location (conftest puts oracle/ on the path)

FIX = os.path.join(ROOT, "tests", "golden", "images", "fixtures.npz")
REF_ASSETS = os.path.join(_O.REFERENCE_ROOT, "assets")
REF_CHECKER = os.path.join(REF_ASSETS, "checkerboard.jpg")


@pytest.fixture(scope="module")
def fixtures():
    z = np.load(FIX)
    return z, [str(n) for n in z["names"]], [int(c) for c in z["comps"]]


def test_fixture_set_covers_the_formats(fixtures):
    _, names, _ = fixtures
    kinds = {n.split("_")[0] for n in names}
    for k in ["g1", "g2", "g4", "g8", "g16", "rgb8", "rgb8i", "rgb16", "ga8", "ga16", "rgba8", "rgba16", "p1", "p2",
              "p4", "p8", "p1t", "p8t", "g8key", "g2key", "rgbkey", "rgb16key", "j444", "j422", "j420", "j440", "jgray",
              "jstb"]:
        assert k in kinds, k
    assert len(names) >= 150


def test_decoder_matches_reference_decoder_bit_for_bit(bte, fixtures):
    z, names, comps = fixtures
    for name, comp in zip(names, comps):
        got = bte.decode_image(z["file_" + name].tobytes())
        exp = z["rgba_" + name]
        assert got.shape == exp.shape, name
        diff = np.argwhere(got != exp)
        assert len(diff) == 0, f"{name}: {len(diff)} bytes differ, first at {diff[:3].tolist()}"


def test_channel_count_matches_reference(bte, fixtures):
    import ctypes as C
    z, names, comps = fixtures
    lib = bte.load_library()
    for name, comp in zip(names, comps):
        buf = z["file_" + name]
        w, h, c = C.c_int(), C.c_int(), C.c_int()
        assert lib.bte_image_decode(buf.ctypes.data_as(C.c_void_p), C.c_longlong(len(buf)), None, C.c_longlong(0),
                                    C.byref(w), C.byref(h), C.byref(c)) == 0
        assert c.value == comp, name


@pytest.mark.skipif(not os.path.exists(REF_CHECKER), reason="reference tree not present")
def test_reference_asset_checkerboard_jpg(bte):
    """The reference's own floor texture (2048x2048 baseline JPEG) against its stb_image, compiled on the host."""
    import ctypes as C
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libstbref.so")
    if not os.path.exists(lib_path):
        import oracle as O
        O.build(ref=True)
    ref = C.CDLL(lib_path)
    data = open(REF_CHECKER, "rb").read()
    got = bte.decode_image(data)
    buf = np.frombuffer(data, np.uint8)
    exp = np.empty_like(got)
    w, h, c = C.c_int(), C.c_int(), C.c_int()
    assert ref.ref_stbi_decode_rgba(buf.ctypes.data_as(C.c_void_p), len(buf), exp.ctypes.data_as(C.c_void_p),
                                    C.c_longlong(exp.size), C.byref(w), C.byref(h), C.byref(c)) == 0
    assert got.shape == (2048, 2048, 4) and np.array_equal(got, exp)


def test_corrupt_and_unsupported_inputs_fail_with_a_message(bte, fixtures):
    z, _, _ = fixtures
    png = z["file_rgb8_31x33"].tobytes()
    jpg = z["file_j420_q60_37x29"].tobytes()
    cases = [
        (png[:40], "PNG"),
        (png[:8] + b"\x00" * 30, "PNG"),
        (jpg[:len(jpg) // 3], "JPEG"),
        (jpg.replace(b"\xff\xc0", b"\xff\xc2", 1), "progressive"),
        (b"GIF89a" + b"\x00" * 20, "unsupported image format"),
    ]
    for data, msg in cases:
        with pytest.raises(bte.BteError, match=msg):
            bte.decode_image(data)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_ASSETS, "scene.xml")), reason="reference tree not present")
def test_reference_scene_xml_materials(bte, monkeypatch, tmp_path):
    """The reference's own assets/scene.xml (its floor textured by assets/checkerboard.jpg), loaded from a
    working directory where assets/ is the reference's, as its application runs: material colours and texture
    bytes equal those of the reference's loader glue with its stb_image.  Its <model> entries name .glb files
    the reference does not ship (its application exits on them, and this loader reports an error), so they are
    taken out of the copy."""
    import ctypes as C
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libbteref_loader.so")
    if not os.path.exists(ref_path):
        import oracle as O
        O.build(ref=True)
    os.symlink(REF_ASSETS, tmp_path / "assets")
    xml = open(os.path.join(REF_ASSETS, "scene.xml")).read()
    (tmp_path / "scene.xml").write_text(re.sub(r"<model\b[^>]*/>", "", xml, flags=re.S))
    monkeypatch.chdir(tmp_path)
    with pytest.raises(bte.BteError, match="sakutaro.glb"):
        bte.load_scene(os.path.join(REF_ASSETS, "scene.xml"))
    sc = bte.load_scene("scene.xml")
    lib = C.CDLL(ref_path)
    lib.refl_load(b"scene.xml")
    n = lib.refl_material_count()
    assert n == len(sc.materials) and n > 0
    textured = 0
    for i in range(n):
        col = np.zeros(3, np.float32)
        w, h = C.c_int(), C.c_int()
        has = lib.refl_material(i, col.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(h), None)
        assert np.array_equal(bits(sc.materials[i]), bits(col)), i
        if has:
            img = np.empty((h.value, w.value, 4), np.uint8)
            lib.refl_material(i, col.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(h), img.ctypes.data_as(C.c_void_p))
            assert np.array_equal(sc.albedo_textures[i], img)
            textured += 1
        else:
            assert sc.albedo_textures[i] is None
    assert textured >= 1


def _textured_cornell(tmp_path, fixtures, textures):
    """The Cornell scene with albedoTexture on its materials, meshes by absolute path."""
    from bluetruthengine_b200 import scenes
    z, _, _ = fixtures
    src = scenes.cornell()
    d = os.path.dirname(src)
    xml = open(src).read()
    xml = re.sub(r'filename="([^"]+)"', lambda m: f'filename="{os.path.join(d, m.group(1))}"', xml)
    for mat, (name, ext) in textures.items():
        f = tmp_path / f"{name}.{ext}"
        f.write_bytes(z["file_" + name].tobytes())
        xml = xml.replace(f'<material name="{mat}" ', f'<material name="{mat}" albedoTexture="{f}" ')
    p = tmp_path / "scene.xml"
    p.write_text(xml)
    return str(p)


def test_textured_materials_match_reference_loader(bte, tmp_path, fixtures):
    """Material colours (the texture's mean, summed in double as src/main.cpp:407-438) and the RGBA8 images of
    textured scene.xml materials against the reference's loader glue with its stb_image; a missing texture
    falls back to white and no image, as the reference's does."""
    import ctypes as C
    path = _textured_cornell(tmp_path, fixtures, {"whiteMat": ("j420_q60_64x48", "jpg"), "redMat": ("rgba16_31x33", "png"),
                                                  "greenMat": ("p4t_9x17", "png")})
    xml = open(path).read().replace('<material name="lightMat" ', '<material name="lightMat" albedoTexture="missing.png" ')
    open(path, "w").write(xml)
    sc = bte.load_scene(path)
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libbteref_loader.so")
    if not os.path.exists(ref_path):
        import oracle as O
        if not O.reference_present():
            pytest.skip("reference loader harness not built")
        O.build(ref=True)
    lib = C.CDLL(ref_path)
    lib.refl_load(path.encode())
    assert lib.refl_material_count() == len(sc.materials) == 4
    for i in range(4):
        col = np.zeros(3, np.float32)
        w, h = C.c_int(), C.c_int()
        has = lib.refl_material(i, col.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(h), None)
        assert np.array_equal(bits(sc.materials[i]), bits(col)), i
        if has:
            img = np.empty((h.value, w.value, 4), np.uint8)
            lib.refl_material(i, col.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(h), img.ctypes.data_as(C.c_void_p))
            assert sc.albedo_textures[i] is not None and np.array_equal(sc.albedo_textures[i], img), i
        else:
            assert sc.albedo_textures[i] is None
    assert sc.albedo_textures[3] is None and np.array_equal(sc.materials[3], [1, 1, 1])
    assert all(m is None for m in sc.mr_textures)


def _png_pixels_via_zlib(png: bytes) -> np.ndarray:
    """A third decoder for our own files (RGBA8, non-interlaced): Python's zlib and the five filters."""
    import struct
    import zlib
    assert png[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = 0
    while pos < len(png):
        n, t = struct.unpack(">I4s", png[pos:pos + 8])
        data = png[pos + 8:pos + 8 + n]
        assert struct.unpack(">I", png[pos + 8 + n:pos + 12 + n])[0] == zlib.crc32(t + data) & 0xffffffff
        if t == b"IHDR":
            w, h, depth, color = struct.unpack(">IIBB", data[:10])
            assert (depth, color) == (8, 6)
        elif t == b"IDAT":
            idat += data
        pos += 12 + n
    raw = zlib.decompress(idat)
    out = np.zeros((h, w * 4), np.int64)
    prior = np.zeros(w * 4, np.int64)
    for y in range(h):
        f = raw[y * (w * 4 + 1)]
        row = np.frombuffer(raw[y * (w * 4 + 1) + 1:(y + 1) * (w * 4 + 1)], np.uint8).astype(np.int64)
        cur = np.zeros(w * 4, np.int64)
        for i in range(w * 4):
            a = cur[i - 4] if i >= 4 else 0
            b = prior[i]
            c = prior[i - 4] if i >= 4 else 0
            p = a + b - c
            pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
            pred = [0, a, b, (a + b) // 2, a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)][f]
            cur[i] = (row[i] + pred) & 255
        out[y] = cur
        prior = cur
    return out.reshape(h, w, 4).astype(np.uint8)


@pytest.mark.parametrize("shape", [(1, 1), (7, 5), (40, 33), (64, 128)])
def test_png_encoder_roundtrip(bte, shape):
    """The screenshot encoder's files decode to the exact pixels with the library's decoder, with a plain
    zlib reader (CRCs checked), and with the reference's stb_image when it is built."""
    import ctypes as C
    rng = np.random.default_rng(shape[0] * 31 + shape[1])
    h, w = shape
    img = np.concatenate([rng.integers(0, 256, size=(h, w // 2 + 1, 4)), np.tile(rng.integers(0, 256, size=(h, 1, 4)),
                                                                                (1, w - w // 2 - 1, 1))], 1)[:, :w]
    img = np.ascontiguousarray(img.astype(np.uint8))
    png = bte.encode_png(img)
    assert np.array_equal(bte.decode_image(png), img)
    assert np.array_equal(_png_pixels_via_zlib(png), img)
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libstbref.so")
    if os.path.exists(lib_path):
        ref = C.CDLL(lib_path)
        buf = np.frombuffer(png, np.uint8)
        out = np.empty_like(img)
        ww, hh, cc = C.c_int(), C.c_int(), C.c_int()
        assert ref.ref_stbi_decode_rgba(buf.ctypes.data_as(C.c_void_p), len(buf), out.ctypes.data_as(C.c_void_p),
                                        C.c_longlong(out.size), C.byref(ww), C.byref(hh), C.byref(cc)) == 0
        assert np.array_equal(out, img)
