"""Writes tests/golden/images/: PNG and JPEG fixtures and, for each, the RGBA8 pixels the reference's own
texture decoder (its vendored stb_image, stbi_load_from_memory(..., 4), compiled on the host into
oracle/_ref/libstbref.so by oracle/Makefile) produces.  Run in a container that has the reference tree:

    make -C oracle ref && python tests/golden/make_image_golden.py

PNG fixtures come from the encoder below (every colour type and bit depth, all five filters, Adam7,
tRNS keys and palette alpha, stored / fixed / dynamic DEFLATE blocks); JPEG fixtures from the encoder
below (baseline, 4:4:4 / 4:2:2 / 4:2:0 / grey, with and without restart intervals) and from the
reference's vendored stb_image_write.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "images")


# ---------------------------------------------------------------- PNG encoder
def _chunk(t: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + t + data + struct.pack(">I", zlib.crc32(t + data) & 0xffffffff)


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)


def _filter_rows(rows, bpp, first_filter=0):
    out = bytearray()
    prior = bytes(len(rows[0])) if rows else b""
    for i, row in enumerate(rows):
        f = (first_filter + i) % 5
        x = bytearray(len(row))
        for k in range(len(row)):
            a = row[k - bpp] if k >= bpp else 0
            b = prior[k]
            c = prior[k - bpp] if k >= bpp else 0
            pred = [0, a, b, (a + b) // 2, _paeth(a, b, c)][f]
            x[k] = (row[k] - pred) & 255
        out.append(f)
        out += x
        prior = row
    return bytes(out)


def _pack_row(samples, depth):
    if depth == 8:
        return bytes(int(v) for v in samples)
    if depth == 16:
        return b"".join(struct.pack(">H", int(v)) for v in samples)
    per = 8 // depth
    out = bytearray()
    for i in range(0, len(samples), per):
        byte = 0
        for j in range(per):
            v = int(samples[i + j]) if i + j < len(samples) else 0
            byte |= v << (8 - depth * (j + 1))
        out.append(byte)
    return bytes(out)


def encode_png(samples, color, depth, interlace=False, level=6, palette=None, trns=None, first_filter=0):
    """samples: [H, W, channels] integers in the sample range of `depth`."""
    h, w, ch = samples.shape
    bpp = max(1, ch * depth // 8)
    passes = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
    raw = b""
    if not interlace:
        rows = [_pack_row(samples[y].reshape(-1), depth) for y in range(h)]
        raw = _filter_rows(rows, bpp, first_filter)
    else:
        for (x0, y0, dx, dy) in passes:
            sub = samples[y0::dy, x0::dx]
            if sub.shape[0] == 0 or sub.shape[1] == 0:
                continue
            rows = [_pack_row(sub[y].reshape(-1), depth) for y in range(sub.shape[0])]
            raw += _filter_rows(rows, bpp, first_filter)
    png = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, color, 0, 0, 1 if interlace else 0))
    png += _chunk(b"tEXt", b"Comment\x00fixture")   # an ancillary chunk to skip
    if palette is not None:
        png += _chunk(b"PLTE", bytes(np.asarray(palette, dtype=np.uint8).reshape(-1)))
    if trns is not None:
        png += _chunk(b"tRNS", trns)
    comp = zlib.compress(raw, level)
    half = len(comp) // 2   # two IDAT chunks
    png += _chunk(b"IDAT", comp[:half]) + _chunk(b"IDAT", comp[half:]) + _chunk(b"IEND", b"")
    return png


# ---------------------------------------------------------------- JPEG encoder (baseline, T.81 Annex K tables)
ZZ = np.array([0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,
               7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31,
               39, 46, 53, 60, 61, 54, 47, 55, 62, 63])
QL = np.array([16, 11, 10, 16, 24, 40, 51, 61, 12, 12, 14, 19, 26, 58, 60, 55, 14, 13, 16, 24, 40, 57, 69, 56, 14, 17,
               22, 29, 51, 87, 80, 62, 18, 22, 37, 56, 68, 109, 103, 77, 24, 35, 55, 64, 81, 104, 113, 92, 49, 64, 78,
               87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99])
QC = np.array([17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99, 24, 26, 56, 99, 99, 99, 99, 99, 47, 66,
               99, 99, 99, 99, 99, 99] + [99] * 32)
DC_L = ([0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0], list(range(12)))
DC_C = ([0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0], list(range(12)))
AC_L = ([0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7d], [
    0x01, 0x02, 0x03, 0x00, 0x04, 0x11, 0x05, 0x12, 0x21, 0x31, 0x41, 0x06, 0x13, 0x51, 0x61, 0x07, 0x22, 0x71, 0x14,
    0x32, 0x81, 0x91, 0xa1, 0x08, 0x23, 0x42, 0xb1, 0xc1, 0x15, 0x52, 0xd1, 0xf0, 0x24, 0x33, 0x62, 0x72, 0x82, 0x09,
    0x0a, 0x16, 0x17, 0x18, 0x19, 0x1a, 0x25, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x34, 0x35, 0x36, 0x37, 0x38, 0x39, 0x3a,
    0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58, 0x59, 0x5a, 0x63, 0x64, 0x65,
    0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88,
    0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a, 0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9,
    0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba, 0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca,
    0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda, 0xe1, 0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea,
    0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa])
AC_C = ([0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77], [
    0x00, 0x01, 0x02, 0x03, 0x11, 0x04, 0x05, 0x21, 0x31, 0x06, 0x12, 0x41, 0x51, 0x07, 0x61, 0x71, 0x13, 0x22, 0x32,
    0x81, 0x08, 0x14, 0x42, 0x91, 0xa1, 0xb1, 0xc1, 0x09, 0x23, 0x33, 0x52, 0xf0, 0x15, 0x62, 0x72, 0xd1, 0x0a, 0x16,
    0x24, 0x34, 0xe1, 0x25, 0xf1, 0x17, 0x18, 0x19, 0x1a, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x35, 0x36, 0x37, 0x38, 0x39,
    0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58, 0x59, 0x5a, 0x63, 0x64,
    0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a, 0x82, 0x83, 0x84, 0x85, 0x86,
    0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a, 0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7,
    0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba, 0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8,
    0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda, 0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9,
    0xea, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa])


def _codes(table):
    counts, vals = table
    code, k, out = 0, 0, {}
    for ln in range(1, 17):
        for _ in range(counts[ln - 1]):
            out[vals[k]] = (code, ln)
            code += 1
            k += 1
        code <<= 1
    return out


class _Bits:
    def __init__(self):
        self.out = bytearray()
        self.acc = 0
        self.n = 0

    def put(self, v, n):
        for i in range(n - 1, -1, -1):
            self.acc = (self.acc << 1) | ((v >> i) & 1)
            self.n += 1
            if self.n == 8:
                self.out.append(self.acc)
                if self.acc == 0xFF:
                    self.out.append(0)
                self.acc, self.n = 0, 0

    def flush(self):
        while self.n:
            self.put(1, 1)


def _dct8(block):
    k = np.arange(8)
    c = np.where(k == 0, np.sqrt(1 / 8), np.sqrt(2 / 8))[:, None] * np.cos((2 * k[None, :] + 1) * k[:, None] * np.pi / 16)
    return c @ block @ c.T


def encode_jpeg(rgb, quality=75, sampling=(1, 1), restart=0, gray=False):
    """rgb: uint8 [H,W,3] (or [H,W] with gray=True). sampling: luma (H, V) factors, chroma 1x1."""
    s = 5000 / quality if quality < 50 else 200 - 2 * quality
    ql = np.clip((QL * s + 50) // 100, 1, 255).astype(int)
    qc = np.clip((QC * s + 50) // 100, 1, 255).astype(int)
    img = rgb.astype(np.float64)
    if gray:
        planes = [img]
        samp = [(1, 1)]
    else:
        r, g, b = img[..., 0], img[..., 1], img[..., 2]
        planes = [0.299 * r + 0.587 * g + 0.114 * b, -0.168736 * r - 0.331264 * g + 0.5 * b + 128,
                  0.5 * r - 0.418688 * g - 0.081312 * b + 128]
        samp = [sampling, (1, 1), (1, 1)]
    H, W = planes[0].shape
    hm, vm = max(s_[0] for s_ in samp), max(s_[1] for s_ in samp)
    mx, my = -(-W // (8 * hm)), -(-H // (8 * vm))
    comps = []
    for p, (sh, sv) in zip(planes, samp):
        fx, fy = hm // sh, vm // sv
        pw, ph = mx * 8 * hm, my * 8 * vm
        full = np.pad(p, ((0, ph - H), (0, pw - W)), mode="edge")
        sub = full.reshape(ph // fy, fy, pw // fx, fx).mean(axis=(1, 3))
        comps.append(sub)
    tabs = [(_codes(DC_L), _codes(AC_L), ql)] + [(_codes(DC_C), _codes(AC_C), qc)] * 2
    bits = _Bits()
    preds = [0] * len(comps)
    out_mcus, rst = 0, 0
    for my_ in range(my):
        for mx_ in range(mx):
            if restart and out_mcus and out_mcus % restart == 0:
                bits.flush()
                bits.out += bytes([0xFF, 0xD0 + rst])
                rst = (rst + 1) % 8
                preds = [0] * len(comps)
            for ci, (sub, (sh, sv)) in enumerate(zip(comps, samp)):
                dct_t, ac_t, q = tabs[ci]
                for v in range(sv):
                    for h_ in range(sh):
                        by, bx = (my_ * sv + v) * 8, (mx_ * sh + h_) * 8
                        blk = _dct8(sub[by:by + 8, bx:bx + 8] - 128).reshape(-1)
                        zz = np.round(blk[ZZ] / q[np.arange(64)]).astype(int)
                        diff = zz[0] - preds[ci]
                        preds[ci] = zz[0]
                        cat = 0 if diff == 0 else int(abs(diff)).bit_length()
                        code, ln = dct_t[cat]
                        bits.put(code, ln)
                        if cat:
                            bits.put(diff if diff > 0 else diff + (1 << cat) - 1, cat)
                        run = 0
                        for k in range(1, 64):
                            a = zz[k]
                            if a == 0:
                                run += 1
                                continue
                            while run > 15:
                                code, ln = ac_t[0xF0]
                                bits.put(code, ln)
                                run -= 16
                            cat = int(abs(a)).bit_length()
                            code, ln = ac_t[(run << 4) | cat]
                            bits.put(code, ln)
                            bits.put(a if a > 0 else a + (1 << cat) - 1, cat)
                            run = 0
                        if run:
                            code, ln = ac_t[0x00]
                            bits.put(code, ln)
            out_mcus += 1
    bits.flush()

    def seg(m, data):
        return bytes([0xFF, m]) + struct.pack(">H", len(data) + 2) + data
    jf = b"\xff\xd8" + seg(0xE0, b"JFIF\x00\x01\x01\x00\x00\x01\x00\x01\x00\x00")
    jf += seg(0xDB, bytes([0]) + bytes(int(v) for v in ql))
    if not gray:
        jf += seg(0xDB, bytes([1]) + bytes(int(v) for v in qc))
    nc = len(comps)
    sof = struct.pack(">BHHB", 8, H, W, nc)
    for ci, (sh, sv) in enumerate(samp):
        sof += bytes([ci + 1, (sh << 4) | sv, 0 if ci == 0 else 1])
    jf += seg(0xC0, sof)
    for cls, th, t in [(0, 0, DC_L), (1, 0, AC_L)] + ([] if gray else [(0, 1, DC_C), (1, 1, AC_C)]):
        jf += seg(0xC4, bytes([(cls << 4) | th]) + bytes(t[0]) + bytes(t[1]))
    if restart:
        jf += seg(0xDD, struct.pack(">H", restart))
    sos = bytes([nc]) + b"".join(bytes([ci + 1, 0 if ci == 0 else 0x11]) for ci in range(nc)) + bytes([0, 63, 0])
    jf += seg(0xDA, sos) + bytes(bits.out) + b"\xff\xd9"
    return jf


# ---------------------------------------------------------------- content and fixtures
def content(h, w, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    base = np.stack([(x * 255 // max(w - 1, 1)), (y * 255 // max(h - 1, 1)), ((x // 4 + y // 4) % 2) * 200 + 20], -1)
    noise = rng.integers(-30, 31, size=(h, w, 3))
    return np.clip(base + noise, 0, 255).astype(np.uint8)


def png_fixtures():
    out = {}
    rng = np.random.default_rng(7)
    sizes = [(1, 1), (5, 3), (9, 17), (31, 33), (48, 64)]
    for i, (h, w) in enumerate(sizes):
        rgb = content(h, w, i).astype(int)
        for depth in (1, 2, 4, 8, 16):
            g = rng.integers(0, 1 << depth, size=(h, w, 1))
            out[f"g{depth}_{h}x{w}"] = encode_png(g, 0, depth, interlace=i % 2 == 1, level=i % 10, first_filter=i)
        out[f"rgb8_{h}x{w}"] = encode_png(rgb, 2, 8, level=9, first_filter=i)
        out[f"rgb8i_{h}x{w}"] = encode_png(rgb, 2, 8, interlace=True, level=0, first_filter=i + 1)
        out[f"rgb16_{h}x{w}"] = encode_png(np.minimum(rgb * 257 + rng.integers(0, 200, size=rgb.shape), 65535), 2, 16,
                                           first_filter=i + 2)
        a = rng.integers(0, 256, size=(h, w, 1))
        out[f"ga8_{h}x{w}"] = encode_png(np.concatenate([rgb[..., :1], a], -1), 4, 8, first_filter=i + 3)
        out[f"ga16_{h}x{w}"] = encode_png(np.concatenate([rgb[..., :1], a], -1) * 257, 4, 16, interlace=True)
        out[f"rgba8_{h}x{w}"] = encode_png(np.concatenate([rgb, a], -1), 6, 8, level=1, first_filter=i + 4)
        out[f"rgba16_{h}x{w}"] = encode_png(np.minimum(np.concatenate([rgb, a], -1) * 257 + 3, 65535), 6, 16,
                                            interlace=i % 2 == 0)
        for depth in (1, 2, 4, 8):
            n = 1 << depth
            pal = rng.integers(0, 256, size=(n, 3))
            idx = rng.integers(0, n, size=(h, w, 1))
            out[f"p{depth}_{h}x{w}"] = encode_png(idx, 3, depth, palette=pal, interlace=i % 2 == 0, first_filter=i)
            alpha = bytes(int(v) for v in rng.integers(0, 256, size=max(1, n // 2)))
            out[f"p{depth}t_{h}x{w}"] = encode_png(idx, 3, depth, palette=pal, trns=alpha, first_filter=i + 1)
        # colour keys: the key equals some pixels
        g8 = rng.integers(0, 4, size=(h, w, 1)) * 60
        out[f"g8key_{h}x{w}"] = encode_png(g8, 0, 8, trns=struct.pack(">H", 60))
        g2 = rng.integers(0, 4, size=(h, w, 1))
        out[f"g2key_{h}x{w}"] = encode_png(g2, 0, 2, trns=struct.pack(">H", 2))
        c8 = (rng.integers(0, 2, size=(h, w, 3)) * 100)
        out[f"rgbkey_{h}x{w}"] = encode_png(c8, 2, 8, trns=struct.pack(">HHH", 100, 0, 100))
        c16 = rng.integers(0, 2, size=(h, w, 3)) * 40000
        out[f"rgb16key_{h}x{w}"] = encode_png(c16, 2, 16, trns=struct.pack(">HHH", 40000, 0, 40000))
    return out


def jpeg_fixtures(ref):
    out = {}
    for i, (h, w) in enumerate([(8, 8), (17, 9), (37, 29), (64, 48), (75, 100)]):
        rgb = content(h, w, 100 + i)
        out[f"j444_q75_{h}x{w}"] = encode_jpeg(rgb, 75, (1, 1))
        out[f"j422_q85_{h}x{w}"] = encode_jpeg(rgb, 85, (2, 1), restart=3 if i % 2 else 0)
        out[f"j420_q60_{h}x{w}"] = encode_jpeg(rgb, 60, (2, 2), restart=2 if i % 2 == 0 else 0)
        out[f"j440_q90_{h}x{w}"] = encode_jpeg(rgb, 90, (1, 2))
        out[f"jgray_q80_{h}x{w}"] = encode_jpeg(rgb[..., 1], 80, gray=True, restart=5 if i > 1 else 0)
        for q in (40, 90, 97):   # the reference's own encoder (stb_image_write)
            path = os.path.join(OUT, "_tmp.jpg")
            if not ref.ref_stbi_write_jpg(path.encode(), w, h, 3, rgb.ctypes.data_as(C.c_void_p), q):
                raise RuntimeError("stbi_write_jpg failed")
            with open(path, "rb") as f:
                out[f"jstb_q{q}_{h}x{w}"] = f.read()
            os.remove(path)
    return out


def stb_decode(ref, data):
    buf = np.frombuffer(data, dtype=np.uint8)
    w, h, c = C.c_int(), C.c_int(), C.c_int()
    if ref.ref_stbi_decode_rgba(buf.ctypes.data_as(C.c_void_p), len(buf), None, C.c_longlong(0), C.byref(w),
                                C.byref(h), C.byref(c)) != 0:
        raise RuntimeError("stb_image failed: " + ref.ref_stbi_failure().decode())
    out = np.empty((h.value, w.value, 4), dtype=np.uint8)
    ref.ref_stbi_decode_rgba(buf.ctypes.data_as(C.c_void_p), len(buf), out.ctypes.data_as(C.c_void_p),
                             C.c_longlong(out.size), C.byref(w), C.byref(h), C.byref(c))
    return out, c.value


def main():
    ref = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libstbref.so"))
    ref.ref_stbi_failure.restype = C.c_char_p
    os.makedirs(OUT, exist_ok=True)
    files = {}
    files.update(png_fixtures())
    files.update(jpeg_fixtures(ref))
    expected, comps, blobs = {}, {}, {}
    for name, data in sorted(files.items()):
        px, c = stb_decode(ref, data)
        expected[name] = px
        comps[name] = c
        blobs[name] = np.frombuffer(data, dtype=np.uint8)
    np.savez_compressed(os.path.join(OUT, "fixtures.npz"), **{"file_" + k: v for k, v in blobs.items()},
                        **{"rgba_" + k: v for k, v in expected.items()},
                        comps=np.array([comps[k] for k in sorted(files)]), names=np.array(sorted(files)))
    print(len(files), "fixtures,", sum(len(v) for v in files.values()), "bytes of files")


if __name__ == "__main__":
    sys.exit(main())
