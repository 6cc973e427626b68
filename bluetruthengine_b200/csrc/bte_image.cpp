// bte_image.cpp -- PNG and JPEG decoding to 8-bit RGBA for material textures.
//
// The reference decodes albedo textures with stb_image, stbi_load(path, &w,
// &h, &channels, 4) (src/main.cpp:407-470): the file's samples expanded to
// 8-bit RGBA, rows top to bottom.  This decoder covers the formats scene
// assets use:
//   PNG  (ISO/IEC 15948; zlib RFC 1950 / DEFLATE RFC 1951): every colour type
//        and bit depth, the five scanline filters, Adam7 interlacing, tRNS
//        (palette alpha, grey / RGB colour keys).  Samples below 8 bits are
//        scaled to 0-255 (x255, x85, x17 for 1, 2, 4 bits), 16-bit samples
//        reduced to their high byte, as stb_image does.  Lossless: the same
//        bytes as stb_image.
//   JPEG (ITU-T T.81, JFIF / T.871): sequential Huffman (SOF0, SOF1), 8-bit,
//        1 or 3 components, any sampling factors, restart intervals, Adobe
//        APP14 colour-transform flag.  The inverse DCT is the integer
//        Loeffler-Ligtenberg-Moschytz algorithm in two passes; 2x chroma is
//        upsampled with the triangle filter (3/4, 1/4 weights); YCbCr -> RGB
//        uses the JFIF coefficients.  T.81 does not fix an IDCT to the bit, so
//        the fixed-point details follow the reference's decoder, so that
//        textures decode to the same bytes: 12-bit constants rounded as
//        (int)(c * 4096 + 0.5) (truncating towards zero for the negative
//        ones), 2 extra bits kept between passes, dequantised coefficients
//        held in 16 bits, 12-bit colour coefficients with the Cb term of green
//        kept to 16 fractional bits, its edge rules for 2x upsampling, and its
//        rule for when three components are RGB rather than YCbCr.
//   Progressive and arithmetic-coded JPEG, 12-bit JPEG, CMYK and the other
//   stb_image formats are reported as unsupported.
#include "bte_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

namespace bte {

namespace {

struct ImageError {
    std::string msg;
};
[[noreturn]] void bad(const std::string& m) { throw ImageError{m}; }

// ================================================================ DEFLATE (RFC 1951)
struct BitReaderLsb {
    const uint8_t* p;
    size_t n, pos = 0;
    uint32_t buf = 0;
    int cnt = 0;
    uint32_t bits(int k)
    {
        while (cnt < k) {
            if (pos >= n) bad("PNG: compressed data ends early");
            buf |= static_cast<uint32_t>(p[pos++]) << cnt;
            cnt += 8;
        }
        const uint32_t v = buf & ((1u << k) - 1u);
        buf = k == 32 ? 0 : buf >> k;
        cnt -= k;
        return v;
    }
};

// Canonical Huffman code: codes per length and the symbols in code order.
struct Canon {
    uint16_t count[16];
    uint16_t symbol[320];
};

// Returns the number of unused codes (0 for a complete code); throws on an over-subscribed one.
int buildCanon(Canon& h, const uint8_t* lengths, int n)
{
    std::memset(h.count, 0, sizeof(h.count));
    for (int i = 0; i < n; ++i) h.count[lengths[i]]++;
    if (h.count[0] == n) return 0;
    int left = 1;
    for (int len = 1; len < 16; ++len) {
        left <<= 1;
        left -= h.count[len];
        if (left < 0) bad("PNG: over-subscribed Huffman code");
    }
    int offs[16];
    offs[1] = 0;
    for (int len = 1; len < 15; ++len) offs[len + 1] = offs[len] + h.count[len];
    for (int i = 0; i < n; ++i)
        if (lengths[i]) h.symbol[offs[lengths[i]]++] = static_cast<uint16_t>(i);
    return left;
}

// DEFLATE packs Huffman codes starting from their most significant bit.
int decodeCanon(BitReaderLsb& in, const Canon& h)
{
    int code = 0, first = 0, index = 0;
    for (int len = 1; len < 16; ++len) {
        code |= static_cast<int>(in.bits(1));
        const int c = h.count[len];
        if (code - c < first) return h.symbol[index + (code - first)];
        index += c;
        first += c;
        first <<= 1;
        code <<= 1;
    }
    bad("PNG: invalid Huffman code");
}

const uint16_t kLenBase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31, 35, 43, 51, 59, 67, 83, 99,
                               115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129, 193, 257, 385, 513, 769, 1025, 1537,
                                2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12,
                                13, 13};

void inflateCodes(BitReaderLsb& in, const Canon& lit, const Canon& dist, std::vector<uint8_t>& out, size_t limit)
{
    while (true) {
        const int sym = decodeCanon(in, lit);
        if (sym < 256) {
            if (out.size() >= limit) bad("PNG: more image data than the header allows");
            out.push_back(static_cast<uint8_t>(sym));
        } else if (sym == 256) {
            return;
        } else {
            const int li = sym - 257;
            if (li >= 29) bad("PNG: invalid length code");
            const size_t len = kLenBase[li] + in.bits(kLenExtra[li]);
            const int di = decodeCanon(in, dist);
            if (di >= 30) bad("PNG: invalid distance code");
            const size_t d = kDistBase[di] + in.bits(kDistExtra[di]);
            if (d > out.size()) bad("PNG: distance before the start of the data");
            if (out.size() + len > limit) bad("PNG: more image data than the header allows");
            const size_t from = out.size() - d;
            for (size_t k = 0; k < len; ++k) out.push_back(out[from + k]);
        }
    }
}

// zlib stream -> bytes (at most `limit`)
std::vector<uint8_t> zlibInflate(const uint8_t* p, size_t n, size_t limit)
{
    if (n < 2) bad("PNG: empty zlib stream");
    const int cmf = p[0], flg = p[1];
    if ((cmf * 256 + flg) % 31 != 0 || (cmf & 15) != 8) bad("PNG: bad zlib header");
    if (flg & 32) bad("PNG: preset dictionary not allowed");
    BitReaderLsb in{p + 2, n - 2};
    std::vector<uint8_t> out;
    out.reserve(limit);
    int final = 0;
    do {
        final = static_cast<int>(in.bits(1));
        const int type = static_cast<int>(in.bits(2));
        if (type == 0) {   // stored
            in.bits(in.cnt & 7);
            const uint32_t len = in.bits(16), nlen = in.bits(16);
            if ((len ^ 0xffffu) != nlen) bad("PNG: stored block length check failed");
            if (out.size() + len > limit) bad("PNG: more image data than the header allows");
            for (uint32_t k = 0; k < len; ++k) out.push_back(static_cast<uint8_t>(in.bits(8)));
        } else if (type == 1) {   // fixed codes
            struct Fixed {
                Canon lit, dist;
                Fixed()
                {
                    uint8_t l[288], d[30];
                    for (int i = 0; i < 144; ++i) l[i] = 8;
                    for (int i = 144; i < 256; ++i) l[i] = 9;
                    for (int i = 256; i < 280; ++i) l[i] = 7;
                    for (int i = 280; i < 288; ++i) l[i] = 8;
                    for (int i = 0; i < 30; ++i) d[i] = 5;
                    buildCanon(lit, l, 288);
                    buildCanon(dist, d, 30);
                }
            };
            static const Fixed fixedCodes;
            inflateCodes(in, fixedCodes.lit, fixedCodes.dist, out, limit);
        } else if (type == 2) {   // dynamic codes
            const int nlen = static_cast<int>(in.bits(5)) + 257, ndist = static_cast<int>(in.bits(5)) + 1,
                      ncode = static_cast<int>(in.bits(4)) + 4;
            if (nlen > 286 || ndist > 30) bad("PNG: bad dynamic block counts");
            static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
            uint8_t cl[19] = {};
            for (int i = 0; i < ncode; ++i) cl[order[i]] = static_cast<uint8_t>(in.bits(3));
            Canon clc;
            if (buildCanon(clc, cl, 19) != 0) bad("PNG: incomplete code-length code");
            uint8_t lens[320] = {};
            int idx = 0;
            while (idx < nlen + ndist) {
                const int sym = decodeCanon(in, clc);
                if (sym < 16) {
                    lens[idx++] = static_cast<uint8_t>(sym);
                } else {
                    int rep = 0;
                    uint8_t val = 0;
                    if (sym == 16) {
                        if (idx == 0) bad("PNG: repeat with no previous length");
                        val = lens[idx - 1];
                        rep = 3 + static_cast<int>(in.bits(2));
                    } else if (sym == 17) {
                        rep = 3 + static_cast<int>(in.bits(3));
                    } else {
                        rep = 11 + static_cast<int>(in.bits(7));
                    }
                    if (idx + rep > nlen + ndist) bad("PNG: too many code lengths");
                    while (rep--) lens[idx++] = val;
                }
            }
            if (lens[256] == 0) bad("PNG: no end-of-block code");
            Canon lit, dist;
            const int litLeft = buildCanon(lit, lens, nlen);
            if (litLeft > 0 && nlen - lit.count[0] != 1) bad("PNG: incomplete literal/length code");
            const int distLeft = buildCanon(dist, lens + nlen, ndist);
            if (distLeft > 0 && ndist - dist.count[0] != 1) bad("PNG: incomplete distance code");
            inflateCodes(in, lit, dist, out, limit);
        } else {
            bad("PNG: invalid block type");
        }
    } while (!final);
    return out;
}

// ================================================================ PNG
uint32_t be32(const uint8_t* p)
{
    return (static_cast<uint32_t>(p[0]) << 24) | (static_cast<uint32_t>(p[1]) << 16) |
           (static_cast<uint32_t>(p[2]) << 8) | p[3];
}

int paeth(int a, int b, int c)
{
    const int p = a + b - c;
    const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    if (pb <= pc) return b;
    return c;
}

struct PngInfo {
    uint32_t w = 0, h = 0;
    int depth = 0, color = 0, interlace = 0, channels = 0;
    uint8_t palette[256][4];
    int paletteSize = 0;
    bool hasKey = false;
    uint16_t key[3] = {0, 0, 0};
};

// Unfilter the `rows` scanlines of `rowBytes` bytes (after their filter byte) at `src` in place.
void unfilter(uint8_t* src, uint32_t rows, size_t rowBytes, int bpp)
{
    std::vector<uint8_t> zero(rowBytes, 0);
    const uint8_t* prior = zero.data();
    for (uint32_t y = 0; y < rows; ++y) {
        uint8_t* f = src + y * (rowBytes + 1);
        const int type = f[0];
        uint8_t* x = f + 1;
        switch (type) {
        case 0: break;
        case 1: for (size_t i = bpp; i < rowBytes; ++i) x[i] = static_cast<uint8_t>(x[i] + x[i - bpp]); break;
        case 2: for (size_t i = 0; i < rowBytes; ++i) x[i] = static_cast<uint8_t>(x[i] + prior[i]); break;
        case 3:
            for (size_t i = 0; i < rowBytes; ++i)
                x[i] = static_cast<uint8_t>(x[i] + ((i >= static_cast<size_t>(bpp) ? x[i - bpp] : 0) + prior[i]) / 2);
            break;
        case 4:
            for (size_t i = 0; i < rowBytes; ++i) {
                const int a = i >= static_cast<size_t>(bpp) ? x[i - bpp] : 0;
                const int c = i >= static_cast<size_t>(bpp) ? prior[i - bpp] : 0;
                x[i] = static_cast<uint8_t>(x[i] + paeth(a, prior[i], c));
            }
            break;
        default: bad("PNG: invalid filter type");
        }
        prior = x;
    }
}

// sample k (0-based, across all channels of the row) of an unfiltered row
uint16_t sampleAt(const uint8_t* row, int depth, size_t k)
{
    if (depth == 8) return row[k];
    if (depth == 16) return static_cast<uint16_t>((row[2 * k] << 8) | row[2 * k + 1]);
    const size_t bit = k * depth;
    const int shift = 8 - depth - static_cast<int>(bit & 7);
    return static_cast<uint16_t>((row[bit >> 3] >> shift) & ((1 << depth) - 1));
}

void pngPixel(const PngInfo& I, const uint8_t* row, uint32_t x, uint8_t* out)
{
    const int ch = I.channels;
    uint16_t s[4];
    for (int c = 0; c < ch; ++c) s[c] = sampleAt(row, I.depth, static_cast<size_t>(x) * ch + c);
    auto to8 = [&](uint16_t v) -> uint8_t {
        if (I.depth == 16) return static_cast<uint8_t>(v >> 8);
        if (I.depth == 8) return static_cast<uint8_t>(v);
        const int scale = I.depth == 1 ? 255 : I.depth == 2 ? 85 : 17;
        return static_cast<uint8_t>(v * scale);
    };
    switch (I.color) {
    case 3: {
        const uint8_t* p = I.palette[s[0]];
        out[0] = p[0]; out[1] = p[1]; out[2] = p[2]; out[3] = p[3];
        return;
    }
    case 0:
        out[0] = out[1] = out[2] = to8(s[0]);
        out[3] = (I.hasKey && s[0] == I.key[0]) ? 0 : 255;
        return;
    case 2:
        out[0] = to8(s[0]); out[1] = to8(s[1]); out[2] = to8(s[2]);
        out[3] = (I.hasKey && s[0] == I.key[0] && s[1] == I.key[1] && s[2] == I.key[2]) ? 0 : 255;
        return;
    case 4:
        out[0] = out[1] = out[2] = to8(s[0]);
        out[3] = to8(s[1]);
        return;
    default:
        out[0] = to8(s[0]); out[1] = to8(s[1]); out[2] = to8(s[2]); out[3] = to8(s[3]);
        return;
    }
}

void decodePng(const uint8_t* d, size_t n, std::vector<uint8_t>& rgba, int& w, int& h, int& channelsInFile,
               std::vector<uint8_t>* rgba16 = nullptr)
{
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (n < 8 || std::memcmp(d, sig, 8) != 0) bad("PNG: bad signature");
    PngInfo I;
    for (auto& p : I.palette) { p[0] = p[1] = p[2] = 0; p[3] = 255; }
    std::vector<uint8_t> idat;
    bool haveHeader = false, end = false;
    size_t pos = 8;
    while (!end) {
        if (pos + 8 > n) bad("PNG: truncated chunk");
        const uint32_t len = be32(d + pos);
        const uint8_t* type = d + pos + 4;
        if (len > n - pos - 8 || n - pos - 8 - len < 4) bad("PNG: truncated chunk");
        const uint8_t* c = d + pos + 8;
        const bool first = pos == 8;
        if (std::memcmp(type, "IHDR", 4) == 0) {
            if (!first || len != 13) bad("PNG: bad IHDR");
            I.w = be32(c); I.h = be32(c + 4);
            I.depth = c[8]; I.color = c[9];
            if (c[10] != 0 || c[11] != 0) bad("PNG: unknown compression or filter method");
            I.interlace = c[12];
            if (I.interlace > 1) bad("PNG: unknown interlace method");
            if (I.w == 0 || I.h == 0 || I.w > (1u << 24) || I.h > (1u << 24)) bad("PNG: bad image size");
            const int dp = I.depth;
            bool ok = false;
            switch (I.color) {
            case 0: ok = dp == 1 || dp == 2 || dp == 4 || dp == 8 || dp == 16; I.channels = 1; break;
            case 2: ok = dp == 8 || dp == 16; I.channels = 3; break;
            case 3: ok = dp == 1 || dp == 2 || dp == 4 || dp == 8; I.channels = 1; break;
            case 4: ok = dp == 8 || dp == 16; I.channels = 2; break;
            case 6: ok = dp == 8 || dp == 16; I.channels = 4; break;
            default: break;
            }
            if (!ok) bad("PNG: bad colour type / bit depth");
            haveHeader = true;
        } else if (!haveHeader) {
            bad("PNG: first chunk is not IHDR");
        } else if (std::memcmp(type, "PLTE", 4) == 0) {
            if (len % 3 != 0 || len / 3 > 256 || len == 0) bad("PNG: bad PLTE");
            I.paletteSize = static_cast<int>(len / 3);
            for (int i = 0; i < I.paletteSize; ++i) {
                I.palette[i][0] = c[3 * i]; I.palette[i][1] = c[3 * i + 1]; I.palette[i][2] = c[3 * i + 2];
            }
        } else if (std::memcmp(type, "tRNS", 4) == 0) {
            if (!idat.empty()) bad("PNG: tRNS after IDAT");
            if (I.color == 3) {
                if (I.paletteSize == 0) bad("PNG: tRNS before PLTE");
                if (static_cast<int>(len) > I.paletteSize) bad("PNG: bad tRNS length");
                for (uint32_t i = 0; i < len; ++i) I.palette[i][3] = c[i];
            } else if (I.color == 0 || I.color == 2) {
                if (len != static_cast<uint32_t>(2 * I.channels)) bad("PNG: bad tRNS length");
                I.hasKey = true;
                for (int k = 0; k < I.channels; ++k) {
                    const uint16_t v = static_cast<uint16_t>((c[2 * k] << 8) | c[2 * k + 1]);
                    // a key below 16 bits is compared in the sample's own range (its low byte, as stb_image)
                    I.key[k] = I.depth == 16 ? v : static_cast<uint16_t>(v & 0xffu);
                }
            } else {
                bad("PNG: tRNS with an alpha channel");
            }
        } else if (std::memcmp(type, "IDAT", 4) == 0) {
            idat.insert(idat.end(), c, c + len);
        } else if (std::memcmp(type, "IEND", 4) == 0) {
            end = true;
        } else if ((type[0] & 32) == 0) {
            bad("PNG: unknown critical chunk");
        }
        pos += 12 + static_cast<size_t>(len);
    }
    if (I.color == 3 && I.paletteSize == 0) bad("PNG: palette image without PLTE");
    if (idat.empty()) bad("PNG: no image data");
    const int bitsPerPixel = I.channels * I.depth;
    const int bpp = bitsPerPixel >= 8 ? bitsPerPixel / 8 : 1;
    auto rowBytes = [&](uint32_t width) { return (static_cast<size_t>(width) * bitsPerPixel + 7) / 8; };
    static const int a7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4}, {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
    size_t total = 0;
    if (I.interlace == 0) {
        total = static_cast<size_t>(I.h) * (rowBytes(I.w) + 1);
    } else {
        for (const auto& p : a7) {
            const uint32_t pw = (I.w - p[0] + p[2] - 1) / p[2], ph = (I.h - p[1] + p[3] - 1) / p[3];
            if (I.w > static_cast<uint32_t>(p[0]) && I.h > static_cast<uint32_t>(p[1]) && pw && ph)
                total += static_cast<size_t>(ph) * (rowBytes(pw) + 1);
        }
    }
    std::vector<uint8_t> raw = zlibInflate(idat.data(), idat.size(), total);
    if (raw.size() < total) bad("PNG: not enough image data");
    w = static_cast<int>(I.w);
    h = static_cast<int>(I.h);
    channelsInFile = I.channels + (I.hasKey ? 1 : 0);   // a colour key adds an alpha channel
    if (I.color == 3) {   // palette: 3 channels, 4 when tRNS gave any entry alpha
        bool alpha = false;
        for (int i = 0; i < I.paletteSize; ++i) alpha = alpha || I.palette[i][3] != 255;
        channelsInFile = alpha ? 4 : 3;
    }
    if (rgba16) {   // 16-bit samples, 4 channels (alpha 65535 where the file has none, 0 under a colour key)
        rgba16->clear();
        if (I.depth != 16) return;
        rgba16->assign(static_cast<size_t>(w) * h * 8, 0);
        auto put16 = [&](const uint8_t* row, uint32_t x, size_t o) {
            uint16_t s[4];
            for (int c = 0; c < I.channels; ++c) s[c] = sampleAt(row, 16, static_cast<size_t>(x) * I.channels + c);
            uint16_t px[4];
            if (I.color == 0) { px[0] = px[1] = px[2] = s[0]; px[3] = (I.hasKey && s[0] == I.key[0]) ? 0 : 65535; }
            else if (I.color == 2) {
                px[0] = s[0]; px[1] = s[1]; px[2] = s[2];
                px[3] = (I.hasKey && s[0] == I.key[0] && s[1] == I.key[1] && s[2] == I.key[2]) ? 0 : 65535;
            } else if (I.color == 4) { px[0] = px[1] = px[2] = s[0]; px[3] = s[1]; }
            else { px[0] = s[0]; px[1] = s[1]; px[2] = s[2]; px[3] = s[3]; }
            for (int c = 0; c < 4; ++c) {
                (*rgba16)[o + 2 * c] = static_cast<uint8_t>(px[c] & 0xff);
                (*rgba16)[o + 2 * c + 1] = static_cast<uint8_t>(px[c] >> 8);
            }
        };
        if (I.interlace == 0) {
            const size_t rb = rowBytes(I.w);
            unfilter(raw.data(), I.h, rb, bpp);
            for (uint32_t y = 0; y < I.h; ++y)
                for (uint32_t x = 0; x < I.w; ++x) put16(raw.data() + y * (rb + 1) + 1, x, (static_cast<size_t>(y) * I.w + x) * 8);
        } else {
            size_t off = 0;
            for (const auto& p : a7) {
                if (I.w <= static_cast<uint32_t>(p[0]) || I.h <= static_cast<uint32_t>(p[1])) continue;
                const uint32_t pw = (I.w - p[0] + p[2] - 1) / p[2], ph = (I.h - p[1] + p[3] - 1) / p[3];
                if (!pw || !ph) continue;
                const size_t rb = rowBytes(pw);
                unfilter(raw.data() + off, ph, rb, bpp);
                for (uint32_t j = 0; j < ph; ++j)
                    for (uint32_t i = 0; i < pw; ++i)
                        put16(raw.data() + off + j * (rb + 1) + 1, i,
                              (static_cast<size_t>(p[1] + j * p[3]) * I.w + p[0] + i * p[2]) * 8);
                off += static_cast<size_t>(ph) * (rb + 1);
            }
        }
        return;
    }
    rgba.assign(static_cast<size_t>(w) * h * 4, 0);
    if (I.interlace == 0) {
        const size_t rb = rowBytes(I.w);
        unfilter(raw.data(), I.h, rb, bpp);
        for (uint32_t y = 0; y < I.h; ++y) {
            const uint8_t* row = raw.data() + y * (rb + 1) + 1;
            for (uint32_t x = 0; x < I.w; ++x) pngPixel(I, row, x, &rgba[(static_cast<size_t>(y) * I.w + x) * 4]);
        }
    } else {
        size_t off = 0;
        for (const auto& p : a7) {
            if (I.w <= static_cast<uint32_t>(p[0]) || I.h <= static_cast<uint32_t>(p[1])) continue;
            const uint32_t pw = (I.w - p[0] + p[2] - 1) / p[2], ph = (I.h - p[1] + p[3] - 1) / p[3];
            if (!pw || !ph) continue;
            const size_t rb = rowBytes(pw);
            unfilter(raw.data() + off, ph, rb, bpp);
            for (uint32_t j = 0; j < ph; ++j) {
                const uint8_t* row = raw.data() + off + j * (rb + 1) + 1;
                const uint32_t y = p[1] + j * p[3];
                for (uint32_t i = 0; i < pw; ++i) {
                    const uint32_t x = p[0] + i * p[2];
                    pngPixel(I, row, i, &rgba[(static_cast<size_t>(y) * I.w + x) * 4]);
                }
            }
            off += static_cast<size_t>(ph) * (rb + 1);
        }
    }
}

// ================================================================ JPEG (sequential Huffman)
const uint8_t kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
                             41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
                             30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// Huffman table (T.81 Annex C / F.2.2.3): maxcode / valptr / mincode per code length.
struct JHuff {
    int mincode[17], maxcode[18], valptr[17];
    uint8_t vals[256];
    bool present = false;
};

void buildJHuff(JHuff& t, const uint8_t* counts, const uint8_t* vals, int nvals)
{
    std::memcpy(t.vals, vals, static_cast<size_t>(nvals));
    int code = 0, k = 0;
    for (int len = 1; len <= 16; ++len) {
        t.valptr[len] = k;
        t.mincode[len] = code;
        code += counts[len - 1];
        k += counts[len - 1];
        t.maxcode[len] = counts[len - 1] ? code - 1 : -1;
        if (code > (1 << len)) bad("JPEG: bad Huffman table");
        code <<= 1;
    }
    t.maxcode[17] = 0x7fffffff;
    t.present = true;
}

struct JComp {
    int id = 0, H = 1, V = 1, tq = 0, td = 0, ta = 0;
    int bw = 0, bh = 0;          // blocks across / down the component's padded plane
    int pred = 0;
    std::vector<uint8_t> plane;  // bw*8 x bh*8 samples
};

struct JpegDecoder {
    const uint8_t* d;
    size_t n, pos = 0;
    uint16_t q[4][64];
    bool qPresent[4] = {false, false, false, false};
    JHuff dc[4], ac[4];
    std::vector<JComp> comps;
    int width = 0, height = 0, hmax = 1, vmax = 1, mcux = 0, mcuy = 0;
    int restartInterval = 0;
    int adobeTransform = -1;   // APP14: -1 absent, else the transform flag
    bool jfif = false;         // APP0 "JFIF" present
    bool frame = false;
    // entropy-coded data reader (MSB first, 0xFF00 stuffing, stops at a marker)
    uint32_t bitBuf = 0;
    int bitCnt = 0;
    bool hitMarker = false;

    uint8_t byte()
    {
        if (pos >= n) bad("JPEG: truncated file");
        return d[pos++];
    }
    int u16()
    {
        const int hi = byte();
        return (hi << 8) | byte();
    }
    void fill()
    {
        while (bitCnt <= 24) {
            uint32_t b = 0;
            if (!hitMarker && pos < n) {
                b = d[pos];
                if (b == 0xFF) {
                    const uint8_t nx = pos + 1 < n ? d[pos + 1] : 0xD9;
                    if (nx == 0x00) {
                        pos += 2;
                    } else {
                        hitMarker = true;
                        b = 0;
                    }
                } else {
                    ++pos;
                }
            }
            bitBuf |= b << (24 - bitCnt);
            bitCnt += 8;
        }
    }
    int bit()
    {
        if (bitCnt < 1) fill();
        const int v = static_cast<int>(bitBuf >> 31);
        bitBuf <<= 1;
        --bitCnt;
        return v;
    }
    int receive(int s)
    {
        if (s == 0) return 0;
        if (bitCnt < s) fill();
        const int v = static_cast<int>(bitBuf >> (32 - s));
        bitBuf <<= s;
        bitCnt -= s;
        return v;
    }
    static int extend(int v, int s) { return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v; }
    int decode(const JHuff& t)
    {
        int code = bit();
        int len = 1;
        while (code > t.maxcode[len]) {
            code = (code << 1) | bit();
            if (++len > 16) bad("JPEG: invalid Huffman code");
        }
        return t.vals[t.valptr[len] + code - t.mincode[len]];
    }
    void resetBits()
    {
        bitBuf = 0;
        bitCnt = 0;
        hitMarker = false;
    }

    void decodeBlock(JComp& c, int* coef)
    {
        std::memset(coef, 0, 64 * sizeof(int));
        const JHuff& hd = dc[c.td];
        const JHuff& ha = ac[c.ta];
        const uint16_t* qt = q[c.tq];
        const int t = decode(hd);
        if (t > 11) bad("JPEG: bad DC magnitude");
        c.pred += t ? extend(receive(t), t) : 0;
        coef[0] = static_cast<int16_t>(c.pred * qt[0]);   // dequantised coefficients are 16-bit
        for (int k = 1; k < 64;) {
            const int rs = decode(ha);
            const int r = rs >> 4, s = rs & 15;
            if (s == 0) {
                if (r != 15) break;
                k += 16;
                continue;
            }
            k += r;
            if (k > 63) bad("JPEG: coefficient index out of range");
            coef[kZigzag[k]] = static_cast<int16_t>(extend(receive(s), s) * qt[k]);
            ++k;
        }
    }

    // ---- inverse DCT: Loeffler, Ligtenberg, Moschytz (ICASSP 1989), integer two-pass form.  The constants
    // are sqrt(2) times sums of c_k = cos(k pi / 16) in 12-bit fixed point, rounded as (int)(v * 4096 + 0.5).
    static int fix12(double v) { return static_cast<int>(v * 4096.0 + 0.5); }
    struct Consts {
        int c0541, c1847n, c0765, c1175, c0298, c2053, c3072, c1501, c0899n, c2562n, c1961n, c0390n;
        Consts()
        {
            const double pi = 3.14159265358979323846, r2 = std::sqrt(2.0);
            double c[8];
            for (int k = 0; k < 8; ++k) c[k] = std::cos(k * pi / 16.0);
            c0541 = fix12(r2 * c[6]);
            c1847n = fix12(-r2 * (c[2] + c[6]));
            c0765 = fix12(r2 * (c[2] - c[6]));
            c1175 = fix12(r2 * c[3]);
            c0298 = fix12(r2 * (-c[1] + c[3] + c[5] - c[7]));
            c2053 = fix12(r2 * (c[1] + c[3] - c[5] + c[7]));
            c3072 = fix12(r2 * (c[1] + c[3] + c[5] - c[7]));
            c1501 = fix12(r2 * (c[1] + c[3] - c[5] - c[7]));
            c0899n = fix12(-r2 * (c[3] - c[7]));
            c2562n = fix12(-r2 * (c[1] + c[3]));
            c1961n = fix12(-r2 * (c[3] + c[5]));
            c0390n = fix12(-r2 * (c[3] - c[5]));
        }
    };

    // one 1-D pass over 8 values at stride `st` of `in`, results (scaled by 2^12) into o[8]
    static void idct1d(const Consts& K, const int* in, int st, long long* o)
    {
        // even part
        long long p2 = in[2 * st], p3 = in[6 * st];
        const long long p1 = (p2 + p3) * K.c0541;
        const long long t2 = p1 + p3 * K.c1847n, t3 = p1 + p2 * K.c0765;
        p2 = in[0];
        p3 = in[4 * st];
        const long long t0 = (p2 + p3) * 4096, t1 = (p2 - p3) * 4096;
        const long long x0 = t0 + t3, x3 = t0 - t3, x1 = t1 + t2, x2 = t1 - t2;
        // odd part
        long long a0 = in[7 * st], a1 = in[5 * st], a2 = in[3 * st], a3 = in[st];
        const long long q3 = a0 + a2, q4 = a1 + a3, q1 = a0 + a3, q2 = a1 + a2;
        const long long q5 = (q3 + q4) * K.c1175;
        a0 *= K.c0298; a1 *= K.c2053; a2 *= K.c3072; a3 *= K.c1501;
        const long long r1 = q5 + q1 * K.c0899n, r2 = q5 + q2 * K.c2562n, r3 = q3 * K.c1961n, r4 = q4 * K.c0390n;
        a3 += r1 + r4; a2 += r2 + r3; a1 += r2 + r4; a0 += r1 + r3;
        o[0] = x0 + a3; o[7] = x0 - a3;
        o[1] = x1 + a2; o[6] = x1 - a2;
        o[2] = x2 + a1; o[5] = x2 - a1;
        o[3] = x3 + a0; o[4] = x3 - a0;
    }

    static void idct(const int* coef, uint8_t* out, int stride)
    {
        static const Consts K;
        int ws[64];
        long long o[8];
        for (int c = 0; c < 8; ++c) {   // columns: keep 2 extra bits (scale 2^12 -> 2^2, rounded)
            const int* in = coef + c;
            if (!in[8] && !in[16] && !in[24] && !in[32] && !in[40] && !in[48] && !in[56]) {
                for (int r = 0; r < 8; ++r) ws[r * 8 + c] = in[0] * 4;
                continue;
            }
            idct1d(K, in, 8, o);
            for (int r = 0; r < 8; ++r) ws[r * 8 + c] = static_cast<int>((o[r] + 512) >> 10);
        }
        for (int r = 0; r < 8; ++r) {   // rows: remove 2^12 * 2^2 * 8 (= 2^17), rounded, and add the level shift
            idct1d(K, ws + r * 8, 1, o);
            for (int c = 0; c < 8; ++c) {
                const long long v = (o[c] + 65536 + (128LL << 17)) >> 17;
                out[r * stride + c] = static_cast<uint8_t>(v < 0 ? 0 : (v > 255 ? 255 : v));
            }
        }
    }

    void parseSof()
    {
        const int len = u16();
        const int precision = byte();
        if (precision != 8) bad("JPEG: only 8-bit samples are supported");
        height = u16();
        width = u16();
        const int nc = byte();
        if (height == 0) bad("JPEG: height from a DNL marker is not supported");
        if (width == 0) bad("JPEG: zero width");
        if (nc != 1 && nc != 3) bad("JPEG: only 1 or 3 components are supported");
        if (len != 8 + 3 * nc) bad("JPEG: bad SOF length");
        comps.assign(static_cast<size_t>(nc), JComp{});
        for (auto& c : comps) {
            c.id = byte();
            const int hv = byte();
            c.H = hv >> 4;
            c.V = hv & 15;
            c.tq = byte();
            if (c.H < 1 || c.H > 4 || c.V < 1 || c.V > 4) bad("JPEG: bad sampling factors");
            if (c.tq > 3) bad("JPEG: bad quantisation table index");
            hmax = std::max(hmax, c.H);
            vmax = std::max(vmax, c.V);
        }
        mcux = (width + 8 * hmax - 1) / (8 * hmax);
        mcuy = (height + 8 * vmax - 1) / (8 * vmax);
        for (auto& c : comps) {
            c.bw = mcux * c.H;
            c.bh = mcuy * c.V;
            c.plane.assign(static_cast<size_t>(c.bw) * c.bh * 64, 0);
        }
        frame = true;
    }

    void parseDht()
    {
        int len = u16() - 2;
        while (len > 0) {
            const int tc = byte();
            const int cls = tc >> 4, th = tc & 15;
            if (cls > 1 || th > 3) bad("JPEG: bad Huffman table id");
            uint8_t counts[16];
            int total = 0;
            for (int i = 0; i < 16; ++i) { counts[i] = byte(); total += counts[i]; }
            if (total > 256) bad("JPEG: bad Huffman table");
            uint8_t vals[256];
            for (int i = 0; i < total; ++i) vals[i] = byte();
            buildJHuff(cls == 0 ? dc[th] : ac[th], counts, vals, total);
            len -= 17 + total;
        }
        if (len != 0) bad("JPEG: bad DHT length");
    }

    void parseDqt()
    {
        int len = u16() - 2;
        while (len > 0) {
            const int pq = byte();
            const int p = pq >> 4, t = pq & 15;
            if (p > 1 || t > 3) bad("JPEG: bad quantisation table");
            for (int i = 0; i < 64; ++i) q[t][i] = static_cast<uint16_t>(p ? u16() : byte());
            qPresent[t] = true;
            len -= 65 + 64 * p;
        }
        if (len != 0) bad("JPEG: bad DQT length");
    }

    void parseSos()
    {
        if (!frame) bad("JPEG: scan before frame header");
        const int len = u16();
        const int ns = byte();
        if (ns < 1 || ns > static_cast<int>(comps.size()) || len != 6 + 2 * ns) bad("JPEG: bad SOS");
        std::vector<JComp*> sc;
        for (int i = 0; i < ns; ++i) {
            const int id = byte(), t = byte();
            JComp* c = nullptr;
            for (auto& x : comps) if (x.id == id) c = &x;
            if (!c) bad("JPEG: scan names an unknown component");
            c->td = t >> 4;
            c->ta = t & 15;
            if (c->td > 3 || c->ta > 3 || !dc[c->td].present || !ac[c->ta].present) bad("JPEG: missing Huffman table");
            if (!qPresent[c->tq]) bad("JPEG: missing quantisation table");
            sc.push_back(c);
        }
        const int ss = byte(), se = byte(), a = byte();
        if (ss != 0 || se != 63 || a != 0) bad("JPEG: not a sequential scan");
        for (auto* c : sc) c->pred = 0;
        resetBits();
        int coef[64];
        int untilRestart = restartInterval;
        int expectRst = 0;
        auto restart = [&]() {
            // align to the marker: skip to the RSTn after the entropy-coded segment
            resetBits();
            while (pos + 1 < n && !(d[pos] == 0xFF && d[pos + 1] >= 0xD0 && d[pos + 1] <= 0xD7)) ++pos;
            if (pos + 1 >= n) bad("JPEG: missing restart marker");
            if (d[pos + 1] != 0xD0 + expectRst) bad("JPEG: restart markers out of order");
            pos += 2;
            expectRst = (expectRst + 1) & 7;
            for (auto* c : sc) c->pred = 0;
            untilRestart = restartInterval;
        };
        if (ns == 1) {   // non-interleaved: the component's own blocks, without the MCU padding
            JComp& c = *sc[0];
            const int cw = (width * c.H + hmax - 1) / hmax, ch = (height * c.V + vmax - 1) / vmax;
            const int bx = (cw + 7) / 8, by = (ch + 7) / 8;
            for (int y = 0; y < by; ++y)
                for (int x = 0; x < bx; ++x) {
                    if (restartInterval && untilRestart == 0) restart();
                    decodeBlock(c, coef);
                    idct(coef, &c.plane[(static_cast<size_t>(y) * 8 * c.bw + x) * 8], c.bw * 8);
                    if (restartInterval) --untilRestart;
                }
        } else {
            for (int my = 0; my < mcuy; ++my)
                for (int mx = 0; mx < mcux; ++mx) {
                    if (restartInterval && untilRestart == 0) restart();
                    for (auto* cp : sc) {
                        JComp& c = *cp;
                        for (int v = 0; v < c.V; ++v)
                            for (int hh = 0; hh < c.H; ++hh) {
                                decodeBlock(c, coef);
                                const int bx = mx * c.H + hh, by = my * c.V + v;
                                idct(coef, &c.plane[(static_cast<size_t>(by) * 8 * c.bw + bx) * 8], c.bw * 8);
                            }
                    }
                    if (restartInterval) --untilRestart;
                }
        }
        // continue after the scan's entropy-coded data at its terminating marker
        resetBits();
        while (pos + 1 < n && !(d[pos] == 0xFF && d[pos + 1] != 0x00 && !(d[pos + 1] >= 0xD0 && d[pos + 1] <= 0xD7)))
            ++pos;
    }

    void decode(std::vector<uint8_t>& rgba, int& w, int& h, int& channelsInFile)
    {
        if (n < 4 || d[0] != 0xFF || d[1] != 0xD8) bad("JPEG: bad SOI");
        pos = 2;
        bool scanned = false;
        while (true) {
            if (pos >= n) {
                if (scanned) break;   // a missing EOI after complete scans is tolerated
                bad("JPEG: truncated file");
            }
            if (d[pos] != 0xFF) { ++pos; continue; }
            while (pos < n && d[pos] == 0xFF) ++pos;   // fill bytes
            if (pos >= n) bad("JPEG: truncated file");
            const int m = d[pos++];
            if (m == 0xD9) break;
            if (m == 0xC0 || m == 0xC1) { if (frame) bad("JPEG: second frame header"); parseSof(); }
            else if (m == 0xC2) bad("JPEG: progressive JPEG is not supported");
            else if (m == 0xC4) parseDht();
            else if (m == 0xDB) parseDqt();
            else if (m == 0xDD) { if (u16() != 4) bad("JPEG: bad DRI"); restartInterval = u16(); }
            else if (m == 0xDA) { parseSos(); scanned = true; }
            else if ((m >= 0xC3 && m <= 0xCF) || m == 0xDC) bad("JPEG: unsupported coding process");
            else if (m == 0xEE || m == 0xE0) {   // APP14 (Adobe colour transform), APP0 (JFIF)
                const int len = u16();
                if (len < 2 || pos + static_cast<size_t>(len) - 2 > n) bad("JPEG: truncated marker");
                if (m == 0xEE && len >= 14 && std::memcmp(d + pos, "Adobe", 5) == 0) adobeTransform = d[pos + 11];
                if (m == 0xE0 && len >= 7 && std::memcmp(d + pos, "JFIF", 5) == 0) jfif = true;
                pos += static_cast<size_t>(len) - 2;
            } else if ((m >= 0xE0 && m <= 0xEF) || m == 0xFE || (m >= 0xF0 && m <= 0xFD)) {
                const int len = u16();
                if (len < 2 || pos + static_cast<size_t>(len) - 2 > n) bad("JPEG: truncated marker");
                pos += static_cast<size_t>(len) - 2;
            } else if (m >= 0xD0 && m <= 0xD7) {
                // stray restart marker between segments
            } else if (m == 0x01) {
            } else {
                bad("JPEG: unknown marker");
            }
        }
        if (!frame || !scanned) bad("JPEG: no image");
        w = width;
        h = height;
        channelsInFile = static_cast<int>(comps.size());
        rgba.assign(static_cast<size_t>(w) * h * 4, 255);
        // each component at full resolution
        std::vector<std::vector<uint8_t>> full(comps.size());
        for (size_t k = 0; k < comps.size(); ++k) upsample(comps[k], full[k]);
        // three components are RGB when named 'R','G','B', or marked untransformed by an Adobe segment without JFIF
        const bool rgbIds = comps.size() == 3 && comps[0].id == 'R' && comps[1].id == 'G' && comps[2].id == 'B';
        const bool ycc = comps.size() == 3 && !(rgbIds || (adobeTransform == 0 && !jfif));
        const size_t np = static_cast<size_t>(w) * h;
        if (comps.size() == 1) {
            for (size_t i = 0; i < np; ++i) rgba[4 * i] = rgba[4 * i + 1] = rgba[4 * i + 2] = full[0][i];
        } else if (!ycc) {
            for (size_t i = 0; i < np; ++i) {
                rgba[4 * i] = full[0][i]; rgba[4 * i + 1] = full[1][i]; rgba[4 * i + 2] = full[2][i];
            }
        } else {
            // JFIF (T.871): R = Y + 1.402 Cr', G = Y - 0.34414 Cb' - 0.71414 Cr', B = Y + 1.772 Cb', in 20-bit fixed
            // point with 12-bit coefficients; the Cb term of G is truncated to 16 fractional bits
            auto coef = [](double v) { return static_cast<int32_t>(v * 4096.0 + 0.5) * 256; };
            const int32_t kR = coef(1.40200), kB = coef(1.77200), kGr = coef(0.71414), kGb = coef(0.34414);
            auto clamp8 = [](int32_t v) { return static_cast<uint8_t>(v < 0 ? 0 : (v > 255 ? 255 : v)); };
            for (size_t i = 0; i < np; ++i) {
                const int32_t y = (static_cast<int32_t>(full[0][i]) << 20) + (1 << 19);
                const int32_t cb = full[1][i] - 128, cr = full[2][i] - 128;
                const int32_t gCb = static_cast<int32_t>(static_cast<uint32_t>(cb * -kGb) & 0xffff0000u);
                rgba[4 * i] = clamp8((y + cr * kR) >> 20);
                rgba[4 * i + 1] = clamp8((y + cr * -kGr + gCb) >> 20);
                rgba[4 * i + 2] = clamp8((y + cb * kB) >> 20);
            }
        }
    }

    // component plane -> width x height samples: triangle filter for 2x, replication otherwise
    void upsample(const JComp& c, std::vector<uint8_t>& out) const
    {
        const int fx = hmax / c.H, fy = vmax / c.V;
        if (hmax % c.H || vmax % c.V) bad("JPEG: sampling factors that do not divide the maximum");
        const int pw = c.bw * 8;
        const int cw = (width * c.H + hmax - 1) / hmax, chh = (height * c.V + vmax - 1) / vmax;
        out.assign(static_cast<size_t>(width) * height, 0);
        auto at = [&](int x, int y) -> int {
            x = x < 0 ? 0 : (x >= cw ? cw - 1 : x);
            y = y < 0 ? 0 : (y >= chh ? chh - 1 : y);
            return c.plane[static_cast<size_t>(y) * pw + x];
        };
        if (fx == 1 && fy == 1) {
            for (int y = 0; y < height; ++y)
                std::memcpy(&out[static_cast<size_t>(y) * width], &c.plane[static_cast<size_t>(y) * pw],
                            static_cast<size_t>(width));
            return;
        }
        if (fx == 2 && cw == 1) {   // one sample across: no horizontal blend (vertical only for 2x2)
            for (int y = 0; y < height; ++y) {
                const int sy = y / fy, ny = fy == 2 ? (y & 1 ? sy + 1 : sy - 1) : sy;
                const int v = fy == 2 ? (3 * at(0, sy) + at(0, ny) + 2) >> 2 : at(0, sy);
                for (int x = 0; x < width; ++x) out[static_cast<size_t>(y) * width + x] = static_cast<uint8_t>(v);
            }
            return;
        }
        if ((fx == 2 || fx == 1) && (fy == 2 || fy == 1)) {
            for (int y = 0; y < height; ++y) {
                const int sy = y / fy;
                // vertical neighbour: the row above for an upper output row, below for a lower one
                const int ny = fy == 2 ? (y & 1 ? sy + 1 : sy - 1) : sy;
                for (int x = 0; x < width; ++x) {
                    const int sx = x / fx;
                    int v;
                    if (fx == 2) {
                        const int nx = x & 1 ? sx + 1 : sx - 1;
                        if (fy == 2) {
                            const int near = 3 * at(sx, sy) + at(sx, ny), far = 3 * at(nx, sy) + at(nx, ny);
                            v = (3 * near + far + 8) >> 4;
                        } else if (!(x & 1) && sx == cw - 1) {
                            // last chroma sample of a row, first of its two outputs: 3/4 of the previous sample,
                            // the edge rule of the reference's decoder (measured against it)
                            v = (3 * at(sx - 1, sy) + at(sx, sy) + 2) >> 2;
                        } else {
                            v = (3 * at(sx, sy) + at(nx, sy) + 2) >> 2;
                        }
                    } else {
                        v = (3 * at(sx, sy) + at(sx, ny) + 2) >> 2;
                    }
                    out[static_cast<size_t>(y) * width + x] = static_cast<uint8_t>(v);
                }
            }
            return;
        }
        for (int y = 0; y < height; ++y)
            for (int x = 0; x < width; ++x) out[static_cast<size_t>(y) * width + x] = static_cast<uint8_t>(at(x / fx, y / fy));
    }
};

}  // namespace

bool decodeImageRGBA8(const uint8_t* data, size_t size, std::vector<uint8_t>& rgba, int& width, int& height,
                      int& channelsInFile, std::string& err)
{
    try {
        if (size >= 8 && data[0] == 137 && data[1] == 'P' && data[2] == 'N' && data[3] == 'G') {
            decodePng(data, size, rgba, width, height, channelsInFile);
        } else if (size >= 3 && data[0] == 0xFF && data[1] == 0xD8 && data[2] == 0xFF) {
            JpegDecoder j{data, size};
            j.decode(rgba, width, height, channelsInFile);
        } else {
            bad("unsupported image format (PNG and JPEG are decoded)");
        }
        return true;
    } catch (const ImageError& e) {
        err = e.msg;
    } catch (const std::bad_alloc&) {
        err = "out of memory decoding the image";
    }
    rgba.clear();
    width = height = channelsInFile = 0;
    return false;
}

bool decodeImageRGBA16(const uint8_t* data, size_t size, std::vector<uint8_t>& rgba16le)
{
    rgba16le.clear();
    if (!(size >= 8 && data[0] == 137 && data[1] == 'P' && data[2] == 'N' && data[3] == 'G')) return false;
    try {
        std::vector<uint8_t> unused;
        int w = 0, h = 0, c = 0;
        decodePng(data, size, unused, w, h, c, &rgba16le);
    } catch (const ImageError&) {
        rgba16le.clear();
    }
    return !rgba16le.empty();
}

bool loadImageRGBA8(const std::string& path, std::vector<uint8_t>& rgba, int& width, int& height, int& channelsInFile,
                    std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "cannot open \"" + path + "\"";
        return false;
    }
    std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    if (!decodeImageRGBA8(bytes.data(), bytes.size(), rgba, width, height, channelsInFile, err)) {
        err = "\"" + path + "\": " + err;
        return false;
    }
    return true;
}

}  // namespace bte

extern "C" {

int bte_image_decode(const uint8_t* bytes, long long size, uint8_t* outRGBA, long long capacity, int* width,
                     int* height, int* channelsInFile)
{
    if (!bytes || size <= 0) { bte::setError("bte_image_decode: no data"); return -1; }
    std::vector<uint8_t> px;
    int w = 0, h = 0, c = 0;
    std::string err;
    if (!bte::decodeImageRGBA8(bytes, static_cast<size_t>(size), px, w, h, c, err)) {
        bte::setError("bte_image_decode: " + err);
        return -1;
    }
    if (width) *width = w;
    if (height) *height = h;
    if (channelsInFile) *channelsInFile = c;
    if (outRGBA) {
        if (capacity < static_cast<long long>(px.size())) { bte::setError("bte_image_decode: output buffer too small"); return -1; }
        std::memcpy(outRGBA, px.data(), px.size());
    }
    return 0;
}

}  // extern "C"
