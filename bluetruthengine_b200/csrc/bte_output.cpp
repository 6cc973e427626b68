// bte_output.cpp -- headless output in place of the reference's window.
//
// The reference displays each frame through an OpenGL pixel buffer and, on
// key presses, saves it as a PNG (captureScreenshot, src/main.cpp:118-142:
// glReadPixels, rows flipped so the file starts at the top, stbi_write_png
// to screenshot_%04d.png) or streams it to FFmpeg (startRecording /
// stopRecording, :72-116, and the per-frame glReadPixels + fwrite of
// :990-997: raw RGBA rows bottom first, `-vf vflip` in the FFmpeg command).
// There is no window here, so the same outputs come from the framebuffer the
// last bte_render packed (row 0 = the bottom row, as the pixel buffer holds
// it):
//   bte_write_png / bte_capture_screenshot   the PNG, top row first
//   bte_record_start / _frame / _stop        raw frames to the same FFmpeg
//                                            command, or to a file
// The PNG encoder is written here: adaptive per-row filters (the one with the
// smallest sum of absolute residuals) and DEFLATE with LZ77 over a 32 KiB
// window and the fixed Huffman codes (RFC 1951 3.2.6).  Any PNG decoder
// reads back the exact pixels; the compressed bytes differ from stb's.
#include "bte_internal.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace bte {

namespace {

// ---------------------------------------------------------------- checksums
uint32_t crc32(const uint8_t* p, size_t n, uint32_t crc = 0)
{
    struct Table {
        uint32_t t[256];
        Table()
        {
            for (uint32_t i = 0; i < 256; ++i) {
                uint32_t c = i;
                for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xedb88320u ^ (c >> 1) : c >> 1;
                t[i] = c;
            }
        }
    };
    static const Table table;
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table.t[(crc ^ p[i]) & 0xffu] ^ (crc >> 8);
    return ~crc;
}

uint32_t adler32(const uint8_t* p, size_t n)
{
    uint32_t a = 1, b = 0;
    while (n) {
        const size_t k = n < 5552 ? n : 5552;
        for (size_t i = 0; i < k; ++i) { a += p[i]; b += a; }
        a %= 65521u;
        b %= 65521u;
        p += k;
        n -= k;
    }
    return (b << 16) | a;
}

// ---------------------------------------------------------------- DEFLATE, fixed codes
struct BitWriter {
    std::vector<uint8_t>& out;
    uint32_t buf = 0;
    int n = 0;
    void put(uint32_t v, int bits)   // LSB first
    {
        buf |= v << n;
        n += bits;
        while (n >= 8) {
            out.push_back(static_cast<uint8_t>(buf));
            buf >>= 8;
            n -= 8;
        }
    }
    void code(uint32_t c, int len)   // Huffman codes go most significant bit first
    {
        uint32_t r = 0;
        for (int i = 0; i < len; ++i) r |= ((c >> i) & 1u) << (len - 1 - i);
        put(r, len);
    }
    void flush()
    {
        if (n > 0) out.push_back(static_cast<uint8_t>(buf));
        buf = 0;
        n = 0;
    }
};

void literal(BitWriter& w, int sym)
{
    if (sym < 144) w.code(0x30u + sym, 8);
    else if (sym < 256) w.code(0x190u + (sym - 144), 9);
    else if (sym < 280) w.code(static_cast<uint32_t>(sym - 256), 7);
    else w.code(0xc0u + (sym - 280), 8);
}

const uint16_t kLenBase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31, 35, 43, 51, 59, 67, 83, 99,
                               115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129, 193, 257, 385, 513, 769, 1025, 1537,
                                2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12,
                                13, 13};

void match(BitWriter& w, int len, int dist)
{
    int li = 28;
    while (kLenBase[li] > len) --li;
    literal(w, 257 + li);
    w.put(static_cast<uint32_t>(len - kLenBase[li]), kLenExtra[li]);
    int di = 29;
    while (kDistBase[di] > dist) --di;
    w.code(static_cast<uint32_t>(di), 5);
    w.put(static_cast<uint32_t>(dist - kDistBase[di]), kDistExtra[di]);
}

// zlib stream of `d`: one fixed-code block, greedy LZ77 with hash chains
std::vector<uint8_t> zlibCompress(const std::vector<uint8_t>& d)
{
    std::vector<uint8_t> out;
    out.reserve(d.size() / 2 + 64);
    out.push_back(0x78);
    out.push_back(0x5e);   // 32 KiB window, default compression level flag
    BitWriter w{out};
    w.put(1, 1);   // final block
    w.put(1, 2);   // fixed codes
    constexpr int kHashBits = 15, kWindow = 32768, kMaxChain = 48, kMaxLen = 258;
    std::vector<int> head(1u << kHashBits, -1), prev(kWindow, -1);
    const int n = static_cast<int>(d.size());
    auto hash = [&](int i) {
        const uint32_t v = (static_cast<uint32_t>(d[i]) << 16) | (static_cast<uint32_t>(d[i + 1]) << 8) | d[i + 2];
        return (v * 2654435761u) >> (32 - kHashBits);
    };
    auto insert = [&](int i) {
        if (i + 2 >= n) return;
        const uint32_t h = hash(i);
        prev[i & (kWindow - 1)] = head[h];
        head[h] = i;
    };
    int i = 0;
    while (i < n) {
        int bestLen = 0, bestDist = 0;
        if (i + 2 < n) {
            int cand = head[hash(i)];
            const int maxLen = n - i < kMaxLen ? n - i : kMaxLen;
            for (int chain = 0; cand >= 0 && i - cand <= kWindow - 1 && chain < kMaxChain; ++chain) {
                if (d[cand + bestLen] == d[i + bestLen]) {
                    int l = 0;
                    while (l < maxLen && d[cand + l] == d[i + l]) ++l;
                    if (l > bestLen) { bestLen = l; bestDist = i - cand; if (l == maxLen) break; }
                }
                const int nx = prev[cand & (kWindow - 1)];
                if (nx >= cand) break;
                cand = nx;
            }
        }
        if (bestLen >= 3) {
            match(w, bestLen, bestDist);
            for (int k = 0; k < bestLen; ++k) insert(i + k);
            i += bestLen;
        } else {
            literal(w, d[i]);
            insert(i);
            ++i;
        }
    }
    literal(w, 256);
    w.flush();
    const uint32_t a = adler32(d.data(), d.size());
    for (int k = 3; k >= 0; --k) out.push_back(static_cast<uint8_t>(a >> (8 * k)));
    return out;
}

// ---------------------------------------------------------------- PNG
void chunk(std::vector<uint8_t>& png, const char* type, const std::vector<uint8_t>& data)
{
    const uint32_t len = static_cast<uint32_t>(data.size());
    for (int k = 3; k >= 0; --k) png.push_back(static_cast<uint8_t>(len >> (8 * k)));
    const size_t start = png.size();
    png.insert(png.end(), type, type + 4);
    png.insert(png.end(), data.begin(), data.end());
    const uint32_t c = crc32(png.data() + start, png.size() - start);
    for (int k = 3; k >= 0; --k) png.push_back(static_cast<uint8_t>(c >> (8 * k)));
}

int paethPredict(int a, int b, int c)
{
    const int p = a + b - c;
    const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    if (pb <= pc) return b;
    return c;
}

// RGBA8 rows (row 0 first in the file) -> PNG bytes
std::vector<uint8_t> encodePng(const uint8_t* rgba, int w, int h)
{
    const size_t rb = static_cast<size_t>(w) * 4;
    std::vector<uint8_t> raw;
    raw.reserve((rb + 1) * h);
    std::vector<uint8_t> zero(rb, 0), cand(rb), best(rb);
    for (int y = 0; y < h; ++y) {
        const uint8_t* x = rgba + static_cast<size_t>(y) * rb;
        const uint8_t* up = y > 0 ? rgba + static_cast<size_t>(y - 1) * rb : zero.data();
        long bestCost = -1;
        int bestF = 0;
        for (int f = 0; f < 5; ++f) {
            long cost = 0;
            for (size_t i = 0; i < rb; ++i) {
                const int a = i >= 4 ? x[i - 4] : 0, b = up[i], c = i >= 4 ? up[i - 4] : 0;
                const int pred = f == 0 ? 0 : f == 1 ? a : f == 2 ? b : f == 3 ? (a + b) / 2 : paethPredict(a, b, c);
                const uint8_t r = static_cast<uint8_t>(x[i] - pred);
                cand[i] = r;
                cost += r < 128 ? r : 256 - r;
            }
            if (bestCost < 0 || cost < bestCost) { bestCost = cost; bestF = f; best.swap(cand); }
        }
        raw.push_back(static_cast<uint8_t>(bestF));
        raw.insert(raw.end(), best.begin(), best.end());
    }
    std::vector<uint8_t> png = {137, 80, 78, 71, 13, 10, 26, 10};
    std::vector<uint8_t> ihdr(13);
    for (int k = 0; k < 4; ++k) {
        ihdr[k] = static_cast<uint8_t>(static_cast<uint32_t>(w) >> (24 - 8 * k));
        ihdr[4 + k] = static_cast<uint8_t>(static_cast<uint32_t>(h) >> (24 - 8 * k));
    }
    ihdr[8] = 8;    // bit depth
    ihdr[9] = 6;    // RGBA
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", zlibCompress(raw));
    chunk(png, "IEND", {});
    return png;
}

// the current framebuffer, rows top first (the pixel buffer's row 0 is the bottom one)
bool framebufferTopFirst(std::vector<uint8_t>& rgba, int& w, int& h)
{
    if (bte_get_framebuffer_size(&w, &h) != 0) return false;
    std::vector<uint32_t> fb(static_cast<size_t>(w) * h);
    if (bte_read_framebuffer(fb.data()) != 0) return false;
    rgba.resize(fb.size() * 4);
    for (int y = 0; y < h; ++y)
        std::memcpy(&rgba[static_cast<size_t>(y) * w * 4], &fb[static_cast<size_t>(h - 1 - y) * w], static_cast<size_t>(w) * 4);
    return true;
}

FILE* g_record = nullptr;
bool g_recordPipe = false;
int g_shot = 0;

}  // namespace

}  // namespace bte

extern "C" {

int bte_encode_png(const uint8_t* rgba, int width, int height, uint8_t* out, long long capacity, long long* size)
{
    if (!rgba || width <= 0 || height <= 0) { bte::setError("bte_encode_png: empty image"); return -1; }
    const std::vector<uint8_t> png = bte::encodePng(rgba, width, height);
    if (size) *size = static_cast<long long>(png.size());
    if (out) {
        if (capacity < static_cast<long long>(png.size())) { bte::setError("bte_encode_png: output buffer too small"); return -1; }
        std::memcpy(out, png.data(), png.size());
    }
    return 0;
}

int bte_write_png(const char* path)
{
    if (!path || !*path) { bte::setError("bte_write_png: no path"); return -1; }
    std::vector<uint8_t> rgba;
    int w = 0, h = 0;
    if (!bte::framebufferTopFirst(rgba, w, h)) return -1;
    const std::vector<uint8_t> png = bte::encodePng(rgba.data(), w, h);
    FILE* f = std::fopen(path, "wb");
    if (!f) { bte::setError(std::string("bte_write_png: cannot open ") + path); return -1; }
    const size_t wrote = std::fwrite(png.data(), 1, png.size(), f);
    const bool ok = std::fclose(f) == 0 && wrote == png.size();
    if (!ok) { bte::setError(std::string("bte_write_png: write failed for ") + path); return -1; }
    return 0;
}

// captureScreenshot (src/main.cpp:118-142): screenshot_0000.png, screenshot_0001.png, ... in the working directory
int bte_capture_screenshot(char* nameOut, int nameCapacity)
{
    char name[64];
    std::snprintf(name, sizeof(name), "screenshot_%04d.png", bte::g_shot);
    if (bte_write_png(name) != 0) return -1;
    ++bte::g_shot;
    if (nameOut && nameCapacity > 0) std::snprintf(nameOut, static_cast<size_t>(nameCapacity), "%s", name);
    return 0;
}

// startRecording (src/main.cpp:79-103): rawPath NULL opens the reference's FFmpeg pipe (H.264 output.mp4 at
// `fps`, frames flipped by FFmpeg); otherwise the raw RGBA frames, rows bottom first, go to that file.
int bte_record_start(const char* rawPath, int fps)
{
    if (bte::g_record) { bte::setError("bte_record_start: already recording"); return -1; }
    int w = 0, h = 0;
    if (bte_get_framebuffer_size(&w, &h) != 0) return -1;
    if (rawPath) {
        bte::g_record = std::fopen(rawPath, "wb");
        bte::g_recordPipe = false;
    } else {
        char cmd[512];
        std::snprintf(cmd, sizeof(cmd),
                      "ffmpeg -y -f rawvideo -pixel_format rgba -video_size %dx%d -r %d -i pipe:0 "
                      "-vf vflip -c:v libx264 -crf 18 -pix_fmt yuv420p output.mp4",
                      w, h, fps > 0 ? fps : 30);
        bte::g_record = popen(cmd, "w");
        bte::g_recordPipe = true;
    }
    if (!bte::g_record) { bte::setError("bte_record_start: could not open the output (is ffmpeg on PATH?)"); return -1; }
    return 0;
}

int bte_record_frame(void)
{
    if (!bte::g_record) { bte::setError("bte_record_frame: not recording"); return -1; }
    int w = 0, h = 0;
    if (bte_get_framebuffer_size(&w, &h) != 0) return -1;
    std::vector<uint32_t> fb(static_cast<size_t>(w) * h);
    if (bte_read_framebuffer(fb.data()) != 0) return -1;
    if (std::fwrite(fb.data(), 4, fb.size(), bte::g_record) != fb.size()) {
        bte::setError("bte_record_frame: write failed");
        return -1;
    }
    return 0;
}

int bte_record_stop(void)
{
    if (!bte::g_record) return 0;
    const int rc = bte::g_recordPipe ? pclose(bte::g_record) : std::fclose(bte::g_record);
    bte::g_record = nullptr;
    if (rc != 0) { bte::setError("bte_record_stop: closing the output failed"); return -1; }
    return 0;
}

}  // extern "C"
