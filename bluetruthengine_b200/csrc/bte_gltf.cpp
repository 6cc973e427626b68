// bte_gltf.cpp -- glTF 2.0 / GLB models flattened into triangles and Disney BSDFs.
//
// The reference's <model> drop-ins (src/gltf_loader.cpp:768-846, loadGltfModel,
// called from src/main.cpp:760-817) read a .gltf / .glb file with tinygltf
// and GLM.  This is a reader of the same files with the same results:
//   * JSON (RFC 8259) and the GLB container (glTF 2.0 spec section 4.4):
//     buffers from the binary chunk, base64 data URIs or files next to the
//     model; accessors of every component type, normalized integers, byte
//     strides (sparse accessors are ignored, as the reference's reader does);
//   * images decoded with the library's decoder as tinygltf asks stb_image
//     for them (4 channels; 16-bit PNGs kept at 16 bits, which the
//     reference's RGBA conversion then reads 4 bytes per pixel,
//     gltf_loader.cpp:279-302 -- reproduced so textures match);
//   * the node graph of the default scene (all nodes when there is none),
//     matrices or translation / rotation / scale, the <model> transform
//     applied outside it (gltf_loader.cpp:37-82);
//   * primitives: triangles, strips and fans; POSITION, NORMAL (transformed
//     by the inverse transpose, else the face normal), TEXCOORD_0
//     (gltf_loader.cpp:486-566);
//   * skipped: nodes named "background" / containing "backgroundgradient",
//     primitives whose material name contains "outline" or is
//     "backgroundgradient", and primitives whose world box is more than 12x
//     the median extent or whose centre is more than 10x it from the median
//     centre, when a model has at least four (:568-720);
//   * materials (disneyFromGltf, :311-455): base colour (factor baked into the
//     texture when there is one), metallic, roughness, KHR_materials_ior /
//     _transmission / _clearcoat / _sheen / _emissive_strength / _unlit,
//     emission; a default material for primitives without one, dropped when
//     unused.
// The transform arithmetic follows GLM's formulation of translate / rotate /
// scale / quaternion-to-matrix / 3x3 inverse and matrix products (float, no
// contraction), operation for operation.
#include "bte_internal.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <new>
#include <set>
#include <string>
#include <vector>

namespace bte {

namespace {

struct GltfError {
    std::string msg;
};
[[noreturn]] void gfail(const std::string& m) { throw GltfError{m}; }

// ================================================================ JSON
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    const Json* get(const char* key) const
    {
        if (kind != Object) return nullptr;
        for (const auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    double numOr(const char* key, double fallback) const
    {
        const Json* v = get(key);
        return (v && v->kind == Number) ? v->num : fallback;
    }
    int intOr(const char* key, int fallback) const
    {
        const Json* v = get(key);
        return (v && v->kind == Number) ? static_cast<int>(v->num) : fallback;
    }
    std::string strOr(const char* key) const
    {
        const Json* v = get(key);
        return (v && v->kind == String) ? v->str : std::string();
    }
    std::vector<double> numbers(const char* key) const
    {
        std::vector<double> out;
        const Json* v = get(key);
        if (v && v->kind == Array)
            for (const auto& e : v->arr) out.push_back(e.kind == Number ? e.num : 0.0);
        return out;
    }
};

struct JsonParser {
    const char* p;
    const char* end;
    int depth = 0;
    void ws() { while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p; }
    [[noreturn]] void err(const char* m) { gfail(std::string("glTF JSON: ") + m); }
    void expect(char c)
    {
        ws();
        if (p >= end || *p != c) err("unexpected character");
        ++p;
    }
    static void utf8(std::string& s, uint32_t cp)
    {
        if (cp < 0x80) s += static_cast<char>(cp);
        else if (cp < 0x800) { s += static_cast<char>(0xc0 | (cp >> 6)); s += static_cast<char>(0x80 | (cp & 63)); }
        else if (cp < 0x10000) {
            s += static_cast<char>(0xe0 | (cp >> 12)); s += static_cast<char>(0x80 | ((cp >> 6) & 63));
            s += static_cast<char>(0x80 | (cp & 63));
        } else {
            s += static_cast<char>(0xf0 | (cp >> 18)); s += static_cast<char>(0x80 | ((cp >> 12) & 63));
            s += static_cast<char>(0x80 | ((cp >> 6) & 63)); s += static_cast<char>(0x80 | (cp & 63));
        }
    }
    uint32_t hex4()
    {
        if (end - p < 4) err("bad \\u escape");
        uint32_t v = 0;
        for (int i = 0; i < 4; ++i) {
            const char c = *p++;
            v <<= 4;
            if (c >= '0' && c <= '9') v |= static_cast<uint32_t>(c - '0');
            else if (c >= 'a' && c <= 'f') v |= static_cast<uint32_t>(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= static_cast<uint32_t>(c - 'A' + 10);
            else err("bad \\u escape");
        }
        return v;
    }
    std::string string()
    {
        expect('"');
        std::string s;
        while (true) {
            if (p >= end) err("unterminated string");
            const char c = *p++;
            if (c == '"') break;
            if (c != '\\') { s += c; continue; }
            if (p >= end) err("unterminated string");
            const char e = *p++;
            switch (e) {
            case '"': s += '"'; break;
            case '\\': s += '\\'; break;
            case '/': s += '/'; break;
            case 'b': s += '\b'; break;
            case 'f': s += '\f'; break;
            case 'n': s += '\n'; break;
            case 'r': s += '\r'; break;
            case 't': s += '\t'; break;
            case 'u': {
                uint32_t cp = hex4();
                if (cp >= 0xd800 && cp < 0xdc00 && end - p >= 6 && p[0] == '\\' && p[1] == 'u') {
                    p += 2;
                    const uint32_t lo = hex4();
                    cp = 0x10000 + ((cp - 0xd800) << 10) + (lo - 0xdc00);
                }
                utf8(s, cp);
                break;
            }
            default: err("bad escape");
            }
        }
        return s;
    }
    Json value()
    {
        if (++depth > 512) err("nesting too deep");
        ws();
        if (p >= end) err("unexpected end");
        Json v;
        const char c = *p;
        if (c == '{') {
            v.kind = Json::Object;
            ++p;
            ws();
            if (p < end && *p == '}') { ++p; }
            else {
                while (true) {
                    ws();
                    std::string k = string();
                    expect(':');
                    Json x = value();
                    v.obj.emplace_back(std::move(k), std::move(x));
                    ws();
                    if (p < end && *p == ',') { ++p; continue; }
                    expect('}');
                    break;
                }
            }
        } else if (c == '[') {
            v.kind = Json::Array;
            ++p;
            ws();
            if (p < end && *p == ']') { ++p; }
            else {
                while (true) {
                    v.arr.push_back(value());
                    ws();
                    if (p < end && *p == ',') { ++p; continue; }
                    expect(']');
                    break;
                }
            }
        } else if (c == '"') {
            v.kind = Json::String;
            v.str = string();
        } else if (end - p >= 4 && std::strncmp(p, "true", 4) == 0) {
            v.kind = Json::Bool; v.b = true; p += 4;
        } else if (end - p >= 5 && std::strncmp(p, "false", 5) == 0) {
            v.kind = Json::Bool; v.b = false; p += 5;
        } else if (end - p >= 4 && std::strncmp(p, "null", 4) == 0) {
            p += 4;
        } else {
            const char* s = p;
            while (p < end && (std::strchr("+-0123456789.eE", *p) != nullptr)) ++p;
            if (p == s) err("unexpected character");
            const std::string t(s, p);
            char* q = nullptr;
            v.kind = Json::Number;
            v.num = std::strtod(t.c_str(), &q);
            if (!q || *q) err("bad number");
        }
        --depth;
        return v;
    }
};

// ================================================================ file access
std::vector<uint8_t> readFile(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) gfail("cannot open \"" + path + "\"");
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

std::vector<uint8_t> base64(const std::string& s, size_t from)
{
    auto val = [](char c) -> int {
        if (c >= 'A' && c <= 'Z') return c - 'A';
        if (c >= 'a' && c <= 'z') return c - 'a' + 26;
        if (c >= '0' && c <= '9') return c - '0' + 52;
        if (c == '+' || c == '-') return 62;
        if (c == '/' || c == '_') return 63;
        return -1;
    };
    std::vector<uint8_t> out;
    uint32_t acc = 0;
    int bits = 0;
    for (size_t i = from; i < s.size(); ++i) {
        const int v = val(s[i]);
        if (v < 0) {
            if (s[i] == '=') break;
            continue;
        }
        acc = (acc << 6) | static_cast<uint32_t>(v);
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out.push_back(static_cast<uint8_t>(acc >> bits));
        }
    }
    return out;
}

std::string percentDecode(const std::string& s)
{
    std::string o;
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] == '%' && i + 2 < s.size() && std::isxdigit(static_cast<unsigned char>(s[i + 1])) &&
            std::isxdigit(static_cast<unsigned char>(s[i + 2]))) {
            o += static_cast<char>(std::strtol(s.substr(i + 1, 2).c_str(), nullptr, 16));
            i += 2;
        } else {
            o += s[i];
        }
    }
    return o;
}

// a buffer or image URI: base64 data URI, or a file relative to the model
std::vector<uint8_t> loadUri(const std::string& uri, const std::string& dir)
{
    if (uri.compare(0, 5, "data:") == 0) {
        const size_t comma = uri.find(',');
        if (comma == std::string::npos || uri.rfind(";base64", comma) == std::string::npos)
            gfail("unsupported data URI");
        return base64(uri, comma + 1);
    }
    return readFile(dir + percentDecode(uri));
}

// ================================================================ GLM-formulated float math
struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };
struct M4 { V4 c[4]; };   // columns
struct M3 { V3 c[3]; };

V4 operator*(const V4& a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
V4 operator+(const V4& a, const V4& b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }

M4 identity()
{
    M4 m{};
    m.c[0] = {1, 0, 0, 0}; m.c[1] = {0, 1, 0, 0}; m.c[2] = {0, 0, 1, 0}; m.c[3] = {0, 0, 0, 1};
    return m;
}
float comp(const V4& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }

// glm::operator*(mat4, mat4): column j = ((A0 B[j][0] + A1 B[j][1]) + A2 B[j][2]) + A3 B[j][3]
M4 mul(const M4& a, const M4& b)
{
    M4 r;
    for (int j = 0; j < 4; ++j) r.c[j] = a.c[0] * b.c[j].x + a.c[1] * b.c[j].y + a.c[2] * b.c[j].z + a.c[3] * b.c[j].w;
    return r;
}
// glm::operator*(mat4, vec4): (m0 v0 + m1 v1) + (m2 v2 + m3 v3)
V4 mulv(const M4& m, const V4& v)
{
    const V4 a0 = m.c[0] * v.x + m.c[1] * v.y;
    const V4 a1 = m.c[2] * v.z + m.c[3] * v.w;
    return a0 + a1;
}
M4 translate(const M4& m, float x, float y, float z)
{
    M4 r = m;
    r.c[3] = m.c[0] * x + m.c[1] * y + m.c[2] * z + m.c[3];
    return r;
}
M4 scale(const M4& m, float x, float y, float z)
{
    M4 r = m;
    r.c[0] = m.c[0] * x; r.c[1] = m.c[1] * y; r.c[2] = m.c[2] * z;
    return r;
}
// glm::rotate(m, angle, axis) with a unit axis
M4 rotate(const M4& m, float angle, float ax, float ay, float az)
{
    const float c = std::cos(angle), s = std::sin(angle);
    const float inv = 1.0f / std::sqrt(ax * ax + ay * ay + az * az);
    const float x = ax * inv, y = ay * inv, z = az * inv;
    const float t0 = (1.0f - c) * x, t1 = (1.0f - c) * y, t2 = (1.0f - c) * z;
    const float r00 = c + t0 * x, r01 = t0 * y + s * z, r02 = t0 * z - s * y;
    const float r10 = t1 * x - s * z, r11 = c + t1 * y, r12 = t1 * z + s * x;
    const float r20 = t2 * x + s * y, r21 = t2 * y - s * x, r22 = c + t2 * z;
    M4 r;
    r.c[0] = m.c[0] * r00 + m.c[1] * r01 + m.c[2] * r02;
    r.c[1] = m.c[0] * r10 + m.c[1] * r11 + m.c[2] * r12;
    r.c[2] = m.c[0] * r20 + m.c[1] * r21 + m.c[2] * r22;
    r.c[3] = m.c[3];
    return r;
}
// glm::mat4_cast(quat(w, x, y, z))
M4 quatToMat(float w, float x, float y, float z)
{
    const float xx = x * x, yy = y * y, zz = z * z, xz = x * z, xy = x * y, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
    M4 r = identity();
    r.c[0].x = 1.0f - 2.0f * (yy + zz); r.c[0].y = 2.0f * (xy + wz); r.c[0].z = 2.0f * (xz - wy);
    r.c[1].x = 2.0f * (xy - wz); r.c[1].y = 1.0f - 2.0f * (xx + zz); r.c[1].z = 2.0f * (yz + wx);
    r.c[2].x = 2.0f * (xz + wy); r.c[2].y = 2.0f * (yz - wx); r.c[2].z = 1.0f - 2.0f * (xx + yy);
    return r;
}
// glm::transpose(glm::inverse(mat3(m)))
M3 normalMatrix(const M4& m4)
{
    const float m00 = m4.c[0].x, m01 = m4.c[0].y, m02 = m4.c[0].z;
    const float m10 = m4.c[1].x, m11 = m4.c[1].y, m12 = m4.c[1].z;
    const float m20 = m4.c[2].x, m21 = m4.c[2].y, m22 = m4.c[2].z;
    const float od = 1.0f / (+m00 * (m11 * m22 - m21 * m12) - m10 * (m01 * m22 - m21 * m02) + m20 * (m01 * m12 - m11 * m02));
    float inv[3][3];
    inv[0][0] = +(m11 * m22 - m21 * m12) * od;
    inv[1][0] = -(m10 * m22 - m20 * m12) * od;
    inv[2][0] = +(m10 * m21 - m20 * m11) * od;
    inv[0][1] = -(m01 * m22 - m21 * m02) * od;
    inv[1][1] = +(m00 * m22 - m20 * m02) * od;
    inv[2][1] = -(m00 * m21 - m20 * m01) * od;
    inv[0][2] = +(m01 * m12 - m11 * m02) * od;
    inv[1][2] = -(m00 * m12 - m10 * m02) * od;
    inv[2][2] = +(m00 * m11 - m10 * m01) * od;
    M3 t;   // transpose: column j of the result = row j of the inverse
    for (int j = 0; j < 3; ++j) t.c[j] = {inv[0][j], inv[1][j], inv[2][j]};
    return t;
}
// glm::normalize(mat3 * v)
Float3 normalXform(const M3& m, float x, float y, float z)
{
    const float a = m.c[0].x * x + m.c[1].x * y + m.c[2].x * z;
    const float b = m.c[0].y * x + m.c[1].y * y + m.c[2].y * z;
    const float c = m.c[0].z * x + m.c[1].z * y + m.c[2].z * z;
    const float inv = 1.0f / std::sqrt(a * a + b * b + c * c);
    return {a * inv, b * inv, c * inv};
}

// ================================================================ the model
struct Accessor { int bufferView = -1, componentType = 0, count = 0, comps = 0; size_t byteOffset = 0; bool normalized = false;
                  std::vector<double> mn, mx; };
struct View { int buffer = -1; size_t byteOffset = 0, byteLength = 0, byteStride = 0; };
struct Prim { std::map<std::string, int> attributes; int indices = -1, material = -1, mode = -1; };
struct Node { std::string name; int mesh = -1; std::vector<int> children; std::vector<double> matrix, t, r, s; };
struct Image { std::vector<uint8_t> pixels; int width = 0, height = 0; };   // RGBA8 as the reference converts it

struct Model {
    std::unique_ptr<Json> json;   // the parsed document; `materials` point into it
    std::string dir;
    std::vector<std::vector<uint8_t>> buffers;
    std::vector<View> views;
    std::vector<Accessor> accessors;
    std::vector<std::vector<Prim>> meshes;
    std::vector<Node> nodes;
    std::vector<const Json*> materials;
    std::vector<int> textureSource;
    std::vector<Image> images;
    std::vector<int> roots;
};

int compSize(int ct)
{
    switch (ct) {
    case 5120: case 5121: return 1;
    case 5122: case 5123: return 2;
    case 5125: case 5126: return 4;
    default: return 0;
    }
}

int typeCount(const std::string& t)
{
    if (t == "SCALAR") return 1;
    if (t == "VEC2") return 2;
    if (t == "VEC3") return 3;
    if (t == "VEC4") return 4;
    return 0;
}

// tinygltf's image load (4 channels; 16-bit PNG samples kept at 16 bits) and the reference's RGBA conversion,
// which reads 4 bytes per pixel whatever the sample size
Image convertImage(const std::vector<uint8_t>& bytes, const std::string& what)
{
    std::vector<uint8_t> rgba8, raw16;
    int w = 0, h = 0, ch = 0;
    std::string err;
    if (!decodeImageRGBA8(bytes.data(), bytes.size(), rgba8, w, h, ch, err)) gfail(what + ": " + err);
    Image im;
    im.width = w;
    im.height = h;
    if (decodeImageRGBA16(bytes.data(), bytes.size(), raw16)) {
        im.pixels.assign(raw16.begin(), raw16.begin() + static_cast<std::ptrdiff_t>(static_cast<size_t>(w) * h * 4));
    } else {
        im.pixels = std::move(rgba8);
    }
    return im;
}

Model parseModel(const std::string& path)
{
    Model M;
    const size_t slash = path.find_last_of("/\\");
    M.dir = slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
    const std::vector<uint8_t> file = readFile(path);
    std::string jsonText;
    std::vector<uint8_t> bin;
    bool glb = false;
    if (file.size() >= 12 && std::memcmp(file.data(), "glTF", 4) == 0) {   // GLB container
        glb = true;
        auto u32 = [&](size_t o) {
            return static_cast<uint32_t>(file[o]) | (static_cast<uint32_t>(file[o + 1]) << 8) |
                   (static_cast<uint32_t>(file[o + 2]) << 16) | (static_cast<uint32_t>(file[o + 3]) << 24);
        };
        if (u32(4) != 2) gfail("GLB: unsupported version");
        const size_t total = std::min<size_t>(u32(8), file.size());
        size_t o = 12;
        bool first = true;
        while (o + 8 <= total) {
            const uint32_t len = u32(o), type = u32(o + 4);
            if (o + 8 + len > total) gfail("GLB: truncated chunk");
            if (first && type != 0x4e4f534au) gfail("GLB: first chunk is not JSON");
            if (type == 0x4e4f534au && first) jsonText.assign(reinterpret_cast<const char*>(&file[o + 8]), len);
            else if (type == 0x004e4942u && bin.empty()) bin.assign(file.begin() + static_cast<std::ptrdiff_t>(o + 8),
                                                                     file.begin() + static_cast<std::ptrdiff_t>(o + 8 + len));
            first = false;
            o += 8 + ((len + 3u) & ~3u);
        }
        if (jsonText.empty()) gfail("GLB: no JSON chunk");
    } else {
        jsonText.assign(file.begin(), file.end());
    }
    JsonParser jp{jsonText.data(), jsonText.data() + jsonText.size()};
    M.json = std::make_unique<Json>(jp.value());
    const Json& J = *M.json;
    if (J.kind != Json::Object) gfail("glTF JSON: top level is not an object");
    auto list = [&](const char* k) -> const std::vector<Json>& {
        static const std::vector<Json> none;
        const Json* v = J.get(k);
        return (v && v->kind == Json::Array) ? v->arr : none;
    };
    for (const auto& b : list("buffers")) {
        const std::string uri = b.strOr("uri");
        if (uri.empty()) {
            if (!glb) gfail("buffer without a uri outside a GLB file");
            M.buffers.push_back(bin);
        } else {
            M.buffers.push_back(loadUri(uri, M.dir));
        }
        const double len = b.numOr("byteLength", 0.0);
        if (len > static_cast<double>(M.buffers.back().size())) gfail("buffer shorter than its byteLength");
    }
    for (const auto& v : list("bufferViews")) {
        View x;
        x.buffer = v.intOr("buffer", -1);
        x.byteOffset = static_cast<size_t>(v.numOr("byteOffset", 0.0));
        x.byteLength = static_cast<size_t>(v.numOr("byteLength", 0.0));
        x.byteStride = static_cast<size_t>(v.numOr("byteStride", 0.0));
        M.views.push_back(x);
    }
    for (const auto& a : list("accessors")) {
        Accessor x;
        x.bufferView = a.intOr("bufferView", -1);
        x.byteOffset = static_cast<size_t>(a.numOr("byteOffset", 0.0));
        x.componentType = a.intOr("componentType", 0);
        x.count = a.intOr("count", 0);
        const Json* nz = a.get("normalized");
        x.normalized = nz && nz->kind == Json::Bool && nz->b;
        x.comps = typeCount(a.strOr("type"));
        x.mn = a.numbers("min");
        x.mx = a.numbers("max");
        M.accessors.push_back(x);
    }
    for (const auto& m : list("meshes")) {
        std::vector<Prim> prims;
        const Json* ps = m.get("primitives");
        if (ps && ps->kind == Json::Array)
            for (const auto& p : ps->arr) {
                Prim x;
                const Json* at = p.get("attributes");
                if (at && at->kind == Json::Object)
                    for (const auto& kv : at->obj)
                        if (kv.second.kind == Json::Number) x.attributes[kv.first] = static_cast<int>(kv.second.num);
                x.indices = p.intOr("indices", -1);
                x.material = p.intOr("material", -1);
                x.mode = p.intOr("mode", -1);
                prims.push_back(std::move(x));
            }
        M.meshes.push_back(std::move(prims));
    }
    for (const auto& n : list("nodes")) {
        Node x;
        x.name = n.strOr("name");
        x.mesh = n.intOr("mesh", -1);
        for (double c : n.numbers("children")) x.children.push_back(static_cast<int>(c));
        x.matrix = n.numbers("matrix");
        x.t = n.numbers("translation");
        x.r = n.numbers("rotation");
        x.s = n.numbers("scale");
        M.nodes.push_back(std::move(x));
    }
    for (const auto& m : list("materials")) M.materials.push_back(&m);
    for (const auto& t : list("textures")) M.textureSource.push_back(t.intOr("source", -1));
    {
        int idx = 0;
        for (const auto& im : list("images")) {
            const std::string what = "glTF image[" + std::to_string(idx++) + "]";
            const std::string uri = im.strOr("uri");
            std::vector<uint8_t> bytes;
            if (!uri.empty()) {
                bytes = loadUri(uri, M.dir);
            } else {
                const int bv = im.intOr("bufferView", -1);
                if (bv < 0 || bv >= static_cast<int>(M.views.size())) gfail(what + ": no data");
                const View& v = M.views[static_cast<size_t>(bv)];
                if (v.buffer < 0 || v.buffer >= static_cast<int>(M.buffers.size()) ||
                    v.byteOffset + v.byteLength > M.buffers[static_cast<size_t>(v.buffer)].size())
                    gfail(what + ": buffer view out of range");
                const auto& b = M.buffers[static_cast<size_t>(v.buffer)];
                bytes.assign(b.begin() + static_cast<std::ptrdiff_t>(v.byteOffset),
                             b.begin() + static_cast<std::ptrdiff_t>(v.byteOffset + v.byteLength));
            }
            M.images.push_back(convertImage(bytes, what));
        }
    }
    const int scene = J.intOr("scene", -1);
    const auto& scenes = list("scenes");
    const int si = scene >= 0 ? scene : 0;
    if (!scenes.empty() && si < static_cast<int>(scenes.size())) {
        for (double r : scenes[static_cast<size_t>(si)].numbers("nodes")) M.roots.push_back(static_cast<int>(r));
    } else {
        for (int i = 0; i < static_cast<int>(M.nodes.size()); ++i) M.roots.push_back(i);
    }
    return M;
}

// ---------------------------------------------------------------- accessors (gltf_loader.cpp:109-255)
float readFloat(const uint8_t* p, int ct, bool normalized)
{
    switch (ct) {
    case 5120: { const float v = static_cast<float>(static_cast<int8_t>(*p)); return normalized ? std::max(v / 127.0f, -1.0f) : v; }
    case 5121: return normalized ? static_cast<float>(*p) / 255.0f : static_cast<float>(*p);
    case 5122: { int16_t v; std::memcpy(&v, p, 2); return normalized ? std::max(static_cast<float>(v) / 32767.0f, -1.0f) : static_cast<float>(v); }
    case 5123: { uint16_t v; std::memcpy(&v, p, 2); return normalized ? static_cast<float>(v) / 65535.0f : static_cast<float>(v); }
    case 5125: { uint32_t v; std::memcpy(&v, p, 4); return static_cast<float>(v); }
    case 5126: { float v; std::memcpy(&v, p, 4); return v; }
    default: return 0.0f;
    }
}

uint32_t readIndex(const uint8_t* p, int ct)
{
    switch (ct) {
    case 5121: return *p;
    case 5123: { uint16_t v; std::memcpy(&v, p, 2); return v; }
    case 5125: { uint32_t v; std::memcpy(&v, p, 4); return v; }
    default: return 0;
    }
}

bool accessorData(const Model& M, int ai, const uint8_t*& ptr, size_t& stride, size_t& count, const Accessor** out)
{
    if (ai < 0 || ai >= static_cast<int>(M.accessors.size())) return false;
    const Accessor& a = M.accessors[static_cast<size_t>(ai)];
    if (a.bufferView < 0 || a.bufferView >= static_cast<int>(M.views.size())) return false;
    const View& v = M.views[static_cast<size_t>(a.bufferView)];
    if (v.buffer < 0 || v.buffer >= static_cast<int>(M.buffers.size())) return false;
    const auto& buf = M.buffers[static_cast<size_t>(v.buffer)];
    const int cs = compSize(a.componentType);
    if (a.comps <= 0 || cs <= 0 || a.count < 0) return false;
    const size_t elem = static_cast<size_t>(a.comps * cs);
    stride = v.byteStride > 0 ? v.byteStride : elem;
    const size_t off = v.byteOffset + a.byteOffset;
    if (off + (a.count ? (static_cast<size_t>(a.count) - 1) * stride + elem : 0) > buf.size()) return false;
    ptr = buf.data() + off;
    count = static_cast<size_t>(a.count);
    if (out) *out = &a;
    return true;
}

std::vector<V3> readVec3(const Model& M, int ai)
{
    std::vector<V3> o;
    const uint8_t* p = nullptr;
    size_t st = 0, n = 0;
    const Accessor* a = nullptr;
    if (!accessorData(M, ai, p, st, n, &a) || a->comps < 3) return o;
    const int cs = compSize(a->componentType);
    o.resize(n);
    for (size_t i = 0; i < n; ++i) {
        const uint8_t* e = p + i * st;
        o[i] = {readFloat(e, a->componentType, a->normalized), readFloat(e + cs, a->componentType, a->normalized),
                readFloat(e + 2 * cs, a->componentType, a->normalized)};
    }
    return o;
}

std::vector<Float2> readVec2(const Model& M, int ai)
{
    std::vector<Float2> o;
    const uint8_t* p = nullptr;
    size_t st = 0, n = 0;
    const Accessor* a = nullptr;
    if (!accessorData(M, ai, p, st, n, &a) || a->comps < 2) return o;
    const int cs = compSize(a->componentType);
    o.resize(n);
    for (size_t i = 0; i < n; ++i) {
        const uint8_t* e = p + i * st;
        o[i] = {readFloat(e, a->componentType, a->normalized), readFloat(e + cs, a->componentType, a->normalized)};
    }
    return o;
}

std::vector<uint32_t> readIndices(const Model& M, int ai, size_t vertexCount)
{
    std::vector<uint32_t> o;
    if (ai < 0) {
        o.resize(vertexCount);
        for (size_t i = 0; i < vertexCount; ++i) o[i] = static_cast<uint32_t>(i);
        return o;
    }
    const uint8_t* p = nullptr;
    size_t st = 0, n = 0;
    const Accessor* a = nullptr;
    if (!accessorData(M, ai, p, st, n, &a)) return o;
    o.resize(n);
    for (size_t i = 0; i < n; ++i) o[i] = readIndex(p + i * st, a->componentType);
    return o;
}

std::vector<uint32_t> triangulate(const std::vector<uint32_t>& ix, int mode)
{
    std::vector<uint32_t> t;
    if (mode == 4) {
        t.assign(ix.begin(), ix.begin() + static_cast<std::ptrdiff_t>(ix.size() - ix.size() % 3));
    } else if (mode == 6 && ix.size() >= 3) {   // fan
        for (size_t i = 1; i + 1 < ix.size(); ++i) { t.push_back(ix[0]); t.push_back(ix[i]); t.push_back(ix[i + 1]); }
    } else if (mode == 5 && ix.size() >= 3) {   // strip, alternate triangles reversed
        for (size_t i = 0; i + 2 < ix.size(); ++i) {
            if (i % 2 == 0) { t.push_back(ix[i]); t.push_back(ix[i + 1]); }
            else { t.push_back(ix[i + 1]); t.push_back(ix[i]); }
            t.push_back(ix[i + 2]);
        }
    }
    return t;
}

// ---------------------------------------------------------------- materials (gltf_loader.cpp:311-481)
double extNumber(const Json* ext, const char* key, double fallback)
{
    if (!ext || ext->kind != Json::Object) return fallback;
    const Json* v = ext->get(key);
    return (v && v->kind == Json::Number) ? v->num : fallback;
}

GltfSlot disneyFromMaterial(const Json& mat, const Model& M)
{
    GltfSlot slot{};
    const Json* pbr = mat.get("pbrMetallicRoughness");
    static const Json empty;
    if (!pbr || pbr->kind != Json::Object) pbr = &empty;
    float base[4] = {1.0f, 1.0f, 1.0f, 1.0f};
    const std::vector<double> bcf = pbr->numbers("baseColorFactor");
    if (pbr->get("baseColorFactor") && bcf.size() >= 3) {
        base[0] = static_cast<float>(bcf[0]); base[1] = static_cast<float>(bcf[1]); base[2] = static_cast<float>(bcf[2]);
        base[3] = bcf.size() >= 4 ? static_cast<float>(bcf[3]) : 1.0f;
    }
    const float metallic = static_cast<float>(pbr->numOr("metallicFactor", 1.0));
    const float roughness = static_cast<float>(pbr->numOr("roughnessFactor", 1.0));
    auto texImage = [&](const char* key, int& texCoord) -> Image {
        texCoord = 0;
        const Json* ti = pbr->get(key);
        const int index = ti ? ti->intOr("index", -1) : -1;
        if (ti) texCoord = ti->intOr("texCoord", 0);
        if (index < 0 || index >= static_cast<int>(M.textureSource.size())) return {};
        const int src = M.textureSource[static_cast<size_t>(index)];
        if (src < 0 || src >= static_cast<int>(M.images.size())) return {};
        return M.images[static_cast<size_t>(src)];
    };
    int tc = 0, tcMr = 0;
    Image albedo = texImage("baseColorTexture", tc);
    if (!albedo.pixels.empty()) {   // factor baked into the texture
        const size_t np = static_cast<size_t>(albedo.width) * albedo.height;
        for (size_t i = 0; i < np; ++i)
            for (int c = 0; c < 4; ++c)
                albedo.pixels[i * 4 + c] = static_cast<uint8_t>(
                    std::clamp((albedo.pixels[i * 4 + c] / 255.0f) * base[c] * 255.0f + 0.5f, 0.0f, 255.0f));
    }
    Image mr = texImage("metallicRoughnessTexture", tcMr);
    float specular = 0.5f, transmission = 0.0f, specularTint = 0.0f, sheen = 0.0f, sheenTint = 0.5f, subsurface = 0.0f,
          anisotropic = 0.0f, clearcoat = 0.0f, clearcoatGloss = 1.0f, eta = 1.5f;
    const Json* exts = mat.get("extensions");
    auto ext = [&](const char* name) -> const Json* { return exts ? exts->get(name) : nullptr; };
    if (const Json* e = ext("KHR_materials_ior")) eta = static_cast<float>(extNumber(e, "ior", eta));
    if (const Json* e = ext("KHR_materials_transmission"))
        transmission = static_cast<float>(extNumber(e, "transmissionFactor", 0.0));
    if (const Json* e = ext("KHR_materials_clearcoat")) {
        clearcoat = static_cast<float>(extNumber(e, "clearcoatFactor", 0.0));
        clearcoatGloss = 1.0f - static_cast<float>(extNumber(e, "clearcoatRoughnessFactor", 0.0));
    }
    if (const Json* e = ext("KHR_materials_sheen")) {
        const Json* sc = e->get("sheenColorFactor");
        if (e->kind == Json::Object && sc && sc->kind == Json::Array && sc->arr.size() >= 3) {
            auto num = [](const Json& v) { return v.kind == Json::Number ? v.num : 0.0; };
            const float r = static_cast<float>(num(sc->arr[0])), g = static_cast<float>(num(sc->arr[1])),
                        b = static_cast<float>(num(sc->arr[2]));
            sheen = 0.2126f * r + 0.7152f * g + 0.0722f * b;
            sheenTint = 1.0f;
        }
    }
    float em[3] = {0.0f, 0.0f, 0.0f};
    const std::vector<double> ef = mat.numbers("emissiveFactor");
    if (ef.size() >= 3) { em[0] = static_cast<float>(ef[0]); em[1] = static_cast<float>(ef[1]); em[2] = static_cast<float>(ef[2]); }
    if (const Json* e = ext("KHR_materials_emissive_strength")) {
        const float s = static_cast<float>(extNumber(e, "emissiveStrength", 1.0));
        em[0] *= s; em[1] *= s; em[2] *= s;
    }
    slot.emission = {em[0], em[1], em[2]};
    slot.isEmitter = (em[0] + em[1] + em[2]) > 1e-4f;
    const bool unlit = ext("KHR_materials_unlit") != nullptr;
    const float outMetallic = unlit ? 0.0f : metallic, outRoughness = unlit ? 1.0f : roughness;
    const float col[3] = {albedo.pixels.empty() ? base[0] : 1.0f, albedo.pixels.empty() ? base[1] : 1.0f,
                          albedo.pixels.empty() ? base[2] : 1.0f};
    BsdfData d{};
    d.type = BSDF_Disney;
    d.p0 = {col[0], col[1], col[2], outRoughness};
    d.p1 = {outMetallic, specular, transmission, specularTint};
    d.p2 = {sheen, sheenTint, subsurface, anisotropic};
    d.p3 = {clearcoat, clearcoatGloss, eta, 0.0f};
    slot.bsdf = d;
    slot.albedo = std::move(albedo.pixels);
    slot.albedoWidth = albedo.width;
    slot.albedoHeight = albedo.height;
    slot.mr = std::move(mr.pixels);
    slot.mrWidth = mr.width;
    slot.mrHeight = mr.height;
    return slot;
}

GltfSlot defaultSlot()
{
    GltfSlot s{};
    s.bsdf.type = BSDF_Disney;
    s.bsdf.p0 = {0.8f, 0.8f, 0.8f, 0.5f};
    s.bsdf.p1 = {0.0f, 0.5f, 0.0f, 0.0f};
    s.bsdf.p2 = {0.0f, 0.5f, 0.0f, 0.0f};
    s.bsdf.p3 = {0.0f, 1.0f, 1.5f, 0.0f};
    return s;
}

// ---------------------------------------------------------------- nodes (gltf_loader.cpp:37-82, 568-766)
M4 nodeMatrix(const Node& n)
{
    if (n.matrix.size() == 16) {
        M4 m;
        for (int j = 0; j < 4; ++j)
            m.c[j] = {static_cast<float>(n.matrix[4 * j]), static_cast<float>(n.matrix[4 * j + 1]),
                      static_cast<float>(n.matrix[4 * j + 2]), static_cast<float>(n.matrix[4 * j + 3])};
        return m;
    }
    M4 T = identity(), R = identity(), S = identity();
    if (n.t.size() == 3) T = translate(identity(), static_cast<float>(n.t[0]), static_cast<float>(n.t[1]), static_cast<float>(n.t[2]));
    if (n.r.size() == 4)
        R = quatToMat(static_cast<float>(n.r[3]), static_cast<float>(n.r[0]), static_cast<float>(n.r[1]), static_cast<float>(n.r[2]));
    if (n.s.size() == 3) S = scale(identity(), static_cast<float>(n.s[0]), static_cast<float>(n.s[1]), static_cast<float>(n.s[2]));
    return mul(mul(T, R), S);
}

M4 xmlMatrix(float px, float py, float pz, float rx, float ry, float rz, float sx, float sy, float sz)
{
    const float d2r = 3.14159265358979323846f / 180.0f;
    M4 m = translate(identity(), px, py, pz);
    m = rotate(m, rz * d2r, 0.0f, 0.0f, 1.0f);
    m = rotate(m, ry * d2r, 0.0f, 1.0f, 0.0f);
    m = rotate(m, rx * d2r, 1.0f, 0.0f, 0.0f);
    return scale(m, sx, sy, sz);
}

std::string lower(std::string s)
{
    for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return s;
}

bool skipNode(const Node& n)
{
    const std::string l = lower(n.name);
    return l == "background" || l.find("backgroundgradient") != std::string::npos;
}

bool skipPrim(const Model& M, const Prim& p)
{
    if (p.material < 0 || p.material >= static_cast<int>(M.materials.size())) return false;
    const std::string l = lower(M.materials[static_cast<size_t>(p.material)]->strOr("name"));
    return l.find("outline") != std::string::npos || l == "backgroundgradient";
}

uint64_t primKey(int node, int prim) { return (static_cast<uint64_t>(static_cast<uint32_t>(node)) << 32) | static_cast<uint32_t>(prim); }

struct PrimStat { uint64_t key; V3 center; float extent; };

bool primBounds(const Model& M, const Prim& p, const M4& world, V3& center, float& extent)
{
    const auto it = p.attributes.find("POSITION");
    if (it == p.attributes.end()) return false;
    if (it->second < 0 || it->second >= static_cast<int>(M.accessors.size())) return false;
    const Accessor& a = M.accessors[static_cast<size_t>(it->second)];
    if (a.mn.size() < 3 || a.mx.size() < 3) return false;
    const float lo[3] = {static_cast<float>(a.mn[0]), static_cast<float>(a.mn[1]), static_cast<float>(a.mn[2])};
    const float hi[3] = {static_cast<float>(a.mx[0]), static_cast<float>(a.mx[1]), static_cast<float>(a.mx[2])};
    V3 wmin = {1e30f, 1e30f, 1e30f}, wmax = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < 8; ++i) {
        const V4 w = mulv(world, {(i & 1) ? hi[0] : lo[0], (i & 2) ? hi[1] : lo[1], (i & 4) ? hi[2] : lo[2], 1.0f});
        wmin = {w.x < wmin.x ? w.x : wmin.x, w.y < wmin.y ? w.y : wmin.y, w.z < wmin.z ? w.z : wmin.z};
        wmax = {wmax.x < w.x ? w.x : wmax.x, wmax.y < w.y ? w.y : wmax.y, wmax.z < w.z ? w.z : wmax.z};
    }
    center = {0.5f * (wmin.x + wmax.x), 0.5f * (wmin.y + wmax.y), 0.5f * (wmin.z + wmax.z)};
    const V3 sz = {wmax.x - wmin.x, wmax.y - wmin.y, wmax.z - wmin.z};
    extent = std::max(sz.x, std::max(sz.y, sz.z));
    return extent > 0.0f;
}

void gatherStats(const Model& M, int ni, const M4& parent, std::vector<PrimStat>& stats, int depth)
{
    if (ni < 0 || ni >= static_cast<int>(M.nodes.size())) return;
    if (depth > 256) gfail("node graph deeper than 256 levels (a cycle?)");
    const Node& n = M.nodes[static_cast<size_t>(ni)];
    if (skipNode(n)) return;
    const M4 world = mul(parent, nodeMatrix(n));
    if (n.mesh >= 0 && n.mesh < static_cast<int>(M.meshes.size())) {
        const auto& prims = M.meshes[static_cast<size_t>(n.mesh)];
        for (int pi = 0; pi < static_cast<int>(prims.size()); ++pi) {
            if (skipPrim(M, prims[static_cast<size_t>(pi)])) continue;
            PrimStat s{primKey(ni, pi), {0, 0, 0}, 0.0f};
            if (primBounds(M, prims[static_cast<size_t>(pi)], world, s.center, s.extent)) stats.push_back(s);
        }
    }
    for (int c : n.children) gatherStats(M, c, world, stats, depth + 1);
}

// upper median: the element nth_element places at n/2
float median(std::vector<float> v)
{
    std::nth_element(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(v.size() / 2), v.end());
    return v[v.size() / 2];
}

std::set<uint64_t> outliers(const std::vector<PrimStat>& st)
{
    std::set<uint64_t> skip;
    if (st.size() < 4) return skip;
    std::vector<float> ex, cx, cy, cz;
    for (const auto& s : st) { ex.push_back(s.extent); cx.push_back(s.center.x); cy.push_back(s.center.y); cz.push_back(s.center.z); }
    const float me = median(ex);
    const V3 mc = {median(cx), median(cy), median(cz)};
    if (me <= 1e-8f) return skip;
    const float maxExtent = 12.0f * me, maxDist = 10.0f * me;
    for (const auto& s : st) {
        const float dx = s.center.x - mc.x, dy = s.center.y - mc.y, dz = s.center.z - mc.z;
        if (s.extent > maxExtent || std::sqrt(dx * dx + dy * dy + dz * dz) > maxDist) skip.insert(s.key);
    }
    return skip;
}

Float3 faceNormal(const Float3& a, const Float3& b, const Float3& c)
{
    const float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
    const float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
    Float3 n = {e1y * e2z - e1z * e2y, e1z * e2x - e1x * e2z, e1x * e2y - e1y * e2x};
    const float len = std::sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
    if (len > 1e-20f) { n.x /= len; n.y /= len; n.z /= len; }
    return n;
}

void emitPrim(const Model& M, const Prim& p, const M4& world, int slot, GltfResult& R)
{
    const auto pit = p.attributes.find("POSITION");
    if (pit == p.attributes.end()) return;
    const std::vector<V3> pos = readVec3(M, pit->second);
    if (pos.empty()) return;
    std::vector<V3> nrm;
    const auto nit = p.attributes.find("NORMAL");
    if (nit != p.attributes.end()) nrm = readVec3(M, nit->second);
    std::vector<Float2> uv;
    const auto uit = p.attributes.find("TEXCOORD_0");
    if (uit != p.attributes.end()) uv = readVec2(M, uit->second);
    std::vector<uint32_t> ix = readIndices(M, p.indices, pos.size());
    const int mode = p.mode < 0 ? 4 : p.mode;
    if (mode != 4 && mode != 5 && mode != 6) return;   // points and lines are skipped
    ix = triangulate(ix, mode);
    const M3 nm = normalMatrix(world);
    auto xp = [&](const V3& v) -> Float3 { const V4 w = mulv(world, {v.x, v.y, v.z, 1.0f}); return {w.x, w.y, w.z}; };
    for (size_t i = 0; i + 2 < ix.size(); i += 3) {
        const uint32_t a = ix[i], b = ix[i + 1], c = ix[i + 2];
        if (a >= pos.size() || b >= pos.size() || c >= pos.size()) continue;
        TriangleData t{};
        t.v0 = xp(pos[a]); t.v1 = xp(pos[b]); t.v2 = xp(pos[c]);
        if (a < nrm.size() && b < nrm.size() && c < nrm.size()) {
            t.n0 = normalXform(nm, nrm[a].x, nrm[a].y, nrm[a].z);
            t.n1 = normalXform(nm, nrm[b].x, nrm[b].y, nrm[b].z);
            t.n2 = normalXform(nm, nrm[c].x, nrm[c].y, nrm[c].z);
        } else {
            t.n0 = t.n1 = t.n2 = faceNormal(t.v0, t.v1, t.v2);
        }
        auto uvAt = [&](uint32_t k) -> Float2 { return k < uv.size() ? uv[k] : Float2{0.0f, 0.0f}; };
        t.uv0 = uvAt(a); t.uv1 = uvAt(b); t.uv2 = uvAt(c);
        R.triangles.push_back(t);
        R.materialIds.push_back(slot);
    }
}

void walk(const Model& M, int ni, const M4& parent, const std::vector<int>& matToSlot, int defSlot,
          const std::set<uint64_t>& skip, GltfResult& R, int depth)
{
    if (ni < 0 || ni >= static_cast<int>(M.nodes.size())) return;
    if (depth > 256) gfail("node graph deeper than 256 levels (a cycle?)");
    const Node& n = M.nodes[static_cast<size_t>(ni)];
    if (skipNode(n)) return;
    const M4 world = mul(parent, nodeMatrix(n));
    if (n.mesh >= 0 && n.mesh < static_cast<int>(M.meshes.size())) {
        const auto& prims = M.meshes[static_cast<size_t>(n.mesh)];
        for (int pi = 0; pi < static_cast<int>(prims.size()); ++pi) {
            const Prim& p = prims[static_cast<size_t>(pi)];
            if (skipPrim(M, p) || skip.count(primKey(ni, pi))) continue;
            int slot = defSlot;
            if (p.material >= 0 && p.material < static_cast<int>(matToSlot.size())) slot = matToSlot[static_cast<size_t>(p.material)];
            emitPrim(M, p, world, slot, R);
        }
    }
    for (int c : n.children) walk(M, c, world, matToSlot, defSlot, skip, R, depth + 1);
}

}  // namespace

bool loadGltf(const std::string& path, const float xf[9], GltfResult& R, std::string& err)
{
    try {
        R = GltfResult{};
        const Model M = parseModel(path);
        std::vector<int> matToSlot(M.materials.size(), 0);
        for (size_t i = 0; i < M.materials.size(); ++i) {
            matToSlot[i] = static_cast<int>(R.materials.size());
            R.materials.push_back(disneyFromMaterial(*M.materials[i], M));
        }
        const int defSlot = static_cast<int>(R.materials.size());
        R.materials.push_back(defaultSlot());
        const M4 xm = xmlMatrix(xf[0], xf[1], xf[2], xf[3], xf[4], xf[5], xf[6], xf[7], xf[8]);
        std::vector<PrimStat> stats;
        for (int r : M.roots) gatherStats(M, r, xm, stats, 0);
        const std::set<uint64_t> skip = outliers(stats);
        for (int r : M.roots) walk(M, r, xm, matToSlot, defSlot, skip, R, 0);
        if (!R.materialIds.empty() && std::find(R.materialIds.begin(), R.materialIds.end(), defSlot) == R.materialIds.end() &&
            defSlot == static_cast<int>(R.materials.size()) - 1)
            R.materials.pop_back();
        if (R.triangles.empty()) gfail("no triangles in \"" + path + "\"");
        R.skippedOutliers = static_cast<int>(skip.size());
        return true;
    } catch (const GltfError& e) {
        err = e.msg;
    } catch (const std::bad_alloc&) {
        err = "out of memory reading \"" + path + "\"";
    }
    return false;
}

}  // namespace bte

// ---------------------------------------------------------------- C-ABI (loadGltfModel, gltf_loader.h:25-30)
struct BteGltf {
    bte::GltfResult r;
};

extern "C" {

int bte_gltf_load(const char* path, const float* xf9, BteGltf** out)
{
    if (!path || !out) { bte::setError("bte_gltf_load: null argument"); return -1; }
    *out = nullptr;
    static const float identityXf[9] = {0, 0, 0, 0, 0, 0, 1, 1, 1};
    BteGltf* g = new (std::nothrow) BteGltf();
    if (!g) { bte::setError("bte_gltf_load: out of memory"); return -1; }
    std::string err;
    if (!bte::loadGltf(path, xf9 ? xf9 : identityXf, g->r, err)) {
        delete g;
        bte::setError("bte_gltf_load: " + err);
        return -1;
    }
    *out = g;
    return 0;
}

int bte_gltf_counts(const BteGltf* g, int* triangles, int* materials, int* skippedOutliers)
{
    if (!g) { bte::setError("bte_gltf_counts: null model"); return -1; }
    if (triangles) *triangles = static_cast<int>(g->r.triangles.size());
    if (materials) *materials = static_cast<int>(g->r.materials.size());
    if (skippedOutliers) *skippedOutliers = g->r.skippedOutliers;
    return 0;
}

int bte_gltf_triangles(const BteGltf* g, TriangleData* triangles, int* materialIds)
{
    if (!g) { bte::setError("bte_gltf_triangles: null model"); return -1; }
    if (triangles) std::memcpy(triangles, g->r.triangles.data(), g->r.triangles.size() * sizeof(TriangleData));
    if (materialIds) std::memcpy(materialIds, g->r.materialIds.data(), g->r.materialIds.size() * sizeof(int));
    return 0;
}

int bte_gltf_material(const BteGltf* g, int index, BsdfData* bsdf, float* emission3, int* isEmitter, int* albedoWH,
                      int* mrWH, uint8_t* albedoRGBA, uint8_t* mrRGBA)
{
    if (!g || index < 0 || index >= static_cast<int>(g->r.materials.size())) {
        bte::setError("bte_gltf_material: bad model or index");
        return -1;
    }
    const bte::GltfSlot& s = g->r.materials[static_cast<size_t>(index)];
    if (bsdf) *bsdf = s.bsdf;
    if (emission3) { emission3[0] = s.emission.x; emission3[1] = s.emission.y; emission3[2] = s.emission.z; }
    if (isEmitter) *isEmitter = s.isEmitter ? 1 : 0;
    if (albedoWH) { albedoWH[0] = s.albedo.empty() ? 0 : s.albedoWidth; albedoWH[1] = s.albedo.empty() ? 0 : s.albedoHeight; }
    if (mrWH) { mrWH[0] = s.mr.empty() ? 0 : s.mrWidth; mrWH[1] = s.mr.empty() ? 0 : s.mrHeight; }
    if (albedoRGBA && !s.albedo.empty()) std::memcpy(albedoRGBA, s.albedo.data(), s.albedo.size());
    if (mrRGBA && !s.mr.empty()) std::memcpy(mrRGBA, s.mr.data(), s.mr.size());
    return 0;
}

void bte_gltf_free(BteGltf* g) { delete g; }

}  // extern "C"
