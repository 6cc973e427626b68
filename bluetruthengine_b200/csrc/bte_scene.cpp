// bte_scene.cpp -- scene.xml / OBJ / Radiance-HDR loader and scene flattening.
//
// Host-side front end of the renderer: turns a Nori-style scene.xml plus OBJ
// meshes into the flattened arrays the bte_init_* entry points take, with the
// semantics of the reference's loader:
//   scene.xml parsing        src/scene.cpp:9-523 (string search, first match,
//                            std::stof for attributes, same required fields)
//   OBJ -> TriangleData      src/main.cpp:267-401 (normal fallback, planar UV
//                            when the file has <= 1 texcoord)
//   transforms               include/mesh_transform.h:9-80
//   BSDF packing             src/main.cpp:629-665
//   emitter tables           src/main.cpp:670-758 (area CDF per emitter,
//                            power CDF lum*area over emitters)
//   spotlights               src/main.cpp:879-904
//   camera basis             src/main.cpp:533-564 (GLM normalize/cross)
//   env map (.hdr)           src/main.cpp:906-930 with stb_image's Radiance
//                            decoding (flat or RLE scanlines, RGBE -> float)
// OBJ numbers are parsed to double and rounded to float (as the reference's
// OBJ parser does); XML attributes with strtof (as std::stof).
// Errors are reported through a status code instead of std::exit.
#include "bte_internal.h"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

namespace bte {

namespace {

struct TransformDesc {
    float posX = 0, posY = 0, posZ = 0;
    float rotX = 0, rotY = 0, rotZ = 0;
    float scaleX = 1, scaleY = 1, scaleZ = 1;
};
struct MeshDesc {
    std::string filename, materialName;
    bool isEmitter = false;
    float radianceR = 0, radianceG = 0, radianceB = 0;
    TransformDesc transform;
};
struct MaterialDesc { std::string name, albedoTexture, bsdfName; };
struct BsdfDesc {
    std::string name, type;
    float albedoR = 1, albedoG = 1, albedoB = 1;
    float intIOR = 1.5f, extIOR = 1.0f;
    float alpha = 0.1f;
    float baseColorR = 0.5f, baseColorG = 0.5f, baseColorB = 0.5f;
    float roughness = 0.1f, metallic = 0, specular = 0.5f, specularTransmission = 0, specularTint = 0;
    float sheen = 0, sheenTint = 0.5f, subsurface = 0, anisotropic = 0, clearcoat = 0, clearcoatGloss = 1, eta = 1.5f;
};
struct SpotDesc {
    float posX = 0, posY = 0, posZ = 0, dirX = 0, dirY = -1, dirZ = 0;
    float radianceR = 1, radianceG = 1, radianceB = 1, intensity = 1, innerConeAngle = 0, outerConeAngle = 180;
};
struct CameraDesc {
    float eyeX = 0, eyeY = 0, eyeZ = 0, lookAtX = 0, lookAtY = 0, lookAtZ = 0, upX = 0, upY = 1, upZ = 0, fovY = 45;
};
struct ModelDesc {
    std::string filename;
    TransformDesc transform;
};
struct SceneDesc {
    std::vector<MeshDesc> meshes;
    std::vector<ModelDesc> models;
    std::vector<MaterialDesc> materials;
    std::vector<BsdfDesc> bsdfs;
    std::vector<SpotDesc> spots;
    CameraDesc camera;
    int width = 1280, height = 720;
    std::string envPath;
    float envIntensity = 1.0f, envRotation = 0.0f;
};

struct LoadError {
    std::string msg;
};

[[noreturn]] void fail(const std::string& m) { throw LoadError{m}; }

std::string readFile(const std::string& path)
{
    std::ifstream ifs(path, std::ios::in | std::ios::binary);
    if (!ifs) return {};
    std::ostringstream ss;
    ss << ifs.rdbuf();
    return ss.str();
}

// "<tag ... >" content (without the closing '>') after `from`; advances `from`.
bool nextTag(const std::string& src, const std::string& tag, size_t& from, std::string& out)
{
    const std::string open = "<" + tag;
    const size_t p = src.find(open, from);
    if (p == std::string::npos) return false;
    const size_t e = src.find('>', p);
    if (e == std::string::npos) return false;
    out = src.substr(p, e - p);
    from = e + 1;
    return true;
}

// attribute value `name="..."` inside a tag's content; empty when absent.
std::string attr(const std::string& tagContent, const std::string& name)
{
    const std::string key = name + "=\"";
    size_t p = tagContent.find(key);
    if (p == std::string::npos) return {};
    p += key.size();
    const size_t q = tagContent.find('"', p);
    if (q == std::string::npos) return {};
    return tagContent.substr(p, q - p);
}

// attribute of the first `<tag` at or after `from` (src/scene.cpp:25-52 semantics)
std::string firstTagAttr(const std::string& src, const std::string& tag, const std::string& name, size_t from = 0,
                         size_t* tagEnd = nullptr)
{
    const std::string open = "<" + tag;
    const size_t p = src.find(open, from);
    if (p == std::string::npos) return {};
    const size_t e = src.find('>', p);
    if (e == std::string::npos) return {};
    if (tagEnd) *tagEnd = e;
    return attr(src.substr(p, e - p), name);
}

float parseFloatStrict(const std::string& s, const std::string& where)
{
    // std::stof: leading whitespace skipped, trailing garbage ignored, throws when nothing parses
    const char* b = s.c_str();
    char* end = nullptr;
    errno = 0;
    const float v = std::strtof(b, &end);
    if (end == b) fail(where + ": invalid float \"" + s + "\"");
    if (errno == ERANGE) fail(where + ": float out of range \"" + s + "\"");
    return v;
}

void readOpt(const std::string& tag, const char* name, float& out, const std::string& where)
{
    const std::string v = attr(tag, name);
    if (v.empty()) return;
    out = parseFloatStrict(v, where + " attribute `" + name + "`");
}

SceneDesc parseScene(const std::string& path)
{
    SceneDesc d;
    const std::string xml = readFile(path);
    if (xml.empty()) fail("scene file \"" + path + "\" is empty or unreadable");

    {   // <bsdf>
        size_t from = 0;
        std::string t;
        while (nextTag(xml, "bsdf", from, t)) {
            BsdfDesc b;
            b.name = attr(t, "name");
            b.type = attr(t, "type");
            if (b.name.empty() || b.type.empty()) fail("<bsdf> missing required `name` and/or `type`");
            const std::string w = "<bsdf name=\"" + b.name + "\">";
            if (b.type == "diffuse" || b.type == "mirror") {
                readOpt(t, "albedoR", b.albedoR, w); readOpt(t, "albedoG", b.albedoG, w); readOpt(t, "albedoB", b.albedoB, w);
            } else if (b.type == "dielectric") {
                readOpt(t, "intIOR", b.intIOR, w); readOpt(t, "extIOR", b.extIOR, w);
            } else if (b.type == "microfacet") {
                readOpt(t, "albedoR", b.albedoR, w); readOpt(t, "albedoG", b.albedoG, w); readOpt(t, "albedoB", b.albedoB, w);
                readOpt(t, "alpha", b.alpha, w); readOpt(t, "intIOR", b.intIOR, w); readOpt(t, "extIOR", b.extIOR, w);
            } else if (b.type == "disney") {
                readOpt(t, "base_colorR", b.baseColorR, w); readOpt(t, "base_colorG", b.baseColorG, w);
                readOpt(t, "base_colorB", b.baseColorB, w); readOpt(t, "roughness", b.roughness, w);
                readOpt(t, "metallic", b.metallic, w); readOpt(t, "specular", b.specular, w);
                readOpt(t, "specular_transmission", b.specularTransmission, w);
                readOpt(t, "specular_tint", b.specularTint, w); readOpt(t, "sheen", b.sheen, w);
                readOpt(t, "sheen_tint", b.sheenTint, w); readOpt(t, "subsurface", b.subsurface, w);
                readOpt(t, "anisotropic", b.anisotropic, w); readOpt(t, "clearcoat", b.clearcoat, w);
                readOpt(t, "clearcoat_gloss", b.clearcoatGloss, w); readOpt(t, "eta", b.eta, w);
            } else {
                fail(w + " unsupported type \"" + b.type + "\" (expected diffuse|dielectric|mirror|microfacet|disney)");
            }
            d.bsdfs.push_back(b);
        }
    }
    {   // <material>
        size_t from = 0;
        std::string t;
        while (nextTag(xml, "material", from, t)) {
            MaterialDesc m;
            m.name = attr(t, "name");
            m.albedoTexture = attr(t, "albedoTexture");
            m.bsdfName = attr(t, "bsdf");
            if (m.name.empty()) fail("<material> missing required attribute `name`");
            if (m.bsdfName.empty()) fail("<material> \"" + m.name + "\" missing required attribute `bsdf`");
            d.materials.push_back(m);
        }
    }
    {   // <mesh>
        size_t from = 0;
        std::string t;
        while (nextTag(xml, "mesh", from, t)) {
            MeshDesc m;
            m.filename = attr(t, "filename");
            m.materialName = attr(t, "material");
            const std::string w = "<mesh filename=\"" + m.filename + "\">";
            const std::string isEm = attr(t, "isEmitter");
            if (!isEm.empty()) {
                if (isEm == "1" || isEm == "true" || isEm == "True") m.isEmitter = true;
                else if (isEm == "0" || isEm == "false" || isEm == "False") m.isEmitter = false;
                else fail(w + " invalid bool attribute `isEmitter`: \"" + isEm + "\"");
            }
            readOpt(t, "radianceR", m.radianceR, w); readOpt(t, "radianceG", m.radianceG, w);
            readOpt(t, "radianceB", m.radianceB, w);
            if (m.isEmitter && m.radianceR == 0.0f && m.radianceG == 0.0f && m.radianceB == 0.0f)
                m.radianceR = m.radianceG = m.radianceB = 10.0f;
            TransformDesc& x = m.transform;
            readOpt(t, "posX", x.posX, w); readOpt(t, "posY", x.posY, w); readOpt(t, "posZ", x.posZ, w);
            readOpt(t, "rotX", x.rotX, w); readOpt(t, "rotY", x.rotY, w); readOpt(t, "rotZ", x.rotZ, w);
            readOpt(t, "scaleX", x.scaleX, w); readOpt(t, "scaleY", x.scaleY, w); readOpt(t, "scaleZ", x.scaleZ, w);
            if (m.filename.empty()) fail("<mesh> missing required attribute `filename`");
            if (m.materialName.empty()) fail(w + " missing required attribute `material`");
            d.meshes.push_back(m);
        }
    }
    {   // <model> (glTF / GLB drop-ins), src/scene.cpp:274-317
        size_t from = 0;
        std::string t;
        while (nextTag(xml, "model", from, t)) {
            ModelDesc m;
            m.filename = attr(t, "filename");
            const std::string w = "<model filename=\"" + m.filename + "\">";
            TransformDesc& x = m.transform;
            readOpt(t, "posX", x.posX, w); readOpt(t, "posY", x.posY, w); readOpt(t, "posZ", x.posZ, w);
            readOpt(t, "rotX", x.rotX, w); readOpt(t, "rotY", x.rotY, w); readOpt(t, "rotZ", x.rotZ, w);
            readOpt(t, "scaleX", x.scaleX, w); readOpt(t, "scaleY", x.scaleY, w); readOpt(t, "scaleZ", x.scaleZ, w);
            if (m.filename.empty()) fail("<model> missing required attribute `filename`");
            d.models.push_back(m);
        }
    }
    for (const auto& mesh : d.meshes) {
        bool ok = false;
        for (const auto& m : d.materials) ok = ok || (m.name == mesh.materialName);
        if (!ok) fail("mesh material reference \"" + mesh.materialName + "\" not found in <material> entries");
    }
    for (const auto& mat : d.materials) {
        bool ok = false;
        for (const auto& b : d.bsdfs) ok = ok || (b.name == mat.bsdfName);
        if (!ok) fail("material bsdf reference \"" + mat.bsdfName + "\" not found in <bsdf> entries");
    }
    {   // <spotlight>
        size_t from = 0;
        std::string t;
        while (nextTag(xml, "spotlight", from, t)) {
            SpotDesc s;
            const std::string w = "<spotlight>";
            readOpt(t, "posX", s.posX, w); readOpt(t, "posY", s.posY, w); readOpt(t, "posZ", s.posZ, w);
            readOpt(t, "dirX", s.dirX, w); readOpt(t, "dirY", s.dirY, w); readOpt(t, "dirZ", s.dirZ, w);
            readOpt(t, "radianceR", s.radianceR, w); readOpt(t, "radianceG", s.radianceG, w);
            readOpt(t, "radianceB", s.radianceB, w); readOpt(t, "intensity", s.intensity, w);
            readOpt(t, "innerConeAngle", s.innerConeAngle, w); readOpt(t, "outerConeAngle", s.outerConeAngle, w);
            d.spots.push_back(s);
        }
    }
    {   // <environment>
        size_t from = 0;
        std::string t;
        if (nextTag(xml, "environment", from, t)) {
            d.envPath = attr(t, "map");
            if (d.envPath.empty()) fail("<environment> tag found but missing required `map` attribute");
            readOpt(t, "intensity", d.envIntensity, "<environment>");
            readOpt(t, "rotation", d.envRotation, "<environment>");
        }
    }
    {   // <window>
        const std::string w = firstTagAttr(xml, "window", "width");
        const std::string h = firstTagAttr(xml, "window", "height");
        if (w.empty() || h.empty()) fail("<window> missing required `width` and/or `height`");
        char* e = nullptr;
        long v = std::strtol(w.c_str(), &e, 10);
        if (e != w.c_str()) d.width = static_cast<int>(v);
        v = std::strtol(h.c_str(), &e, 10);
        if (e != h.c_str()) d.height = static_cast<int>(v);
    }
    {   // <camera>
        size_t from = 0;
        std::string t;
        if (!nextTag(xml, "camera", from, t)) fail("no <camera ...> tag found in \"" + path + "\"");
        auto req = [&](const char* n) {
            const std::string v = attr(t, n);
            if (v.empty()) fail(std::string("<camera> missing required attribute `") + n + "`");
            return parseFloatStrict(v, std::string("<camera> `") + n + "`");
        };
        CameraDesc& c = d.camera;
        c.eyeX = req("eyeX"); c.eyeY = req("eyeY"); c.eyeZ = req("eyeZ");
        c.lookAtX = req("lookAtX"); c.lookAtY = req("lookAtY"); c.lookAtZ = req("lookAtZ");
        c.upX = req("upX"); c.upY = req("upY"); c.upZ = req("upZ");
        c.fovY = req("fovY");
    }
    if (d.meshes.empty() && d.models.empty()) fail("no <mesh> or <model> elements found in \"" + path + "\"");
    if (!d.meshes.empty() && d.materials.empty()) fail("no <material ...> elements found; OBJ <mesh> entries require materials");
    if (!d.meshes.empty() && d.bsdfs.empty()) fail("no <bsdf ...> elements found; OBJ <mesh> entries require BSDFs");
    return d;
}

// include/mesh_transform.h:9-80 (Scale -> Rx -> Ry -> Rz -> Translate, FP32 std::cos/std::sin)
Float3 xformPoint(const Float3& p, const TransformDesc& t)
{
    float x = p.x * t.scaleX, y = p.y * t.scaleY, z = p.z * t.scaleZ;
    const float d2r = 3.14159265358979323846f / 180.0f;
    const float rx = t.rotX * d2r, ry = t.rotY * d2r, rz = t.rotZ * d2r;
    { const float c = std::cos(rx), s = std::sin(rx); const float y2 = y * c - z * s, z2 = y * s + z * c; y = y2; z = z2; }
    { const float c = std::cos(ry), s = std::sin(ry); const float x2 = x * c + z * s, z2 = -x * s + z * c; x = x2; z = z2; }
    { const float c = std::cos(rz), s = std::sin(rz); const float x2 = x * c - y * s, y2 = x * s + y * c; x = x2; y = y2; }
    return {x + t.posX, y + t.posY, z + t.posZ};
}

Float3 xformNormal(const Float3& n, const TransformDesc& t)
{
    float x = n.x, y = n.y, z = n.z;
    const float d2r = 3.14159265358979323846f / 180.0f;
    const float rx = t.rotX * d2r, ry = t.rotY * d2r, rz = t.rotZ * d2r;
    { const float c = std::cos(rx), s = std::sin(rx); const float y2 = y * c - z * s, z2 = y * s + z * c; y = y2; z = z2; }
    { const float c = std::cos(ry), s = std::sin(ry); const float x2 = x * c + z * s, z2 = -x * s + z * c; x = x2; z = z2; }
    { const float c = std::cos(rz), s = std::sin(rz); const float x2 = x * c - y * s, y2 = x * s + y * c; x = x2; y = y2; }
    const float len = std::sqrt(x * x + y * y + z * z);
    if (len > 1e-8f) { x /= len; y /= len; z /= len; }
    return {x, y, z};
}

// ---- minimal OBJ reader (v / vn / vt / f; o, g, s, usemtl, mtllib ignored) ----
struct ObjIndex { int v, vt, vn; };
struct ObjData {
    std::vector<float> v, vn, vt;
    std::vector<ObjIndex> idx;   // triangulated
};

inline const char* skipWs(const char* p, const char* e) { while (p < e && (*p == ' ' || *p == '\t')) ++p; return p; }
inline const char* tokEnd(const char* p, const char* e) { while (p < e && *p != ' ' && *p != '\t' && *p != '\r') ++p; return p; }

float objReal(const char*& p, const char* e)
{
    p = skipWs(p, e);
    const char* q = tokEnd(p, e);
    double v = 0.0;
    if (q > p) {
        std::string tok(p, q);
        char* end = nullptr;
        v = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str()) v = 0.0;
    }
    p = q;
    return static_cast<float>(v);
}

int fixIndex(long i, size_t n)
{
    if (i > 0) return static_cast<int>(i - 1);
    if (i < 0) return static_cast<int>(static_cast<long>(n) + i);
    return -1;
}

ObjData readObj(const std::string& path)
{
    const std::string txt = readFile(path);
    if (txt.empty()) fail("failed to load OBJ: " + path);
    ObjData o;
    const char* p = txt.data();
    const char* end = p + txt.size();
    std::vector<ObjIndex> poly;
    while (p < end) {
        const char* le = static_cast<const char*>(std::memchr(p, '\n', static_cast<size_t>(end - p)));
        if (!le) le = end;
        const char* s = skipWs(p, le);
        if (s + 1 < le && s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            s += 2;
            o.v.push_back(objReal(s, le)); o.v.push_back(objReal(s, le)); o.v.push_back(objReal(s, le));
        } else if (s + 2 < le && s[0] == 'v' && s[1] == 'n' && (s[2] == ' ' || s[2] == '\t')) {
            s += 3;
            o.vn.push_back(objReal(s, le)); o.vn.push_back(objReal(s, le)); o.vn.push_back(objReal(s, le));
        } else if (s + 2 < le && s[0] == 'v' && s[1] == 't' && (s[2] == ' ' || s[2] == '\t')) {
            s += 3;
            o.vt.push_back(objReal(s, le)); o.vt.push_back(objReal(s, le));
        } else if (s + 1 < le && s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            s += 2;
            poly.clear();
            const size_t nv = o.v.size() / 3, nt = o.vt.size() / 2, nn = o.vn.size() / 3;
            while (true) {
                s = skipWs(s, le);
                if (s >= le || *s == '\r') break;
                const char* te = tokEnd(s, le);
                ObjIndex ix{-1, -1, -1};
                long a = std::strtol(s, nullptr, 10);
                ix.v = fixIndex(a, nv);
                const char* sl = static_cast<const char*>(std::memchr(s, '/', static_cast<size_t>(te - s)));
                if (sl) {
                    if (sl + 1 < te && sl[1] != '/') ix.vt = fixIndex(std::strtol(sl + 1, nullptr, 10), nt);
                    const char* sl2 = static_cast<const char*>(std::memchr(sl + 1, '/', static_cast<size_t>(te - sl - 1)));
                    if (sl2 && sl2 + 1 < te) ix.vn = fixIndex(std::strtol(sl2 + 1, nullptr, 10), nn);
                }
                poly.push_back(ix);
                s = te;
            }
            for (size_t k = 1; k + 1 < poly.size(); ++k) {   // fan triangulation
                o.idx.push_back(poly[0]); o.idx.push_back(poly[k]); o.idx.push_back(poly[k + 1]);
            }
        }
        p = le + 1;
    }
    return o;
}

// Parsed OBJ files of the scene being loaded: a file referenced by several
// <mesh> elements (instances with different transforms) is parsed once.
thread_local std::unordered_map<std::string, ObjData> t_objCache;

// src/main.cpp:267-401
std::vector<TriangleData> loadTriangles(const std::string& path, const TransformDesc& xf)
{
    auto it = t_objCache.find(path);
    if (it == t_objCache.end()) it = t_objCache.emplace(path, readObj(path)).first;
    const ObjData& o = it->second;
    std::vector<TriangleData> tris;
    auto V = [&](int i) -> Float3 {
        if (i < 0 || static_cast<size_t>(3 * i + 2) >= o.v.size()) fail("invalid vertex index in \"" + path + "\"");
        return {o.v[3 * i], o.v[3 * i + 1], o.v[3 * i + 2]};
    };
    auto N = [&](int i) -> Float3 {
        if (i < 0 || o.vn.empty()) return {0, 0, 0};
        return {o.vn[3 * i], o.vn[3 * i + 1], o.vn[3 * i + 2]};
    };
    auto UV = [&](int i) -> Float2 {
        if (i < 0 || o.vt.empty()) return {0, 0};
        return {o.vt[2 * i], o.vt[2 * i + 1]};
    };
    const bool realUV = o.vt.size() > 2;
    auto planarUV = [](const Float3& pos, const Float3& n) -> Float2 {
        const float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
        if (ay >= ax && ay >= az) return {pos.x, pos.z};
        if (ax >= ay && ax >= az) return {pos.y, pos.z};
        return {pos.x, pos.y};
    };
    tris.reserve(o.idx.size() / 3);
    for (size_t i = 0; i + 2 < o.idx.size(); i += 3) {
        const ObjIndex a = o.idx[i], b = o.idx[i + 1], c = o.idx[i + 2];
        TriangleData t{};
        t.v0 = xformPoint(V(a.v), xf);
        t.v1 = xformPoint(V(b.v), xf);
        t.v2 = xformPoint(V(c.v), xf);
        const bool hasN = a.vn >= 0 && b.vn >= 0 && c.vn >= 0 && !o.vn.empty();
        if (hasN) {
            t.n0 = xformNormal(N(a.vn), xf);
            t.n1 = xformNormal(N(b.vn), xf);
            t.n2 = xformNormal(N(c.vn), xf);
        } else {
            const Float3 e1 = {t.v1.x - t.v0.x, t.v1.y - t.v0.y, t.v1.z - t.v0.z};
            const Float3 e2 = {t.v2.x - t.v0.x, t.v2.y - t.v0.y, t.v2.z - t.v0.z};
            Float3 g = {e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
            const float len = std::sqrt(g.x * g.x + g.y * g.y + g.z * g.z);
            if (len > 1e-8f) { g.x /= len; g.y /= len; g.z /= len; }
            t.n0 = t.n1 = t.n2 = g;
        }
        if (realUV) {
            t.uv0 = UV(a.vt); t.uv1 = UV(b.vt); t.uv2 = UV(c.vt);
        } else {
            t.uv0 = planarUV(t.v0, t.n0); t.uv1 = planarUV(t.v1, t.n0); t.uv2 = planarUV(t.v2, t.n0);
        }
        tris.push_back(t);
    }
    if (tris.empty()) fail("no triangles found in OBJ: " + path);
    return tris;
}

// src/main.cpp:475-489
float triangleArea(const TriangleData& t)
{
    const float ax = t.v1.x - t.v0.x, ay = t.v1.y - t.v0.y, az = t.v1.z - t.v0.z;
    const float bx = t.v2.x - t.v0.x, by = t.v2.y - t.v0.y, bz = t.v2.z - t.v0.z;
    const float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    const float len = std::sqrt(cx * cx + cy * cy + cz * cz);
    return 0.5f * len;
}

// Radiance .hdr decode (RGBE, flat or RLE scanlines) to RGBA float (alpha 1).
bool loadHdr(const std::string& path, std::vector<float>& rgba, int& W, int& H, std::string& err)
{
    const std::string f = readFile(path);
    if (f.empty()) { err = "cannot read"; return false; }
    size_t pos = 0;
    auto line = [&]() {
        const size_t e = f.find('\n', pos);
        std::string l = f.substr(pos, (e == std::string::npos ? f.size() : e) - pos);
        pos = (e == std::string::npos) ? f.size() : e + 1;
        return l;
    };
    const std::string magic = line();
    if (magic != "#?RADIANCE" && magic != "#?RGBE") { err = "not HDR"; return false; }
    bool valid = false;
    while (true) {
        const std::string l = line();
        if (l.empty()) break;
        if (l == "FORMAT=32-bit_rle_rgbe") valid = true;
        if (pos >= f.size()) { err = "truncated header"; return false; }
    }
    if (!valid) { err = "unsupported HDR format"; return false; }
    std::string dims = line();
    if (dims.compare(0, 3, "-Y ") != 0) { err = "unsupported data layout"; return false; }
    const char* s = dims.c_str() + 3;
    char* e = nullptr;
    H = static_cast<int>(std::strtol(s, &e, 10));
    while (*e == ' ') ++e;
    if (std::strncmp(e, "+X ", 3) != 0) { err = "unsupported data layout"; return false; }
    W = static_cast<int>(std::strtol(e + 3, nullptr, 10));
    if (W <= 0 || H <= 0) { err = "bad dimensions"; return false; }
    rgba.assign(static_cast<size_t>(W) * H * 4, 0.0f);
    const unsigned char* d = reinterpret_cast<const unsigned char*>(f.data());
    const size_t n = f.size();
    auto get = [&]() -> int { return pos < n ? d[pos++] : 0; };
    auto conv = [&](size_t pix, const unsigned char* q) {
        float* o = &rgba[pix * 4];
        if (q[3] != 0) {
            const float f1 = static_cast<float>(std::ldexp(1.0f, q[3] - (128 + 8)));
            o[0] = q[0] * f1; o[1] = q[1] * f1; o[2] = q[2] * f1;
        } else {
            o[0] = o[1] = o[2] = 0.0f;
        }
        o[3] = 1.0f;
    };
    auto flat = [&](size_t startPix) {
        for (size_t pix = startPix; pix < static_cast<size_t>(W) * H; ++pix) {
            unsigned char q[4] = {static_cast<unsigned char>(get()), static_cast<unsigned char>(get()),
                                  static_cast<unsigned char>(get()), static_cast<unsigned char>(get())};
            conv(pix, q);
        }
    };
    if (W < 8 || W >= 32768) { flat(0); return true; }
    std::vector<unsigned char> sl(static_cast<size_t>(W) * 4);
    for (int j = 0; j < H; ++j) {
        const int c1 = get(), c2 = get(), lenHi = get();
        if (c1 != 2 || c2 != 2 || (lenHi & 0x80)) {
            // not run-length encoded: this and all remaining data are flat pixels (stb semantics)
            unsigned char q[4] = {static_cast<unsigned char>(c1), static_cast<unsigned char>(c2),
                                  static_cast<unsigned char>(lenHi), static_cast<unsigned char>(get())};
            conv(0, q);
            flat(1);
            return true;
        }
        const int len = (lenHi << 8) | get();
        if (len != W) { err = "invalid decoded scanline length"; return false; }
        for (int k = 0; k < 4; ++k) {
            int i = 0;
            while (W - i > 0) {
                int count = get();
                if (count > 128) {
                    const int value = get();
                    count -= 128;
                    if (count == 0 || count > W - i) { err = "bad RLE data"; return false; }
                    for (int z = 0; z < count; ++z) sl[static_cast<size_t>(i++) * 4 + k] = static_cast<unsigned char>(value);
                } else {
                    if (count == 0 || count > W - i) { err = "bad RLE data"; return false; }
                    for (int z = 0; z < count; ++z) sl[static_cast<size_t>(i++) * 4 + k] = static_cast<unsigned char>(get());
                }
            }
        }
        for (int i = 0; i < W; ++i) conv(static_cast<size_t>(j) * W + i, &sl[static_cast<size_t>(i) * 4]);
    }
    return true;
}

std::string dirOf(const std::string& p)
{
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string() : p.substr(0, s + 1);
}

// Paths in scene.xml are relative to the process working directory in the
// reference (src/main.cpp:704-709); the loader also accepts them relative to
// the scene file so generated scenes are self-contained.
std::string resolve(const std::string& scenePath, const std::string& p)
{
    if (p.empty() || p[0] == '/') return p;
    std::ifstream f(p);
    if (f.good()) return p;
    return dirOf(scenePath) + p;
}

}  // namespace

// src/main.cpp:523-930, minus the window/GL parts.
int sceneLoad(const char* path, SceneData& S, std::string& err)
{
    struct CacheReset { ~CacheReset() { t_objCache.clear(); } } cacheReset;
    t_objCache.clear();
    try {
        const std::string sp(path ? path : "");
        SceneDesc d = parseScene(sp);
        S = SceneData{};
        S.width = d.width;
        S.height = d.height;
        {   // camera basis (GLM normalize / cross, float)
            const Float3 eye = {d.camera.eyeX, d.camera.eyeY, d.camera.eyeZ};
            const Float3 tgt = {d.camera.lookAtX, d.camera.lookAtY, d.camera.lookAtZ};
            const Float3 up = {d.camera.upX, d.camera.upY, d.camera.upZ};
            auto sub = [](Float3 a, Float3 b) { return Float3{a.x - b.x, a.y - b.y, a.z - b.z}; };
            auto cross = [](Float3 a, Float3 b) {
                return Float3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
            };
            auto norm = [](Float3 a) {
                const float inv = 1.0f / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
                return Float3{a.x * inv, a.y * inv, a.z * inv};
            };
            const Float3 fwd = norm(sub(tgt, eye));
            const Float3 right = norm(cross(fwd, up));
            const Float3 tup = cross(right, fwd);
            const float rl = std::sqrt(right.x * right.x + right.y * right.y + right.z * right.z);
            if (!(rl >= 1e-6f)) fail("invalid camera basis: `up` must not be colinear with forward");
            if (d.height <= 0) fail("invalid window height");
            S.camera.origin = eye;
            S.camera.forward = fwd;
            S.camera.right = right;
            S.camera.up = tup;
            S.camera.fovYRadians = d.camera.fovY * 0.01745329251994329576923690768489f;
            S.camera.aspect = static_cast<float>(d.width) / static_cast<float>(d.height);
        }
        for (size_t i = 0; i < d.materials.size(); ++i) {
            // loadTextureAverage + loadImageRGBA, src/main.cpp:407-470 and :600-612: the material colour is the
            // texture's mean (per-pixel value / 255 summed in double, divided by the pixel count), white when
            // there is no texture or it fails to load; the image itself becomes the material's albedo texture.
            Float3 colour = {1.0f, 1.0f, 1.0f};
            std::vector<uint8_t> px;
            int tw = 1, th = 1, tc = 0;
            const std::string& tex = d.materials[i].albedoTexture;
            if (!tex.empty()) {
                std::string e2;
                if (loadImageRGBA8(resolve(sp, tex), px, tw, th, tc, e2)) {
                    double acc[3] = {0.0, 0.0, 0.0};
                    const size_t np = static_cast<size_t>(tw) * th;
                    for (size_t k = 0; k < np; ++k)
                        for (int c = 0; c < 3; ++c) acc[c] += px[4 * k + c] / 255.0;
                    colour = {static_cast<float>(acc[0] / static_cast<double>(np)),
                              static_cast<float>(acc[1] / static_cast<double>(np)),
                              static_cast<float>(acc[2] / static_cast<double>(np))};
                } else {
                    std::fprintf(stderr, "[bte] texture %s; material will use its BSDF colour\n", e2.c_str());
                    px.clear();
                    tw = th = 1;
                }
            }
            S.materials.push_back(colour);
            S.albedoImages.push_back(std::move(px));
            S.albedoWidths.push_back(tw);
            S.albedoHeights.push_back(th);
            S.mrImages.emplace_back();   // XML materials have no metallic-roughness map
            S.mrWidths.push_back(1);
            S.mrHeights.push_back(1);
        }
        for (const auto& b : d.bsdfs) {   // src/main.cpp:629-665
            BsdfData x{};
            if (b.type == "diffuse") {
                x.type = BSDF_Diffuse; x.p0 = {b.albedoR, b.albedoG, b.albedoB, 0.0f};
            } else if (b.type == "dielectric") {
                x.type = BSDF_Dielectric; x.p1 = {b.intIOR, b.extIOR, 0.0f, 0.0f};
            } else if (b.type == "mirror") {
                x.type = BSDF_Mirror;
                x.p0 = {b.albedoR > 0.0f ? b.albedoR : 1.0f, b.albedoG > 0.0f ? b.albedoG : 1.0f,
                        b.albedoB > 0.0f ? b.albedoB : 1.0f, 0.0f};
            } else if (b.type == "microfacet") {
                x.type = BSDF_Microfacet;
                const float ks = 1.0f - std::fmax(b.albedoR, std::fmax(b.albedoG, b.albedoB));
                x.p0 = {b.albedoR, b.albedoG, b.albedoB, 0.0f};
                x.p1 = {b.alpha, b.intIOR, b.extIOR, ks};
            } else {
                x.type = BSDF_Disney;
                x.p0 = {b.baseColorR, b.baseColorG, b.baseColorB, b.roughness};
                x.p1 = {b.metallic, b.specular, b.specularTransmission, b.specularTint};
                x.p2 = {b.sheen, b.sheenTint, b.subsurface, b.anisotropic};
                x.p3 = {b.clearcoat, b.clearcoatGloss, b.eta, 0.0f};
            }
            S.bsdfs.push_back(x);
        }
        auto matIndex = [&](const std::string& n) {
            for (size_t i = 0; i < d.materials.size(); ++i) if (d.materials[i].name == n) return static_cast<int>(i);
            return -1;
        };
        auto bsdfIndex = [&](const std::string& n) {
            for (size_t i = 0; i < d.bsdfs.size(); ++i) if (d.bsdfs[i].name == n) return static_cast<int>(i);
            return -1;
        };
        S.sceneEmitterCdf.push_back(0.0f);
        float weightSum = 0.0f;
        auto finishEmitter = [&](int triOff, int cdfOff, float area, const Float3& em) {   // src/main.cpp:686-701
            const float lum = 0.2126f * em.x + 0.7152f * em.y + 0.0722f * em.z;
            const float w = area * lum;
            weightSum += w;
            S.sceneEmitterCdf.push_back(weightSum);
            EmitterData e{};
            e.triIndexOffset = triOff;
            e.triCount = static_cast<int>(S.emitterTriIndices.size()) - triOff;
            e.cdfOffset = cdfOff;
            e.radiance = em;
            e.areaSum = area;
            e.powerWeight = w;
            S.emitters.push_back(e);
        };
        for (const auto& mesh : d.meshes) {   // src/main.cpp:704-758
            const int matId = matIndex(mesh.materialName);
            std::vector<TriangleData> mt = loadTriangles(resolve(sp, mesh.filename), mesh.transform);
            const int bsdfId = bsdfIndex(d.materials[static_cast<size_t>(matId)].bsdfName);
            const Float3 em = {mesh.radianceR, mesh.radianceG, mesh.radianceB};
            int triOff = 0, cdfOff = 0;
            float area = 0.0f;
            if (mesh.isEmitter) {
                triOff = static_cast<int>(S.emitterTriIndices.size());
                cdfOff = static_cast<int>(S.emitterTriCdf.size());
                S.emitterTriCdf.push_back(0.0f);
            }
            for (const auto& t : mt) {
                S.triangles.push_back(t);
                S.triangleMaterialIds.push_back(matId);
                S.triangleBsdfIds.push_back(bsdfId);
                S.triangleEmitterFlags.push_back(mesh.isEmitter ? 1 : 0);
                if (mesh.isEmitter) {
                    S.triangleEmission.push_back(em);
                    const int ti = static_cast<int>(S.triangles.size()) - 1;
                    area += triangleArea(t);
                    S.emitterTriIndices.push_back(ti);
                    S.emitterTriCdf.push_back(area);
                } else {
                    S.triangleEmission.push_back({0.0f, 0.0f, 0.0f});
                }
            }
            if (mesh.isEmitter) finishEmitter(triOff, cdfOff, area, em);
        }
        for (const auto& md : d.models) {   // glTF / GLB drop-ins, src/main.cpp:760-817
            const TransformDesc& x = md.transform;
            const float xf[9] = {x.posX, x.posY, x.posZ, x.rotX, x.rotY, x.rotZ, x.scaleX, x.scaleY, x.scaleZ};
            GltfResult g;
            std::string e2;
            if (!loadGltf(resolve(sp, md.filename), xf, g, e2)) fail("glTF model \"" + md.filename + "\": " + e2);
            const int matOffset = static_cast<int>(S.materials.size());
            const int bsdfOffset = static_cast<int>(S.bsdfs.size());
            const int firstTri = static_cast<int>(S.triangles.size());
            for (auto& slot : g.materials) {
                S.bsdfs.push_back(slot.bsdf);
                S.materials.push_back({1.0f, 1.0f, 1.0f});
                S.albedoWidths.push_back(slot.albedoWidth > 0 ? slot.albedoWidth : 1);
                S.albedoHeights.push_back(slot.albedoHeight > 0 ? slot.albedoHeight : 1);
                S.albedoImages.push_back(std::move(slot.albedo));
                S.mrWidths.push_back(slot.mrWidth > 0 ? slot.mrWidth : 1);
                S.mrHeights.push_back(slot.mrHeight > 0 ? slot.mrHeight : 1);
                S.mrImages.push_back(std::move(slot.mr));
            }
            for (size_t i = 0; i < g.triangles.size(); ++i) {
                const int local = g.materialIds[i];
                const GltfSlot& slot = g.materials[static_cast<size_t>(local)];
                S.triangles.push_back(g.triangles[i]);
                S.triangleMaterialIds.push_back(matOffset + local);
                S.triangleBsdfIds.push_back(bsdfOffset + local);
                S.triangleEmitterFlags.push_back(slot.isEmitter ? 1 : 0);
                S.triangleEmission.push_back(slot.isEmitter ? slot.emission : Float3{0.0f, 0.0f, 0.0f});
            }
            for (size_t mi = 0; mi < g.materials.size(); ++mi) {   // one emitter per emissive material
                const GltfSlot& slot = g.materials[mi];
                if (!slot.isEmitter) continue;
                const int triOff = static_cast<int>(S.emitterTriIndices.size());
                const int cdfOff = static_cast<int>(S.emitterTriCdf.size());
                S.emitterTriCdf.push_back(0.0f);
                float area = 0.0f;
                const int matId = matOffset + static_cast<int>(mi);
                for (int ti = firstTri; ti < static_cast<int>(S.triangles.size()); ++ti) {
                    if (S.triangleMaterialIds[static_cast<size_t>(ti)] != matId) continue;
                    area += triangleArea(S.triangles[static_cast<size_t>(ti)]);
                    S.emitterTriIndices.push_back(ti);
                    S.emitterTriCdf.push_back(area);
                }
                if (area > 0.0f) finishEmitter(triOff, cdfOff, area, slot.emission);
            }
        }
        if (S.triangles.empty()) fail("scene has no triangles after loading meshes and models");
        for (const auto& sd : d.spots) {   // src/main.cpp:879-904
            SpotlightData sp2{};
            sp2.position = {sd.posX, sd.posY, sd.posZ};
            float dx = sd.dirX, dy = sd.dirY, dz = sd.dirZ;
            const float dl = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (dl > 1e-6f) { dx /= dl; dy /= dl; dz /= dl; }
            sp2.direction = {dx, dy, dz};
            sp2.radiance = {sd.radianceR, sd.radianceG, sd.radianceB};
            sp2.intensity = sd.intensity;
            const float kPi = 3.14159265358979323846f;
            sp2.innerConeCosine = std::cos(sd.innerConeAngle * kPi / 180.0f);
            sp2.outerConeCosine = std::cos(sd.outerConeAngle * kPi / 180.0f);
            S.spotlights.push_back(sp2);
        }
        if (!d.envPath.empty()) {   // src/main.cpp:906-930
            std::string e2;
            if (!loadHdr(resolve(sp, d.envPath), S.envRGBA, S.envWidth, S.envHeight, e2))
                fail("failed to load environment map \"" + d.envPath + "\": " + e2);
            S.envIntensity = d.envIntensity;
            S.envRotationDeg = d.envRotation;
        }
        return 0;
    } catch (const LoadError& e) {
        err = e.msg;
        return -1;
    } catch (const std::exception& e) {
        err = e.what();
        return -1;
    }
}

}  // namespace bte
