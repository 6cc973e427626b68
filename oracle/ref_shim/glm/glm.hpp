/* oracle/ref_shim/glm/glm.hpp -- ORACLE shim (test infrastructure only).
 *
 * GLM 1.0.1 is fetched by the reference's CMake build and is not in this tree, so
 * src/gltf_loader.cpp is compiled against this restatement of the part of GLM it
 * uses: float vectors with xyzw / rgba names, column-major mat3 / mat4, quat,
 * translate / rotate / scale, mat4_cast, make_mat4, inverse / transpose of a mat3,
 * normalize / length / min / max, and the matrix products, each with GLM's order of
 * floating-point operations (mat4 * vec4 sums its products in pairs; mat4 * mat4
 * sums them left to right; normalize multiplies by 1 / sqrt(dot)).  The product's
 * glTF reader (bluetruthengine_b200/csrc/bte_gltf.cpp) uses the same formulation. */
#pragma once
#include <cmath>

namespace glm {

struct vec2 {
    union { float x; float r; };
    union { float y; float g; };
    vec2() : x(0), y(0) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
};

struct vec4;
struct vec3 {
    union { float x; float r; };
    union { float y; float g; };
    union { float z; float b; };
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b_, float c) : x(a), y(b_), z(c) {}
    explicit vec3(const vec4& v);
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
};

struct vec4 {
    union { float x; float r; };
    union { float y; float g; };
    union { float z; float b; };
    union { float w; float a; };
    vec4() : x(0), y(0), z(0), w(0) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a_, float b_, float c, float d) : x(a_), y(b_), z(c), w(d) {}
    vec4(const vec3& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

inline vec3 make3(const vec4& v) { return vec3(v.x, v.y, v.z); }
inline vec3::vec3(const vec4& v) : x(v.x), y(v.y), z(v.z) {}

inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec4 operator+(const vec4& a, const vec4& b) { return vec4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline vec4 operator*(const vec4& a, float s) { return vec4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline vec4 operator*(const vec4& a, const vec4& b) { return vec4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }

inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline vec3 normalize(const vec3& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline vec3 min(const vec3& x, const vec3& y)
{
    return vec3(y.x < x.x ? y.x : x.x, y.y < x.y ? y.y : x.y, y.z < x.z ? y.z : x.z);
}
inline vec3 max(const vec3& x, const vec3& y)
{
    return vec3(x.x < y.x ? y.x : x.x, x.y < y.y ? y.y : x.y, x.z < y.z ? y.z : x.z);
}

struct mat4;
struct mat3 {
    vec3 c[3];
    mat3() {}
    explicit mat3(float d) { c[0] = vec3(d, 0, 0); c[1] = vec3(0, d, 0); c[2] = vec3(0, 0, d); }
    explicit mat3(const mat4& m);
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};

struct mat4 {
    vec4 c[4];
    mat4() {}
    explicit mat4(float d) { c[0] = vec4(d, 0, 0, 0); c[1] = vec4(0, d, 0, 0); c[2] = vec4(0, 0, d, 0); c[3] = vec4(0, 0, 0, d); }
    explicit mat4(const mat3& m)
    {
        c[0] = vec4(m[0], 0); c[1] = vec4(m[1], 0); c[2] = vec4(m[2], 0); c[3] = vec4(0, 0, 0, 1);
    }
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};

inline mat3::mat3(const mat4& m) { c[0] = make3(m[0]); c[1] = make3(m[1]); c[2] = make3(m[2]); }

inline mat4 operator*(const mat4& a, const mat4& b)
{
    mat4 r;
    for (int j = 0; j < 4; ++j) r[j] = a[0] * b[j][0] + a[1] * b[j][1] + a[2] * b[j][2] + a[3] * b[j][3];
    return r;
}
inline vec4 operator*(const mat4& m, const vec4& v)
{
    const vec4 add0 = m[0] * v[0] + m[1] * v[1];
    const vec4 add1 = m[2] * v[2] + m[3] * v[3];
    return add0 + add1;
}
inline vec3 operator*(const mat3& m, const vec3& v)
{
    return vec3(m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
                m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z);
}

inline mat3 transpose(const mat3& m)
{
    mat3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i][j] = m[j][i];
    return r;
}
inline mat3 inverse(const mat3& m)
{
    const float od = 1.0f / (+m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
                             m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
                             m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]));
    mat3 r;
    r[0][0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * od;
    r[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * od;
    r[2][0] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * od;
    r[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * od;
    r[1][1] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * od;
    r[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * od;
    r[0][2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * od;
    r[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * od;
    r[2][2] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * od;
    return r;
}

}  // namespace glm
