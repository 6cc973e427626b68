/* ORACLE shim (see glm/glm.hpp): translate / rotate / scale with GLM's operation order. */
#pragma once
#include "../glm.hpp"

namespace glm {

inline mat4 translate(const mat4& m, const vec3& v)
{
    mat4 r = m;
    r[3] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2] + m[3];
    return r;
}
inline mat4 scale(const mat4& m, const vec3& v)
{
    mat4 r = m;
    r[0] = m[0] * v[0];
    r[1] = m[1] * v[1];
    r[2] = m[2] * v[2];
    return r;
}
inline mat4 rotate(const mat4& m, float angle, const vec3& v)
{
    const float c = std::cos(angle), s = std::sin(angle);
    const vec3 axis = normalize(v);
    const vec3 temp = (1.0f - c) * axis;
    mat4 rot(0.0f);
    rot[0][0] = c + temp[0] * axis[0];
    rot[0][1] = temp[0] * axis[1] + s * axis[2];
    rot[0][2] = temp[0] * axis[2] - s * axis[1];
    rot[1][0] = temp[1] * axis[0] - s * axis[2];
    rot[1][1] = c + temp[1] * axis[1];
    rot[1][2] = temp[1] * axis[2] + s * axis[0];
    rot[2][0] = temp[2] * axis[0] + s * axis[1];
    rot[2][1] = temp[2] * axis[1] - s * axis[0];
    rot[2][2] = c + temp[2] * axis[2];
    mat4 r;
    r[0] = m[0] * rot[0][0] + m[1] * rot[0][1] + m[2] * rot[0][2];
    r[1] = m[0] * rot[1][0] + m[1] * rot[1][1] + m[2] * rot[1][2];
    r[2] = m[0] * rot[2][0] + m[1] * rot[2][1] + m[2] * rot[2][2];
    r[3] = m[3];
    return r;
}

}  // namespace glm
