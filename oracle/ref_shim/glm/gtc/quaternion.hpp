/* ORACLE shim (see glm/glm.hpp): quat(w, x, y, z) and mat4_cast with GLM's operation order. */
#pragma once
#include "../glm.hpp"

namespace glm {

struct quat {
    float x, y, z, w;
    quat(float w_, float x_, float y_, float z_) : x(x_), y(y_), z(z_), w(w_) {}
};

inline mat4 mat4_cast(const quat& q)
{
    mat3 r(1.0f);
    const float qxx = q.x * q.x, qyy = q.y * q.y, qzz = q.z * q.z;
    const float qxz = q.x * q.z, qxy = q.x * q.y, qyz = q.y * q.z;
    const float qwx = q.w * q.x, qwy = q.w * q.y, qwz = q.w * q.z;
    r[0][0] = 1.0f - 2.0f * (qyy + qzz);
    r[0][1] = 2.0f * (qxy + qwz);
    r[0][2] = 2.0f * (qxz - qwy);
    r[1][0] = 2.0f * (qxy - qwz);
    r[1][1] = 1.0f - 2.0f * (qxx + qzz);
    r[1][2] = 2.0f * (qyz + qwx);
    r[2][0] = 2.0f * (qxz + qwy);
    r[2][1] = 2.0f * (qyz - qwx);
    r[2][2] = 1.0f - 2.0f * (qxx + qyy);
    return mat4(r);
}

}  // namespace glm
