/* ORACLE shim (see glm/glm.hpp): make_mat4 from 16 column-major floats. */
#pragma once
#include "../glm.hpp"

namespace glm {

inline mat4 make_mat4(const float* p)
{
    mat4 m;
    for (int j = 0; j < 4; ++j) m[j] = vec4(p[4 * j], p[4 * j + 1], p[4 * j + 2], p[4 * j + 3]);
    return m;
}

}  // namespace glm
