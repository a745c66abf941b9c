// Stand-in for glm/gtc/type_ptr.hpp (see glm/glm.hpp in this directory):
// value_ptr(v) is the address of the first component.
#pragma once
#include "../glm.hpp"

namespace glm {
template <int L, typename T> GLMS_FN T *value_ptr(vec<L, T> &v) { return &v.x; }
template <int L, typename T> GLMS_FN const T *value_ptr(const vec<L, T> &v) { return &v.x; }
} // namespace glm
