// math.hpp -- the math header of the drop-in host API (the reference's src/math/math.hpp).
#pragma once

#include "vec3.hpp"
#include "vec4.hpp"
#include "quat.hpp"

namespace math
{
constexpr float pi = 3.14159265358979323846f;
}
