// AABB.hpp -- axis-aligned box of the drop-in host API, with the reference's interface
// (src/bvh/AABB.hpp): the empty box is (+inf, -inf); clipTriangleToAABB clips a triangle to a
// box (Sutherland-Hodgman) and returns the clipped polygon's box. Implemented in
// librt_b200.so (csrc/shim.cpp).
#pragma once

#include "../math/math.hpp"

using math::vec3;

enum class Axis { AXIS_X = 0, AXIS_Y = 1, AXIS_Z = 2 };

struct AABB
{
    vec3 min, max;

    AABB();
    AABB(vec3 p1, vec3 p2);

    void extend(vec3 p);
    void extend(const AABB& b);

    vec3  center() const;
    float half_area() const;
    Axis  largest_axis() const;
    bool  valid() const;
};

AABB merge(const AABB& a, const AABB& b);
AABB clipAABB(const AABB& box, int axis, float splitPos, bool leftSide);
AABB clipTriangleToAABB(vec3 v0, vec3 v1, vec3 v2, const AABB& clipRegion);
