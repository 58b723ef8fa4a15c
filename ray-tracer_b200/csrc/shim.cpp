// shim.cpp -- the reference's C++ host interface on top of the C ABI, so code written against
// src/bvh/bvh.hpp, bvh_traverse.hpp and AABB.hpp (the reference's tests among it) compiles and
// links unchanged against librt_b200.so:
//   bvh::bakeBVH  (src/bvh/bvh_bake.cpp:180-194)   -> rt_bake_scene (GPU build, .bvh written)
//   bvh::loadBVH  (src/bvh/bvh_traverse.cpp:182-235) -> rt_load_bvh (one current BVH, as the
//                                                      reference keeps one static BVH)
//   bvh::trace    (src/bvh/bvh_traverse.cpp:237-246) -> rt_trace_host, a batch of one ray
//   AABB          (src/bvh/AABB.cpp:4-171)          -> host box helpers with the same results
#define BAKING
#include "bvh.hpp"
#include "bvh_traverse.hpp"
#include "AABB.hpp"

#include "../../include/rt_b200.h"

#include <cstdio>
#include <limits>
#include <mutex>

// ---- AABB ------------------------------------------------------------------------------------

AABB::AABB() : min(vec3(std::numeric_limits<float>::infinity())), max(vec3(-std::numeric_limits<float>::infinity())) {}
AABB::AABB(vec3 p1, vec3 p2) : min(math::min(p1, p2)), max(math::max(p1, p2)) {}

void AABB::extend(vec3 p)
{
    min = math::min(min, p);
    max = math::max(max, p);
}

void AABB::extend(const AABB& b)
{
    min = math::min(min, b.min);
    max = math::max(max, b.max);
}

vec3 AABB::center() const { return (min + max) * 0.5f; }

float AABB::half_area() const
{
    const vec3 d = max - min;
    return d.x * d.y + d.y * d.z + d.z * d.x;
}

Axis AABB::largest_axis() const
{
    const vec3 d = max - min;
    if (d.x >= d.y && d.x >= d.z) { return Axis::AXIS_X; }
    return d.y >= d.z ? Axis::AXIS_Y : Axis::AXIS_Z;
}

bool AABB::valid() const { return min.x <= max.x && min.y <= max.y && min.z <= max.z; }

AABB merge(const AABB& a, const AABB& b)
{
    AABB r;
    r.min = math::min(a.min, b.min);
    r.max = math::max(a.max, b.max);
    return r;
}

// The half of a box on one side of an axis plane; empty when the box lies entirely on the
// other side (a plane exactly on the box's face leaves nothing).
AABB clipAABB(const AABB& box, int axis, float split, bool left_side)
{
    AABB r = box;
    if (left_side)
    {
        if (box.min[axis] >= split) { return AABB(); }
        r.max[axis] = split < box.max[axis] ? split : box.max[axis];
    }
    else
    {
        if (box.max[axis] <= split) { return AABB(); }
        r.min[axis] = box.min[axis] < split ? split : box.min[axis];
    }
    return r;
}

// Sutherland-Hodgman: clip the polygon against min then max plane of x, y, z in turn.
AABB clipTriangleToAABB(vec3 v0, vec3 v1, vec3 v2, const AABB& region)
{
    vec3 poly[12], next[12];
    int n = 3;
    poly[0] = v0; poly[1] = v1; poly[2] = v2;
    for (int axis = 0; axis < 3; axis++)
    {
        for (int side = 0; side < 2; side++)
        {
            const float plane = side == 0 ? region.min[axis] : region.max[axis];
            int m = 0;
            for (int i = 0; i < n; i++)
            {
                const int j = i + 1 == n ? 0 : i + 1;
                const float a = poly[i][axis], b = poly[j][axis];
                const bool in_a = side == 0 ? a >= plane : a <= plane;
                const bool in_b = side == 0 ? b >= plane : b <= plane;
                if (in_a) { next[m++] = poly[i]; }
                if (in_a != in_b)
                {
                    const float t = (plane - a) / (b - a);
                    next[m++] = poly[i] + t * (poly[j] - poly[i]);
                }
            }
            for (int i = 0; i < m; i++) { poly[i] = next[i]; }
            n = m;
            if (n == 0) { return AABB(); }
        }
    }
    AABB r;
    for (int i = 0; i < n; i++) { r.extend(poly[i]); }
    return r;
}

// ---- bake / load / trace ---------------------------------------------------------------------

namespace
{
std::mutex g_mu;
rt_bvh* g_current = nullptr;  // the loaded BVH (the reference keeps one static BVH as well)
} // namespace

namespace bvh
{

bool bakeBVH(const std::string& scenePath)
{
    const int e = rt_bake_scene(scenePath.c_str(), nullptr, nullptr);
    if (e != RT_OK)
    {
        std::fprintf(stderr, "Error : %s on bakeBVH()\n", rt_last_error());
        return false;
    }
    return true;
}

bool loadBVH(const std::string& path)
{
    rt_bvh* b = nullptr;
    if (rt_load_bvh(path.c_str(), &b) != RT_OK)
    {
        if (rt_last_error()[0]) { std::fprintf(stderr, "Error : %s on loadBVH()\n", rt_last_error()); }
        return false;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_current) { rt_bvh_free(g_current); }
    g_current = b;
    return true;
}

Hit trace(const Ray& ray)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_current)
    {
        std::fprintf(stderr, "Error : BVH not loaded on trace()\n");
        return Hit{};
    }
    rt_ray r = { { ray.origin.x, ray.origin.y, ray.origin.z }, ray.tmin, { ray.dir.x, ray.dir.y, ray.dir.z }, ray.tmax };
    rt_hit h;
    const int e = rt_trace_host(g_current, &r, &h, 1, RT_TRACE_CLOSEST);
    Hit out;
    if (e != RT_OK && e != RT_E_STACK)
    {
        std::fprintf(stderr, "Error : %s on trace()\n", rt_last_error());
        return out;
    }
    if (h.flags & RT_HIT_FLAG_HIT)
    {
        out.hit = true;
        out.t = h.t;
        out.u = h.u;
        out.v = h.v;
        out.triIndex = h.tri;
        out.normal = math::vec3(h.n[0], h.n[1], h.n[2]);
    }
    return out;
}

} // namespace bvh
