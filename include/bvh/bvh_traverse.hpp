// bvh_traverse.hpp -- ray tracing of the drop-in host API (the reference's
// src/bvh/bvh_traverse.hpp): bvh::loadBVH uploads a .bvh file to the GPU and bvh::trace traces
// one ray there (a batch of one; rt_trace in rt_b200.h is the batched form).
#pragma once

#include <limits>
#include <string>

#include "../math/math.hpp"
#include "bvh_defines.hpp"

namespace bvh
{
struct Ray
{
    math::vec3 origin;
    math::vec3 dir;
    float tmin = 0.f;
    float tmax = std::numeric_limits<float>::infinity();
};

struct Hit
{
    bool       hit = false;
    float      t = 0.f;
    float      u = 0.f;
    float      v = 0.f;
    uint       triIndex = 0;
    math::vec3 normal;
};

bool loadBVH(const std::string& path);
Hit  trace(const Ray& ray);
} // namespace bvh
