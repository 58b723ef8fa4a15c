// bvh_defines.hpp -- the reference's build constants (src/bvh/bvh_defines.hpp) as the defaults
// of this library's runtime configuration (rt_build_cfg_default in rt_b200.h).
#pragma once

#include <cstdint>

using uint = uint32_t;

constexpr uint  INVALID_NODE_INDEX          = 0xFFFFFFFF;
constexpr int   BVH_LBVH_THRESHOLD          = 64;
constexpr int   BVH_SAH_BINS_MIN            = 8;
constexpr int   BVH_SAH_BINS_MAX            = 32;
constexpr float BVH_C_TRAV                  = 1.0f;
constexpr float BVH_C_ISECT                 = 1.2f;
constexpr float BVH_CENTROID_EPS            = 1e-6f;
constexpr float BVH_SPATIAL_EPS             = 1e-6f;
constexpr int   BVH_MAX_LEAF_SIZE           = 16;
constexpr int   MORTON_UNIT_BIT_SIZE        = 21;
constexpr uint  MORTON_UNIT_MAX             = (1u << MORTON_UNIT_BIT_SIZE) - 1;
constexpr uint  BVH_FILE_VERSION            = 1;
constexpr float SPATIAL_TRICOUNT_MULTIPLIER = 1.5f;
