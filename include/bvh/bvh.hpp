// bvh.hpp -- shared types of the drop-in host API (the reference's src/bvh/bvh.hpp): the .bvh v1
// records (Triangle 12 B, BVHNode 48 B, Vertex 24 B) and, with BAKING defined, bvh::bakeBVH,
// which here reads the .scn on the host, builds on the GPU (librt_b200.so) and writes the .bvh.
#pragma once

#include <string>

#include "AABB.hpp"
#include "bvh_defines.hpp"

struct Triangle
{
    uint v[3];
};

struct BVHNode
{
    AABB aabb;
    bool isLeaf;
    union
    {
        uint childID[2];
        struct
        {
            uint beginTriIndex;
            uint triSize;
        };
    };
};

struct Vertex
{
    float x, y, z, nx, ny, nz;
    float operator[](int axis) const { return axis == 0 ? x : (axis == 1 ? y : z); }
};

static_assert(sizeof(Triangle) == 12 && sizeof(BVHNode) == 48 && sizeof(Vertex) == 24, ".bvh v1 record sizes");

#ifdef BAKING
namespace bvh
{
bool bakeBVH(const std::string& scenePath);
}
#endif
