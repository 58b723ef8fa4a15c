// sah.cuh -- binned SAH / spatial-split subtree builder (sah.cu).
#pragma once

#include "rt_internal.h"

#include <vector>

namespace rtb
{

constexpr int SAH_MAX_BINS = 32;

// A range of the Morton-sorted triangles handed to the binned SAH (a boundary node of the
// Morton-split tree, or the root).
struct SahRoot
{
    uint32_t kid;    // Karras node id
    uint32_t first;  // first sorted position
    uint32_t count;  // triangles
    uint32_t depth;  // depth in the whole tree (BFS level of the reference's queue)
    uint32_t rank;   // left-spine rank in the Morton-split tree
    float    box[6]; // exact range box
    uint32_t scene;  // scene of a batched build (0 otherwise)
};

struct SahInput
{
    const rt_vertex*   verts;
    const rt_triangle* tris;
    const float4*      lo;
    const float4*      hi;
    const float*       cz;
    const uint32_t*    perm;
    uint32_t           n, cap;
    SahRoot*           roots;  // device, arbitrary order
    uint32_t           n_roots;
    uint32_t*          wnode;  // per start key weights to fill for the roots
    uint32_t*          wtri;   // (the roots' keys are cleared here and in kpos: not in Morton leaves)
    uint8_t*           kpos;
    uint32_t*          status;  // the build's status word (ST_* flags)
    // spatial-split budget per scene (one scene unless batched): references in use at the
    // start (the scene's triangles) and the cap (bvh_morton.cpp:46-47)
    std::vector<uint32_t> budget_used, budget_cap;
};

struct SahResult
{
    uint32_t spatial_taken = 0, spatial_refused = 0, leaves = 0, nodes = 0, levels = 0;
    const SahRoot* sorted_roots = nullptr;  // device, sorted by (depth, first)
};

int sah_build(rt_bvh* B, const rt_build_cfg& cfg, const SahInput& in, cudaStream_t st, SahResult* res);
int sah_emit(rt_bvh* B, uint32_t n_roots, const uint32_t* snode, const uint32_t* stri, const rt_triangle* tris,
             cudaStream_t st, const SahResult& res, uint32_t max_nodes, uint32_t max_tris, uint32_t* status);

} // namespace rtb
