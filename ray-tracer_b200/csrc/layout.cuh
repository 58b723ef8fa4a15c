// layout.cuh -- writing .bvh v1 node records (src/bvh/bvh.hpp:16-30) from device code.
#pragma once

#include "device_math.cuh"
#include "rt_internal.h"

namespace rtb
{

// Writes one 48-byte node. The padding lane of each box is 0 once a point was added and
// keeps the +inf / -inf of the empty box otherwise (the reference's vec3 lanes); padding
// bytes are zero.
__device__ __forceinline__ void write_node(rt_bvh_node* out, uint32_t at, const rtd::box3& b, uint8_t leaf,
                                           uint32_t a, uint32_t bb)
{
    rt_bvh_node nd;
    const bool empty = !(b.mn[0] <= b.mx[0]) && b.mn[0] == rtd::bits2f(0x7f800000u);
    for (int k = 0; k < 3; k++) { nd.bmin[k] = b.mn[k]; nd.bmax[k] = b.mx[k]; }
    nd.bmin[3] = empty ? rtd::bits2f(0x7f800000u) : 0.f;
    nd.bmax[3] = empty ? rtd::bits2f(0xff800000u) : 0.f;
    nd.is_leaf = leaf;
    nd.pad0[0] = nd.pad0[1] = nd.pad0[2] = 0;
    nd.a = a;
    nd.b = bb;
    nd.pad1 = 0;
    out[at] = nd;
}

} // namespace rtb
