// sah.cu -- the reference's binned SAH with spatial splits (trySAHSplit,
// src/bvh/bvh_sah.cpp:24-460) for every subtree the Morton-split build hands over, processed
// level by level over all subtrees at once, one thread block per node.
//
// The reference processes its node queue breadth-first (src/bvh/bvh_bfs.cpp:72-134) and lets
// spatial splits draw on one global budget of triangle references in that order
// (bvh_sah.cpp:390-394). Levels here are the reference's BFS levels; inside a level the nodes
// are kept in the reference's queue order (subtree roots by key position, then children in
// parent order), so the budget is granted in the same order. When the whole level fits in
// the remaining budget the grants need no ordering at all.
//
// The reference reorders triangle references with std::partition, whose result is Hoare's
// scheme: the k-th element from the left that fails the predicate is exchanged with the k-th
// element from the right that satisfies it, for k = 1, 2, ... while the two cursors have not
// met. cta_partition computes that permutation with block scans instead of a serial loop, so
// leaf contents come out in the reference's exact order.
#include "sah.cuh"
#include "device_math.cuh"
#include "cta_utils.cuh"
#include "layout.cuh"

#include <cuda/atomic>

#include <algorithm>
#include <vector>

namespace rtb
{
using namespace rtd;

namespace
{

constexpr int SBLK = 256;
enum : int { K_LEAF = 0, K_OBJECT = 1, K_SPATIAL = 2 };

struct LvlNode
{
    uint32_t ref_off, count, out, root, root_first, pad;
    float    box[6];
};

struct OutNode
{
    float    box[6];
    uint32_t is_leaf, a, b;  // inner: a, b = child out ids; leaf: a = leaf-store offset, b = count
    uint32_t root;           // index into the sorted roots
    uint32_t size, refs;     // subtree node count and triangle references
    uint32_t pre, toff;      // pre-order index and triangle offset inside the subtree
    uint32_t pad[2];
};

// Split decision of one node. For pre_spatial decisions the two spatial partitions
// (axis sp_axis, plane) are applied first, as the reference does before falling back
// (bvh_sah.cpp:303-330, 335-394).
struct Dec
{
    int      kind, pre_spatial;
    int      axis, bin;          // object split (kind == K_OBJECT) / spatial axis (K_SPATIAL)
    float    cmin, scale;
    float    plane;
    int      sp_axis;
    int      nb;
    uint32_t n, straddle, right;
    uint32_t oleft;              // left side of the object split that kind K_OBJECT applies
    int      fb_kind, oaxis, obin;
    float    ocmin, oscale;
};

struct Ctx
{
    const rt_vertex*   verts;
    const rt_triangle* tris;
    const float4*      lo;
    const float4*      hi;
    const float*       cz;
    uint32_t           max_leaf, bins_min, bins_max;
    float              c_trav, c_isect, centroid_eps, spatial_eps;
};

__device__ __forceinline__ float centroid(const Ctx& C, uint32_t t, int axis)
{
    return axis == 0 ? C.lo[t].w : (axis == 1 ? C.hi[t].w : C.cz[t]);
}
__device__ __forceinline__ box3 tri_box(const Ctx& C, uint32_t t)
{
    const float4 a = C.lo[t], c = C.hi[t];
    box3 b;
    b.mn[0] = a.x; b.mn[1] = a.y; b.mn[2] = a.z; b.mx[0] = c.x; b.mx[1] = c.y; b.mx[2] = c.z;
    return b;
}
__device__ __forceinline__ float tri_lo(const Ctx& C, uint32_t t, int axis)
{
    const float4 a = C.lo[t];
    return axis == 0 ? a.x : (axis == 1 ? a.y : a.z);
}
__device__ __forceinline__ float tri_hi(const Ctx& C, uint32_t t, int axis)
{
    const float4 a = C.hi[t];
    return axis == 0 ? a.x : (axis == 1 ? a.y : a.z);
}
__device__ __forceinline__ void tri_verts(const Ctx& C, uint32_t t, f3& a, f3& b, f3& c)
{
    const rt_triangle tr = C.tris[t];
    const rt_vertex* v = C.verts;
    a = mk3(v[tr.v[0]].x, v[tr.v[0]].y, v[tr.v[0]].z);
    b = mk3(v[tr.v[1]].x, v[tr.v[1]].y, v[tr.v[1]].z);
    c = mk3(v[tr.v[2]].x, v[tr.v[2]].y, v[tr.v[2]].z);
}

// std_clampi(x86_f2i(x), 0, nb - 1) with top = nb - 1 (at most 31) as a float, without a
// float-to-int conversion (those issue on the narrow conversion pipe, which the binning loops
// would saturate): NaN, x < 1 and x >= 2^31 (x86's out-of-range result, INT_MIN) give 0, any
// other x min(floor(x), top). floor(y) of y in [0, 31] is read from the bits of y + 2^23 added
// with rounding toward zero (the sum's unit in the last place is 1).
__device__ __forceinline__ int bin_clamp(float x, float top)
{
    const float y = fminf(fmaxf(x, 0.0f), top);  // fmaxf(NaN, 0) = 0
    const int b = __float_as_int(__fadd_rz(y, 8388608.0f)) - 0x4B000000;
    return x < 2147483648.0f ? b : 0;
}

// Object-split bin of a centroid (bvh_sah.cpp:85, :260); in [0, nb) for centroids inside
// [cmin, cmax], which is the only case the reference meets.
__device__ __forceinline__ int obj_bin(float c, float cmin, float scale, int nb)
{
    return bin_clamp((c - cmin) * scale, (float)(nb - 1));
}

// Where an evaluation reads its references' data: straight from the triangle arrays through
// the node's reference list, or from a warp's copy of them in shared memory. Reference i is
// the node's i-th; both give the same floats.
struct GlobalRefs
{
    const float4*      lo;
    const float4*      hi;
    const float*       cz;
    const rt_triangle* tris;
    const rt_vertex*   verts;
    const uint32_t*    R;
    __device__ __forceinline__ GlobalRefs(const Ctx& C, const uint32_t* R_)
        : lo(C.lo), hi(C.hi), cz(C.cz), tris(C.tris), verts(C.verts), R(R_) {}
    __device__ __forceinline__ float cen(uint32_t i, int axis) const
    {
        const uint32_t t = R[i];
        return axis == 0 ? lo[t].w : (axis == 1 ? hi[t].w : cz[t]);
    }
    __device__ __forceinline__ float lo_of(uint32_t i, int axis) const
    {
        const float4 a = lo[R[i]];
        return axis == 0 ? a.x : (axis == 1 ? a.y : a.z);
    }
    __device__ __forceinline__ float hi_of(uint32_t i, int axis) const
    {
        const float4 a = hi[R[i]];
        return axis == 0 ? a.x : (axis == 1 ? a.y : a.z);
    }
    __device__ __forceinline__ box3 box(uint32_t i) const
    {
        const uint32_t t = R[i];
        const float4 a = lo[t], c = hi[t];
        box3 b;
        b.mn[0] = a.x; b.mn[1] = a.y; b.mn[2] = a.z; b.mx[0] = c.x; b.mx[1] = c.y; b.mx[2] = c.z;
        return b;
    }
    __device__ __forceinline__ void tri_verts(uint32_t i, f3& a, f3& b, f3& c) const
    {
        const rt_triangle tr = tris[R[i]];
        a = mk3(verts[tr.v[0]].x, verts[tr.v[0]].y, verts[tr.v[0]].z);
        b = mk3(verts[tr.v[1]].x, verts[tr.v[1]].y, verts[tr.v[1]].z);
        c = mk3(verts[tr.v[2]].x, verts[tr.v[2]].y, verts[tr.v[2]].z);
    }
};

// A warp's shared copy of at most EVAL_STAGE references: bounds with the x / y centroids in
// lane 3 (as in Ctx::lo / hi), z centroids, and the three vertices (9 floats: an odd stride,
// so a warp reading consecutive references hits distinct banks).
constexpr uint32_t EVAL_STAGE = 64;
struct StageBuf
{
    float4 lo[EVAL_STAGE], hi[EVAL_STAGE];
    float  cz[EVAL_STAGE];
    float  v[EVAL_STAGE * 9];
};
struct StagedRefs
{
    const StageBuf* S;
    const uint32_t* R;
    __device__ __forceinline__ float cen(uint32_t i, int axis) const
    {
        return axis == 0 ? S->lo[i].w : (axis == 1 ? S->hi[i].w : S->cz[i]);
    }
    __device__ __forceinline__ float lo_of(uint32_t i, int axis) const
    {
        const float4 a = S->lo[i];
        return axis == 0 ? a.x : (axis == 1 ? a.y : a.z);
    }
    __device__ __forceinline__ float hi_of(uint32_t i, int axis) const
    {
        const float4 a = S->hi[i];
        return axis == 0 ? a.x : (axis == 1 ? a.y : a.z);
    }
    __device__ __forceinline__ box3 box(uint32_t i) const
    {
        const float4 a = S->lo[i], c = S->hi[i];
        box3 b;
        b.mn[0] = a.x; b.mn[1] = a.y; b.mn[2] = a.z; b.mx[0] = c.x; b.mx[1] = c.y; b.mx[2] = c.z;
        return b;
    }
    __device__ __forceinline__ void tri_verts(uint32_t i, f3& a, f3& b, f3& c) const
    {
        const float* v = S->v + 9 * i;
        a = mk3(v[0], v[1], v[2]);
        b = mk3(v[3], v[4], v[5]);
        c = mk3(v[6], v[7], v[8]);
    }
};

// Copies references [0, n) of R (n <= EVAL_STAGE) into S, one warp.
__device__ __forceinline__ void stage_refs(const Ctx& C, const uint32_t* R, uint32_t n, StageBuf& S)
{
    for (uint32_t i = threadIdx.x & 31; i < n; i += 32)
    {
        const uint32_t t = R[i];
        S.lo[i] = C.lo[t];
        S.hi[i] = C.hi[t];
        S.cz[i] = C.cz[t];
        const rt_triangle tr = C.tris[t];
        float* v = S.v + 9 * i;
#pragma unroll
        for (int k = 0; k < 3; k++)
        {
            const rt_vertex& q = C.verts[tr.v[k]];
            v[3 * k] = q.x; v[3 * k + 1] = q.y; v[3 * k + 2] = q.z;
        }
    }
    __syncwarp();
}

// Shared box accumulator in the order-preserving uint encoding.
struct SBox { uint32_t m[3], M[3]; };
__device__ __forceinline__ void sbox_clear(SBox& s) { for (int k = 0; k < 3; k++) { s.m[k] = 0xffffffffu; s.M[k] = 0u; } }
__device__ __forceinline__ void sbox_add(SBox& s, const box3& b)
{
    for (int k = 0; k < 3; k++) { atomicMin(&s.m[k], f2ord(b.mn[k])); atomicMax(&s.M[k], f2ord(b.mx[k])); }
}
// A thread's own accumulation in the same encoding, merged into a shared SBox once per warp
// (min / max of the encoded values are exact and order-free, so the result is the same as
// adding every box to the SBox directly).
struct OBox { uint32_t m[3], M[3]; };
__device__ __forceinline__ void obox_clear(OBox& o) { for (int k = 0; k < 3; k++) { o.m[k] = 0xffffffffu; o.M[k] = 0u; } }
__device__ __forceinline__ void obox_add(OBox& o, const box3& b)
{
    for (int k = 0; k < 3; k++) { o.m[k] = min(o.m[k], f2ord(b.mn[k])); o.M[k] = max(o.M[k], f2ord(b.mx[k])); }
}
__device__ __forceinline__ void obox_flush_warp(OBox o, SBox& s)
{
    for (int k = 0; k < 3; k++)
    {
        o.m[k] = __reduce_min_sync(0xffffffffu, o.m[k]);
        o.M[k] = __reduce_max_sync(0xffffffffu, o.M[k]);
    }
    if ((threadIdx.x & 31) == 0 && !(o.m[0] == 0xffffffffu && o.M[0] == 0u))
    {
        for (int k = 0; k < 3; k++) { atomicMin(&s.m[k], o.m[k]); atomicMax(&s.M[k], o.M[k]); }
    }
}
__device__ __forceinline__ box3 sbox_get(const SBox& s)
{
    box3 b;
    for (int k = 0; k < 3; k++) { b.mn[k] = ord2f(s.m[k]); b.mx[k] = ord2f(s.M[k]); }
    return b;
}
// Reads the union of the contributions of a whole block; the empty box when none.
__device__ __forceinline__ box3 sbox_result(const SBox& s)
{
    box3 b = box_empty();
    if (s.m[0] != 0xffffffffu) { b = sbox_get(s); }
    return b;
}

// Hoare-scheme partition of in[0, n) by pred into out[0, n) (in == out allowed). Returns the
// number of elements satisfying pred. flags/pos: n scratch entries each.
template <int BS, class Pred>
__device__ uint32_t cta_partition(const uint32_t* in, uint32_t* out, uint32_t n, Pred pred, uint8_t* flags,
                                  uint32_t* pos, uint32_t* sh)
{
    const int tid = threadIdx.x;
    uint32_t c = 0;
    for (uint32_t i = tid; i < n; i += BS)
    {
        const uint8_t f = pred(in[i]) ? 1 : 0;
        flags[i] = f;
        c += f;
    }
    const uint32_t m = block_sum<BS>(c, sh);
    // satisfying elements right of the split point, in ascending order
    uint32_t run = 0;
    for (uint32_t base = m; base < n; base += BS)
    {
        const uint32_t i = base + tid;
        const uint32_t f = (i < n) ? flags[i] : 0u;
        uint32_t tot;
        const uint32_t e = block_excl_scan<BS>(f, sh, &tot);
        if (f) { pos[run + e] = i; }
        run += tot;
    }
    __syncthreads();
    const uint32_t tr = run;  // equals the failing elements left of the split point
    // exchange the k-th failing element from the left with the k-th satisfying one from the right
    uint32_t k0 = 0;
    for (uint32_t base = 0; base < m; base += BS)
    {
        const uint32_t i = base + tid;
        const uint32_t f = (i < m) ? (flags[i] ? 0u : 1u) : 0u;
        uint32_t tot;
        const uint32_t e = block_excl_scan<BS>(f, sh, &tot);
        if (i < m)
        {
            if (f)
            {
                const uint32_t q = pos[tr - 1u - (k0 + e)];
                const uint32_t a = in[i], b = in[q];
                out[i] = b;
                out[q] = a;
            }
            else if (in != out) { out[i] = in[i]; }
        }
        k0 += tot;
    }
    if (in != out)
    {
        for (uint32_t i = m + tid; i < n; i += BS)
        {
            if (!flags[i]) { out[i] = in[i]; }
        }
    }
    __syncthreads();
    return m;
}

// The best candidate so far, in the reference's evaluation order.
struct Best
{
    float cost, cmin, scale, node_min, sscale;
    int   axis, bin, spatial;
};

// The candidate sweeps of bvh_sah.cpp:88-126 (object splits: centroid bins, counts from both
// sides) and :198-243 (spatial splits: entry counts from the left, exit counts from the right,
// clipped boxes), bins b = nb-1 .. 1, strict improvement only -- across one warp: lane b holds
// bin b; the left and right unions are
// inclusive scans of the order-preserving box encoding (min / max are exact there, so the
// decoded boxes -- and the costs -- equal the serial ones: the serial union of float boxes
// differs only in the sign of zero bounds, which leaves extents and areas unchanged), and the
// winner is the candidate the serial loop keeps: the lowest cost, on ties the first in its
// order (bins b = nb-1 .. 1), taken only if strictly below the best so far. All 32 lanes call
// these with the same B and return the same B.
__device__ __forceinline__ void warp_box_scan_up(uint32_t (&m)[3], uint32_t (&M)[3], uint32_t& c, int lane)
{
#pragma unroll 1  // (rolled: the sweeps are inlined at several places; code size over loop overhead)
    for (int o = 1; o < 32; o <<= 1)
    {
        uint32_t tm[3], tM[3];
        for (int k = 0; k < 3; k++) { tm[k] = __shfl_up_sync(0xffffffffu, m[k], o); tM[k] = __shfl_up_sync(0xffffffffu, M[k], o); }
        const uint32_t tc = __shfl_up_sync(0xffffffffu, c, o);
        if (lane >= o)
        {
            for (int k = 0; k < 3; k++) { m[k] = min(m[k], tm[k]); M[k] = max(M[k], tM[k]); }
            c += tc;
        }
    }
}
__device__ __forceinline__ void warp_box_scan_down(uint32_t (&m)[3], uint32_t (&M)[3], uint32_t& c, int lane)
{
#pragma unroll 1  // (rolled: the sweeps are inlined at several places; code size over loop overhead)
    for (int o = 1; o < 32; o <<= 1)
    {
        uint32_t tm[3], tM[3];
        for (int k = 0; k < 3; k++) { tm[k] = __shfl_down_sync(0xffffffffu, m[k], o); tM[k] = __shfl_down_sync(0xffffffffu, M[k], o); }
        const uint32_t tc = __shfl_down_sync(0xffffffffu, c, o);
        if (lane + o < 32)
        {
            for (int k = 0; k < 3; k++) { m[k] = min(m[k], tm[k]); M[k] = max(M[k], tM[k]); }
            c += tc;
        }
    }
}
__device__ __forceinline__ box3 ord_box(const uint32_t (&m)[3], const uint32_t (&M)[3])
{
    box3 b = box_empty();
    if (m[0] != 0xffffffffu) { for (int k = 0; k < 3; k++) { b.mn[k] = ord2f(m[k]); b.mx[k] = ord2f(M[k]); } }
    return b;
}

// cl / cr: the counts that enter the left / right sweeps (object: the bin count for both;
// spatial: entries and exits); has_box(b): whether bin b's box joins the unions.
__device__ __forceinline__ bool warp_sweep(const uint32_t* cl, const uint32_t* cr, const SBox* bins, bool object, int nb,
                                           float parent_inv_area, const Ctx& C, float& best_cost, int& best_bin)
{
    const int lane = threadIdx.x & 31;
    uint32_t lm[3], lM[3], rm[3], rM[3], lc = 0, rc = 0;
    for (int k = 0; k < 3; k++) { lm[k] = rm[k] = 0xffffffffu; lM[k] = rM[k] = 0u; }
    if (lane < nb)
    {
        const SBox& sb = bins[lane];
        const bool use = object ? (cl[lane] != 0u) : true;
        if (use) { for (int k = 0; k < 3; k++) { lm[k] = rm[k] = sb.m[k]; lM[k] = rM[k] = sb.M[k]; } }
        lc = cl[lane];
        rc = cr[lane];
    }
    warp_box_scan_up(lm, lM, lc, lane);    // lane b: bins 0..b
    warp_box_scan_down(rm, rM, rc, lane);  // lane b: bins b..31 (empty beyond nb)
    // candidate b pairs the left union up to b-1 with the right union from b
    uint32_t pm[3], pM[3];
    for (int k = 0; k < 3; k++) { pm[k] = __shfl_up_sync(0xffffffffu, lm[k], 1); pM[k] = __shfl_up_sync(0xffffffffu, lM[k], 1); }
    const uint32_t pc = __shfl_up_sync(0xffffffffu, lc, 1);
    float cost = __int_as_float(0x7f800000);
    if (lane >= 1 && lane < nb && pc != 0u && rc != 0u)
    {
        const box3 lb = ord_box(pm, pM), rb = ord_box(rm, rM);
        cost = C.c_trav + C.c_isect * (box_half_area(lb) * (float)pc + box_half_area(rb) * (float)rc) * parent_inv_area;
        if (!(cost <= 3.402823466e38f)) { cost = __int_as_float(0x7f800000); }  // a NaN never wins, as in the serial loop
    }
    // lowest cost; ties to the larger bin (visited first by the serial loop)
    float bc = cost;
    int bb = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
        const int obb = __shfl_xor_sync(0xffffffffu, bb, o);
        if (oc < bc || (oc == bc && obb > bb)) { bc = oc; bb = obb; }
    }
    if (bc < best_cost) { best_cost = bc; best_bin = bb; return true; }
    return false;
}

__device__ __forceinline__ void warp_eval_object_axis(const uint32_t* cnt, const SBox* bins, int nb, int axis, float cmin,
                                                      float scale, float parent_inv_area, const Ctx& C, Best& B)
{
    int bin = -1;
    if (warp_sweep(cnt, cnt, bins, true, nb, parent_inv_area, C, B.cost, bin))
    {
        B.axis = axis; B.bin = bin; B.cmin = cmin; B.scale = scale;
    }
}

__device__ __forceinline__ void warp_eval_spatial_axis(const uint32_t* cin, const uint32_t* cout, const SBox* bins, int nb,
                                                       int axis, float node_min, float sscale, float parent_inv_area,
                                                       const Ctx& C, Best& B)
{
    int bin = -1;
    if (warp_sweep(cin, cout, bins, false, nb, parent_inv_area, C, B.cost, bin))
    {
        B.axis = axis; B.bin = bin; B.spatial = 1; B.node_min = node_min; B.sscale = sscale;
    }
}

// bnd[b] = node_min + b / sscale for b = 0 .. nb, by threads t of `count` (the region bounds of
// bvh_sah.cpp:180-181, computed once per axis instead of once per clipped triangle).
__device__ __forceinline__ void bin_bounds(float* bnd, float node_min, float sscale, int nb, int t, int count)
{
    for (int b = t; b <= nb; b += count) { bnd[b] = node_min + (float)b / sscale; }
}

// Spatial binning of references R[i0 + lane] (i0 + lane < n) along `axis` by one whole warp:
// entry / exit counts, then every (triangle, bin) pair of the 32 references clipped and added to
// its bin -- the pairs spread evenly over the lanes (a warp-wide scan of each reference's bin
// count, each lane finding the owner of its pair by a binary search over the lanes), since the
// references span different numbers of bins. The same clips as bvh_sah.cpp:175-193; the bin
// boxes are exact unions, so their order does not matter. bnd[b] = node_min + b / sscale, the
// bins' bounds (b = 0 .. nb), computed once per axis by the caller (bin_bounds).
template <class Src>
__device__ __forceinline__ void spatial_bin_warp(const Src& src, uint32_t i0, uint32_t n, int axis, const box3& nbox,
                                                 float node_min, float sscale, int nb, const float* bnd, uint32_t* cin,
                                                 uint32_t* cout, SBox* bins, bool count = true)
{
    const int lane = threadIdx.x & 31;
    const uint32_t i = i0 + (uint32_t)lane;
    const float top = (float)(nb - 1);
    int bmin = 0, bmax = -1;
    if (i < n)
    {
        bmin = bin_clamp((src.lo_of(i, axis) - node_min) * sscale, top);
        bmax = bin_clamp((src.hi_of(i, axis) - node_min) * sscale, top);
        if (count)
        {
            atomicAdd(&cin[bmin], 1u);
            atomicAdd(&cout[bmax], 1u);
        }
    }
    const uint32_t c = bmin <= bmax ? (uint32_t)(bmax - bmin + 1) : 0u;
    const uint32_t incl = warp_incl_scan(c);
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t j0 = 0; j0 < total; j0 += 32)
    {
        const uint32_t j = j0 + (uint32_t)lane;
        int o = 0;  // the lane whose pairs hold pair j: the number of lanes with incl <= j
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1)
        {
            if (__shfl_sync(0xffffffffu, incl, o + step - 1) <= j) { o += step; }
        }
        const uint32_t to = i0 + (uint32_t)o;
        const int bo = __shfl_sync(0xffffffffu, bmin, o);
        const uint32_t eo = __shfl_sync(0xffffffffu, incl - c, o);
        if (j < total)
        {
            const int b = bo + (int)(j - eo);
            f3 v0, v1, v2;
            src.tri_verts(to, v0, v1, v2);
            const float lo_b = bnd[b], hi_b = bnd[b + 1];
            box3 region;
#pragma unroll
            for (int k = 0; k < 3; k++)
            {
                region.mn[k] = k == axis ? lo_b : nbox.mn[k];
                region.mx[k] = k == axis ? hi_b : nbox.mx[k];
            }
            const box3 cl = clip_triangle(v0, v1, v2, region);
            if (box_valid(cl)) { sbox_add(bins[b], cl); }
        }
    }
}

// Spatial candidates that cannot win, found before any clipping. The clipped box of a (triangle,
// bin) pair contains every vertex of the triangle that lies in the bin's region (a clip keeps
// such vertices unchanged), so the boxes of those vertices alone lie inside each bin's box, the
// sweep's unions likewise, and -- the cost being monotone in the two areas when c_isect >= 0 --
// every candidate's cost is bounded from below (an empty union counting as area 0; the float
// operations are the cost's own, and rounding is monotone). When no candidate's bound is below
// the best cost so far, none can win the strict comparison and the axis's clipping is skipped:
// the decision is the one the full evaluation makes.
//
// The entry / exit counts (the exact ones) and the vertex boxes of references i0 + lane < n.
template <class Src>
__device__ __forceinline__ void spatial_bound_warp(const Src& src, uint32_t i0, uint32_t n, int axis, const box3& nbox,
                                                   float node_min, float sscale, int nb, const float* bnd, uint32_t* cin,
                                                   uint32_t* cout, SBox* bins)
{
    const uint32_t i = i0 + (threadIdx.x & 31u);
    if (i >= n) { return; }
    const float top = (float)(nb - 1);
    const int bmin = bin_clamp((src.lo_of(i, axis) - node_min) * sscale, top);
    const int bmax = bin_clamp((src.hi_of(i, axis) - node_min) * sscale, top);
    atomicAdd(&cin[bmin], 1u);
    atomicAdd(&cout[bmax], 1u);
    if (bmin > bmax) { return; }
    f3 v[3];
    src.tri_verts(i, v[0], v[1], v[2]);
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
        const float x = v[k].x, y = v[k].y, z = v[k].z;
        const float c = axis == 0 ? x : (axis == 1 ? y : z);
        bool in = true;
        if (axis != 0) { in = in && x >= nbox.mn[0] && x <= nbox.mx[0]; }
        if (axis != 1) { in = in && y >= nbox.mn[1] && y <= nbox.mx[1]; }
        if (axis != 2) { in = in && z >= nbox.mn[2] && z <= nbox.mx[2]; }
        const int vb = bin_clamp((c - node_min) * sscale, top);
        if (!in || vb < bmin || vb > bmax || !(c >= bnd[vb] && c <= bnd[vb + 1])) { continue; }
        SBox& sb = bins[vb];
        atomicMin(&sb.m[0], f2ord(x)); atomicMin(&sb.m[1], f2ord(y)); atomicMin(&sb.m[2], f2ord(z));
        atomicMax(&sb.M[0], f2ord(x)); atomicMax(&sb.M[1], f2ord(y)); atomicMax(&sb.M[2], f2ord(z));
    }
}

// Whether any spatial candidate's lower bound (from spatial_bound_warp's bins) is below
// best_cost, or is not a number; every lane of the calling warp returns the same.
__device__ __forceinline__ bool warp_spatial_can_win(const uint32_t* cin, const uint32_t* cout, const SBox* bins, int nb,
                                                     float parent_inv_area, const Ctx& C, float best_cost)
{
    const int lane = threadIdx.x & 31;
    uint32_t lm[3], lM[3], rm[3], rM[3], lc = 0, rc = 0;
    for (int k = 0; k < 3; k++) { lm[k] = rm[k] = 0xffffffffu; lM[k] = rM[k] = 0u; }
    if (lane < nb)
    {
        const SBox& sb = bins[lane];
        for (int k = 0; k < 3; k++) { lm[k] = rm[k] = sb.m[k]; lM[k] = rM[k] = sb.M[k]; }
        lc = cin[lane];
        rc = cout[lane];
    }
    warp_box_scan_up(lm, lM, lc, lane);
    warp_box_scan_down(rm, rM, rc, lane);
    uint32_t pm[3], pM[3];
    for (int k = 0; k < 3; k++) { pm[k] = __shfl_up_sync(0xffffffffu, lm[k], 1); pM[k] = __shfl_up_sync(0xffffffffu, lM[k], 1); }
    const uint32_t pc = __shfl_up_sync(0xffffffffu, lc, 1);
    bool can = false;
    if (lane >= 1 && lane < nb && pc != 0u && rc != 0u)
    {
        const float al = pm[0] == 0xffffffffu ? 0.f : box_half_area(ord_box(pm, pM));
        const float ar = rm[0] == 0xffffffffu ? 0.f : box_half_area(ord_box(rm, rM));
        const float cost = C.c_trav + C.c_isect * (al * (float)pc + ar * (float)rc) * parent_inv_area;
        can = !(cost >= best_cost);
    }
    return __any_sync(0xffffffffu, can);
}

// Nodes with more references than this are evaluated and partitioned by many blocks (the
// wide kernels below); nodes with at most WARP_MAX references are evaluated by one warp each
// (k_sah_eval_warp); the rest by one block each.
constexpr uint32_t WIDE_MIN = 16384;
constexpr uint32_t WARP_MAX = 512;
constexpr int      EVAL_WPB = 8;  // warps (nodes) per block of k_sah_eval_warp

// The evaluation of k_sah_eval below for one small node per warp: the same candidates, bins
// and serial sweeps (lane 0), with warp reductions in place of block ones.
struct EvalWS
{
    uint32_t cnt[SAH_MAX_BINS], cin[SAH_MAX_BINS], cout[SAH_MAX_BINS];
    SBox     bins[SAH_MAX_BINS];
    float    bnd[SAH_MAX_BINS + 1];
};

template <class Src>
__device__ __forceinline__ void eval_node_warp(const Src& src, const LvlNode& nd, uint32_t n, const Ctx& C, EvalWS& S,
                                               Dec& d)
{
    const int lane = threadIdx.x & 31;
    const int nb = std_clampi((int)n / 4, (int)C.bins_min, (int)C.bins_max);
    box3 nbox;
    for (int k = 0; k < 3; k++) { nbox.mn[k] = nd.box[k]; nbox.mx[k] = nd.box[3 + k]; }
    const float parent_inv_area = 1.0f / box_half_area(nbox);
    Best Bw;  // identical in every lane
    Bw.cost = C.c_isect * (float)n;  // leaf cost, bvh_sah.cpp:32
    Bw.axis = -1; Bw.bin = -1; Bw.cmin = 0.f; Bw.scale = 0.f; Bw.spatial = 0; Bw.node_min = 0.f; Bw.sscale = 0.f;
    // phase 1: centroid-binned object split (bvh_sah.cpp:52-126)
    for (int axis = 0; axis < 3; axis++)
    {
        uint32_t m = 0xffffffffu, M = 0u;
        for (uint32_t i = lane; i < n; i += 32)
        {
            const uint32_t o = f2ord(src.cen(i, axis));
            m = min(m, o); M = max(M, o);
        }
        m = __reduce_min_sync(0xffffffffu, m);
        M = __reduce_max_sync(0xffffffffu, M);
        const float cmin = std_min(3.402823466e38f, ord2f(m));
        const float cmax = std_max(-3.402823466e38f, ord2f(M));
        if (cmax - cmin < C.centroid_eps) { continue; }
        const float scale = (float)nb / (cmax - cmin);
        for (int b = lane; b < nb; b += 32) { S.cnt[b] = 0u; sbox_clear(S.bins[b]); }
        __syncwarp();
        for (uint32_t i = lane; i < n; i += 32)
        {
            const int b = obj_bin(src.cen(i, axis), cmin, scale, nb);
            atomicAdd(&S.cnt[b], 1u);
            sbox_add(S.bins[b], src.box(i));
        }
        __syncwarp();
        warp_eval_object_axis(S.cnt, S.bins, nb, axis, cmin, scale, parent_inv_area, C, Bw);
        __syncwarp();
    }
    const int oa = Bw.axis, ob = Bw.bin;
    const float oc = Bw.cmin, os = Bw.scale;
    // phase 2: spatial bins over the node box, triangles clipped per bin (bvh_sah.cpp:135-243)
    const bool prune = C.c_isect >= 0.f;  // (the bound needs a cost monotone in the areas)
    for (int axis = 0; axis < 3; axis++)
    {
        const float node_min = nbox.mn[axis], node_max = nbox.mx[axis];
        if (node_max - node_min < C.spatial_eps) { continue; }
        const float sscale = (float)nb / (node_max - node_min);
        for (int b = lane; b < nb; b += 32) { S.cin[b] = 0u; S.cout[b] = 0u; sbox_clear(S.bins[b]); }
        bin_bounds(S.bnd, node_min, sscale, nb, lane, 32);
        __syncwarp();
        if (prune)
        {
            for (uint32_t i0 = 0; i0 < n; i0 += 32)
            {
                spatial_bound_warp(src, i0, n, axis, nbox, node_min, sscale, nb, S.bnd, S.cin, S.cout, S.bins);
            }
            __syncwarp();
            const bool can = warp_spatial_can_win(S.cin, S.cout, S.bins, nb, parent_inv_area, C, Bw.cost);
            __syncwarp();
            if (!can) { continue; }
            for (int b = lane; b < nb; b += 32) { sbox_clear(S.bins[b]); }  // the exact boxes; the counts stay
            __syncwarp();
        }
        for (uint32_t i0 = 0; i0 < n; i0 += 32)
        {
            spatial_bin_warp(src, i0, n, axis, nbox, node_min, sscale, nb, S.bnd, S.cin, S.cout, S.bins, !prune);
        }
        __syncwarp();
        warp_eval_spatial_axis(S.cin, S.cout, S.bins, nb, axis, node_min, sscale, parent_inv_area, C, Bw);
        __syncwarp();
    }
    // decision and partition side counts (bvh_sah.cpp:249-394)
    const Best B = Bw;
    d.nb = nb;
    d.oaxis = oa; d.obin = ob; d.ocmin = oc; d.oscale = os;
    if (B.axis == -1)
    {
        d.kind = K_LEAF;
    }
    else if (!B.spatial)
    {
        uint32_t l = 0;
        for (uint32_t i = lane; i < n; i += 32)
        {
            l += obj_bin(src.cen(i, B.axis), B.cmin, B.scale, nb) < B.bin ? 1u : 0u;
        }
        l = __reduce_add_sync(0xffffffffu, l);
        d.kind = (l == 0 || l == n) ? K_LEAF : K_OBJECT;
        d.oleft = l;
        d.axis = B.axis; d.bin = B.bin; d.cmin = B.cmin; d.scale = B.scale;
    }
    else
    {
        const float plane = B.node_min + (float)B.bin / B.sscale;
        const int axis = B.axis;
        uint32_t lo_ = 0, st_ = 0, ol = 0;
        for (uint32_t i = lane; i < n; i += 32)
        {
            if (src.hi_of(i, axis) <= plane) { lo_++; }
            else if (src.lo_of(i, axis) < plane) { st_++; }
            if (oa != -1) { ol += obj_bin(src.cen(i, oa), oc, os, nb) < ob ? 1u : 0u; }
        }
        lo_ = __reduce_add_sync(0xffffffffu, lo_);
        st_ = __reduce_add_sync(0xffffffffu, st_);
        ol = __reduce_add_sync(0xffffffffu, ol);
        const uint32_t ri = n - lo_ - st_;
        const int fb = (oa == -1 || ol == 0 || ol == n) ? K_LEAF : K_OBJECT;
        d.sp_axis = axis; d.plane = plane; d.straddle = st_; d.right = ri; d.fb_kind = fb; d.oleft = ol;
        if ((lo_ + st_ == 0) || (st_ + ri == 0))
        {
            // the saved object split, applied after the spatial partitions (bvh_sah.cpp:331-333)
            d.kind = fb; d.pre_spatial = 1;
            d.axis = oa; d.bin = ob; d.cmin = oc; d.scale = os;
        }
        else
        {
            d.kind = K_SPATIAL;
            d.axis = axis;
        }
    }
}

// STAGED: the nodes of at most EVAL_STAGE references (leaves included), read from a shared
// copy; else the nodes of EVAL_STAGE + 1 .. WARP_MAX references, read from global memory.
// Each warp takes the level's nodes one at a time from a counter (*ctr, zero at launch), so a
// warp that meets leaves or another kernel's nodes moves on at once and the grid need only
// fill the GPU.
template <bool STAGED>
__global__ void __launch_bounds__(EVAL_WPB * 32, 4)  // (64 registers: occupancy over spills)
k_sah_eval_warp(const LvlNode* __restrict__ lv, const uint32_t* __restrict__ refs, Ctx C, Dec* __restrict__ dec,
                uint32_t n_lvl, uint32_t* __restrict__ ctr)
{
    __shared__ EvalWS ws[EVAL_WPB];
    __shared__ StageBuf stage[STAGED ? EVAL_WPB : 1];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;)
    {
        uint32_t node = 0;
        if (lane == 0) { node = atomicAdd(ctr, 1u); }
        node = __shfl_sync(0xffffffffu, node, 0);
        if (node >= n_lvl) { return; }
        const LvlNode nd = lv[node];
        const uint32_t n = nd.count;
        if (STAGED ? n > EVAL_STAGE : (n <= EVAL_STAGE || n > WARP_MAX)) { continue; }  // another kernel's node
        const uint32_t* R = refs + nd.ref_off;
        Dec d;
        memset(&d, 0, sizeof(d));
        d.n = n;
        if (n <= C.max_leaf)
        {
            if (lane == 0) { d.kind = K_LEAF; dec[node] = d; }
            continue;
        }
        if constexpr (STAGED)
        {
            stage_refs(C, R, n, stage[w]);
            eval_node_warp(StagedRefs{ &stage[w], R }, nd, n, C, ws[w], d);
        }
        else
        {
            eval_node_warp(GlobalRefs(C, R), nd, n, C, ws[w], d);
        }
        if (lane == 0) { dec[node] = d; }
        __syncwarp();  // every lane done with the shared copy and bins before the next node
    }
}

// One block per node: evaluates every object and spatial candidate in the reference's order
// and writes the decision with the side counts of its partitions.
__global__ void __launch_bounds__(SBLK)
k_sah_eval(const LvlNode* __restrict__ lv, const uint32_t* __restrict__ refs, Ctx C, Dec* __restrict__ dec)
{
    __shared__ uint32_t cnt[SAH_MAX_BINS], cin[SAH_MAX_BINS], cout[SAH_MAX_BINS];
    __shared__ SBox bins[SAH_MAX_BINS];
    __shared__ float bnd[SAH_MAX_BINS + 1];
    __shared__ uint32_t s_red[SBLK / 32 + 1];
    __shared__ uint32_t s_cm, s_cM;
    __shared__ Best sB;
    __shared__ int o_axis, o_bin, s_can;
    __shared__ float o_cmin, o_scale;

    const LvlNode nd = lv[blockIdx.x];
    const uint32_t n = nd.count;
    const uint32_t* R = refs + nd.ref_off;
    const int tid = threadIdx.x;
    Dec d;
    memset(&d, 0, sizeof(d));
    d.n = n;
    if (n <= WARP_MAX || n > WIDE_MIN) { return; }  // k_sah_eval_warp or the wide kernels decide this node
    if (n <= C.max_leaf)
    {
        if (tid == 0) { d.kind = K_LEAF; dec[blockIdx.x] = d; }
        return;
    }
    const int nb = std_clampi((int)n / 4, (int)C.bins_min, (int)C.bins_max);
    box3 nbox;
    for (int k = 0; k < 3; k++) { nbox.mn[k] = nd.box[k]; nbox.mx[k] = nd.box[3 + k]; }
    const float parent_inv_area = 1.0f / box_half_area(nbox);
    if (tid == 0)
    {
        sB.cost = C.c_isect * (float)n;  // leaf cost, bvh_sah.cpp:32
        sB.axis = -1; sB.bin = -1; sB.cmin = 0.f; sB.scale = 0.f; sB.spatial = 0; sB.node_min = 0.f; sB.sscale = 0.f;
    }

    // phase 1: centroid-binned object split (bvh_sah.cpp:52-126)
    for (int axis = 0; axis < 3; axis++)
    {
        if (tid == 0) { s_cm = 0xffffffffu; s_cM = 0u; }
        __syncthreads();
        uint32_t m = 0xffffffffu, M = 0u;
        for (uint32_t i = tid; i < n; i += SBLK)
        {
            const uint32_t o = f2ord(centroid(C, R[i], axis));
            m = min(m, o); M = max(M, o);
        }
        atomicMin(&s_cm, m); atomicMax(&s_cM, M);
        __syncthreads();
        // std::min / std::max folds starting from +FLT_MAX / -FLT_MAX (bvh_sah.cpp:54-61)
        const float cmin = std_min(3.402823466e38f, ord2f(s_cm));
        const float cmax = std_max(-3.402823466e38f, ord2f(s_cM));
        __syncthreads();  // everyone has read s_cm / s_cM before the next axis resets them
        if (cmax - cmin < C.centroid_eps) { continue; }
        const float scale = (float)nb / (cmax - cmin);
        if (tid < nb) { cnt[tid] = 0u; sbox_clear(bins[tid]); }
        __syncthreads();
        for (uint32_t i = tid; i < n; i += SBLK)
        {
            const uint32_t t = R[i];
            const int b = obj_bin(centroid(C, t, axis), cmin, scale, nb);
            atomicAdd(&cnt[b], 1u);
            sbox_add(bins[b], tri_box(C, t));
        }
        __syncthreads();
        if (tid < 32)
        {
            Best b = sB;
            warp_eval_object_axis(cnt, bins, nb, axis, cmin, scale, parent_inv_area, C, b);
            if (tid == 0) { sB = b; }
        }
        __syncthreads();
    }
    if (tid == 0) { o_axis = sB.axis; o_bin = sB.bin; o_cmin = sB.cmin; o_scale = sB.scale; }
    __syncthreads();

    // phase 2: spatial bins over the node box, triangles clipped per bin (bvh_sah.cpp:135-243)
    const bool prune = C.c_isect >= 0.f;  // (the bound needs a cost monotone in the areas)
    for (int axis = 0; axis < 3; axis++)
    {
        const float node_min = nbox.mn[axis], node_max = nbox.mx[axis];
        if (node_max - node_min < C.spatial_eps) { continue; }
        const float sscale = (float)nb / (node_max - node_min);
        if (tid < nb) { cin[tid] = 0u; cout[tid] = 0u; sbox_clear(bins[tid]); }
        bin_bounds(bnd, node_min, sscale, nb, tid, SBLK);
        __syncthreads();
        if (prune)
        {
            // the lower bounds first (spatial_bound_warp): skip the clipping when none can win
            for (uint32_t i0 = (uint32_t)(tid & ~31); i0 < n; i0 += SBLK)
            {
                spatial_bound_warp(GlobalRefs(C, R), i0, n, axis, nbox, node_min, sscale, nb, bnd, cin, cout, bins);
            }
            __syncthreads();
            if (tid < 32)
            {
                const bool can = warp_spatial_can_win(cin, cout, bins, nb, parent_inv_area, C, sB.cost);
                if (tid == 0) { s_can = can ? 1 : 0; }
            }
            __syncthreads();
            if (!s_can) { continue; }
            if (tid < nb) { sbox_clear(bins[tid]); }
            __syncthreads();
        }
        for (uint32_t i0 = (uint32_t)(tid & ~31); i0 < n; i0 += SBLK)
        {
            spatial_bin_warp(GlobalRefs(C, R), i0, n, axis, nbox, node_min, sscale, nb, bnd, cin, cout, bins, !prune);
        }
        __syncthreads();
        if (tid < 32)
        {
            Best b = sB;
            warp_eval_spatial_axis(cin, cout, bins, nb, axis, node_min, sscale, parent_inv_area, C, b);
            if (tid == 0) { sB = b; }
        }
        __syncthreads();
    }

    // decision and partition side counts (bvh_sah.cpp:249-394)
    const Best B = sB;
    d.nb = nb;
    d.oaxis = o_axis; d.obin = o_bin; d.ocmin = o_cmin; d.oscale = o_scale;
    if (B.axis == -1)
    {
        d.kind = K_LEAF;
    }
    else if (!B.spatial)
    {
        uint32_t l = 0;
        for (uint32_t i = tid; i < n; i += SBLK)
        {
            l += obj_bin(centroid(C, R[i], B.axis), B.cmin, B.scale, nb) < B.bin ? 1u : 0u;
        }
        l = block_sum<SBLK>(l, s_red);
        d.kind = (l == 0 || l == n) ? K_LEAF : K_OBJECT;
        d.oleft = l;
        d.axis = B.axis; d.bin = B.bin; d.cmin = B.cmin; d.scale = B.scale;
    }
    else
    {
        const float plane = B.node_min + (float)B.bin / B.sscale;
        const int axis = B.axis;
        const int oa = o_axis, ob = o_bin;
        const float oc = o_cmin, os = o_scale;
        uint32_t lo_ = 0, st_ = 0, ol = 0;
        for (uint32_t i = tid; i < n; i += SBLK)
        {
            const uint32_t t = R[i];
            if (tri_hi(C, t, axis) <= plane) { lo_++; }
            else if (tri_lo(C, t, axis) < plane) { st_++; }
            if (oa != -1) { ol += obj_bin(centroid(C, t, oa), oc, os, nb) < ob ? 1u : 0u; }
        }
        lo_ = block_sum<SBLK>(lo_, s_red);
        st_ = block_sum<SBLK>(st_, s_red);
        ol = block_sum<SBLK>(ol, s_red);
        const uint32_t ri = n - lo_ - st_;
        const int fb = (oa == -1 || ol == 0 || ol == n) ? K_LEAF : K_OBJECT;
        d.sp_axis = axis; d.plane = plane; d.straddle = st_; d.right = ri; d.fb_kind = fb; d.oleft = ol;
        if ((lo_ + st_ == 0) || (st_ + ri == 0))
        {
            // the saved object split, applied after the spatial partitions (bvh_sah.cpp:331-333)
            d.kind = fb; d.pre_spatial = 1;
            d.axis = oa; d.bin = ob; d.cmin = oc; d.scale = os;
        }
        else
        {
            d.kind = K_SPATIAL;
            d.axis = axis;
        }
    }
    if (tid == 0) { dec[blockIdx.x] = d; }
}

// ---- the wide path: nodes with more than WIDE_MIN references ----
// The top levels of a large build hold a few nodes with up to millions of references. Their
// candidates are binned by many blocks at once (WIDE_CH references each) into per-node bins in
// global memory -- counts by atomic adds, boxes by atomic min / max on the order-preserving
// encoding, which are the same values the one-block path accumulates in shared memory -- and
// then evaluated by one thread per node with the same serial code, so the decisions are the
// ones the one-block path makes.
constexpr uint32_t WIDE_CH = 4096;

struct WideAcc
{
    uint32_t cm[3], cM[3];
    uint32_t ocnt[3][SAH_MAX_BINS];
    SBox     obox[3][SAH_MAX_BINS];
    uint32_t cin[3][SAH_MAX_BINS], cout[3][SAH_MAX_BINS];
    SBox     sbox[3][SAH_MAX_BINS];
    uint32_t cnt[4];
    Best     B;
    int      o_axis, o_bin;
    float    o_cmin, o_scale;
    // the partitions (k_wp_*): per pass the satisfied count and the swapped pairs; child boxes
    uint32_t pm[3], ftot[3];
    SBox     cb[2];
};

// The wide nodes of a level in level order (wl) with their first block (wco, exclusive prefix
// of ceil(count / WIDE_CH)); io[8] = wide nodes, io[9] = blocks.
__global__ void __launch_bounds__(1024)
k_wide_list(const LvlNode* __restrict__ lv, uint32_t n_lvl, uint32_t* __restrict__ wl, uint32_t* __restrict__ wco,
            uint32_t max_wide, uint32_t* __restrict__ io)
{
    __shared__ uint32_t sh[33];
    uint32_t nw = 0, nch = 0;
    for (uint32_t base = 0; base < n_lvl; base += 1024)
    {
        const uint32_t i = base + threadIdx.x;
        const uint32_t n = i < n_lvl ? lv[i].count : 0u;
        const uint32_t f = n > WIDE_MIN ? 1u : 0u;
        const uint32_t c = f ? (n + WIDE_CH - 1) / WIDE_CH : 0u;
        uint32_t tf, tc;
        const uint32_t ef = block_excl_scan<1024>(f, sh, &tf);
        const uint32_t ec = block_excl_scan<1024>(c, sh, &tc);
        if (f && nw + ef < max_wide) { wl[nw + ef] = i; wco[nw + ef] = nch + ec; }
        nw += tf;
        nch += tc;
    }
    if (threadIdx.x == 0)
    {
        if (nw <= max_wide) { wco[nw] = nch; }
        io[8] = nw;
        io[9] = nch;
    }
}

// wide node k and chunk c of block g
__device__ __forceinline__ uint32_t wide_item(const uint32_t* __restrict__ wco, uint32_t nw, uint32_t g, uint32_t& c)
{
    uint32_t lo = 0, hi = nw;  // wco[lo] <= g < wco[hi]
    while (hi - lo > 1)
    {
        const uint32_t mid = (lo + hi) >> 1;
        if (wco[mid] <= g) { lo = mid; } else { hi = mid; }
    }
    c = g - wco[lo];
    return lo;
}

__global__ void __launch_bounds__(SBLK) k_wide_init(WideAcc* __restrict__ acc)
{
    WideAcc& A = acc[blockIdx.x];
    uint32_t* w = reinterpret_cast<uint32_t*>(&A);
    // counts 0, box minima ~0: the SBox members are written below
    for (uint32_t i = threadIdx.x; i < sizeof(WideAcc) / 4; i += SBLK) { w[i] = 0u; }
    __syncthreads();
    if (threadIdx.x < 3) { A.cm[threadIdx.x] = 0xffffffffu; A.cM[threadIdx.x] = 0u; }
    for (uint32_t j = threadIdx.x; j < 3 * SAH_MAX_BINS; j += SBLK)
    {
        sbox_clear(A.obox[j / SAH_MAX_BINS][j % SAH_MAX_BINS]);
        sbox_clear(A.sbox[j / SAH_MAX_BINS][j % SAH_MAX_BINS]);
    }
    if (threadIdx.x < 2) { sbox_clear(A.cb[threadIdx.x]); }
}

__device__ __forceinline__ void chunk_range(uint32_t n, uint32_t c, uint32_t& b, uint32_t& e)
{
    b = c * WIDE_CH;
    e = min(n, b + WIDE_CH);
}

// centroid bounds per axis
__global__ void __launch_bounds__(SBLK)
k_wide_bounds(const LvlNode* __restrict__ lv, const uint32_t* __restrict__ refs, Ctx C, const uint32_t* __restrict__ wl,
              const uint32_t* __restrict__ wco, uint32_t nw, WideAcc* __restrict__ acc)
{
    __shared__ uint32_t sm[3], sM[3];
    uint32_t c;
    const uint32_t k = wide_item(wco, nw, blockIdx.x, c);
    const LvlNode nd = lv[wl[k]];
    const uint32_t* R = refs + nd.ref_off;
    uint32_t b, e;
    chunk_range(nd.count, c, b, e);
    if (threadIdx.x < 3) { sm[threadIdx.x] = 0xffffffffu; sM[threadIdx.x] = 0u; }
    __syncthreads();
    uint32_t m[3] = { 0xffffffffu, 0xffffffffu, 0xffffffffu }, M[3] = { 0u, 0u, 0u };
    for (uint32_t i = b + threadIdx.x; i < e; i += SBLK)
    {
        const uint32_t t = R[i];
        for (int a = 0; a < 3; a++)
        {
            const uint32_t o = f2ord(centroid(C, t, a));
            m[a] = min(m[a], o); M[a] = max(M[a], o);
        }
    }
    for (int a = 0; a < 3; a++)
    {
        for (int o = 16; o > 0; o >>= 1)
        {
            m[a] = min(m[a], __shfl_xor_sync(0xffffffffu, m[a], o));
            M[a] = max(M[a], __shfl_xor_sync(0xffffffffu, M[a], o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&sm[a], m[a]); atomicMax(&sM[a], M[a]); }
    }
    __syncthreads();
    if (threadIdx.x < 3)
    {
        atomicMin(&acc[k].cm[threadIdx.x], sm[threadIdx.x]);
        atomicMax(&acc[k].cM[threadIdx.x], sM[threadIdx.x]);
    }
}

__device__ __forceinline__ void wide_axis_scale(const WideAcc& A, int axis, int nb, const Ctx& C, float& cmin, float& scale)
{
    // std::min / std::max folds starting from +FLT_MAX / -FLT_MAX (bvh_sah.cpp:54-61)
    cmin = std_min(3.402823466e38f, ord2f(A.cm[axis]));
    const float cmax = std_max(-3.402823466e38f, ord2f(A.cM[axis]));
    scale = (cmax - cmin < C.centroid_eps) ? 0.f : (float)nb / (cmax - cmin);
}

__device__ __forceinline__ void sbox_merge_global(SBox& g, const SBox& s)
{
    if (s.m[0] == 0xffffffffu && s.M[0] == 0u) { return; }  // nothing added
    for (int k = 0; k < 3; k++) { atomicMin(&g.m[k], s.m[k]); atomicMax(&g.M[k], s.M[k]); }
}

// object bins of the three axes and spatial bins with clipping, one chunk per block
__global__ void __launch_bounds__(SBLK)
k_wide_bins(const LvlNode* __restrict__ lv, const uint32_t* __restrict__ refs, Ctx C, const uint32_t* __restrict__ wl,
            const uint32_t* __restrict__ wco, uint32_t nw, WideAcc* __restrict__ acc)
{
    __shared__ uint32_t ocnt[3][SAH_MAX_BINS], cin[3][SAH_MAX_BINS], cout[3][SAH_MAX_BINS];
    __shared__ SBox obox[3][SAH_MAX_BINS], sbx[3][SAH_MAX_BINS];
    __shared__ float bnd[3][SAH_MAX_BINS + 1];
    uint32_t c;
    const uint32_t k = wide_item(wco, nw, blockIdx.x, c);
    const LvlNode nd = lv[wl[k]];
    const uint32_t n = nd.count;
    const uint32_t* R = refs + nd.ref_off;
    uint32_t b0, e0;
    chunk_range(n, c, b0, e0);
    const int nb = std_clampi((int)n / 4, (int)C.bins_min, (int)C.bins_max);
    WideAcc& A = acc[k];
    float cmin[3], scale[3], node_min[3], sscale[3];
    box3 nbox;
    for (int a = 0; a < 3; a++)
    {
        wide_axis_scale(A, a, nb, C, cmin[a], scale[a]);
        nbox.mn[a] = nd.box[a]; nbox.mx[a] = nd.box[3 + a];
        node_min[a] = nd.box[a];
        const float node_max = nd.box[3 + a];
        sscale[a] = (node_max - node_min[a] < C.spatial_eps) ? 0.f : (float)nb / (node_max - node_min[a]);
    }
    for (uint32_t j = threadIdx.x; j < 3 * SAH_MAX_BINS; j += SBLK)
    {
        const uint32_t a = j / SAH_MAX_BINS, bb = j % SAH_MAX_BINS;
        ocnt[a][bb] = 0u; cin[a][bb] = 0u; cout[a][bb] = 0u;
        sbox_clear(obox[a][bb]); sbox_clear(sbx[a][bb]);
    }
    for (int a = 0; a < 3; a++)
    {
        if (sscale[a] != 0.f) { bin_bounds(bnd[a], node_min[a], sscale[a], nb, threadIdx.x, SBLK); }
    }
    __syncthreads();
    for (uint32_t i = b0 + threadIdx.x; i < e0; i += SBLK)
    {
        const uint32_t t = R[i];
        const box3 tb = tri_box(C, t);
        for (int a = 0; a < 3; a++)
        {
            if (scale[a] == 0.f) { continue; }
            const int b = obj_bin(centroid(C, t, a), cmin[a], scale[a], nb);
            atomicAdd(&ocnt[a][b], 1u);
            sbox_add(obox[a][b], tb);
        }
        f3 v0, v1, v2;
        bool have_v = false;
        const float top = (float)(nb - 1);
        for (int a = 0; a < 3; a++)
        {
            if (sscale[a] == 0.f) { continue; }
            const int bmin = bin_clamp((tri_lo(C, t, a) - node_min[a]) * sscale[a], top);
            const int bmax = bin_clamp((tri_hi(C, t, a) - node_min[a]) * sscale[a], top);
            atomicAdd(&cin[a][bmin], 1u);
            atomicAdd(&cout[a][bmax], 1u);
            if (bmin <= bmax)
            {
                if (!have_v) { tri_verts(C, t, v0, v1, v2); have_v = true; }
                box3 region = nbox;
                for (int b = bmin; b <= bmax; b++)
                {
                    region.mn[a] = bnd[a][b];
                    region.mx[a] = bnd[a][b + 1];
                    const box3 cl = clip_triangle(v0, v1, v2, region);
                    if (box_valid(cl)) { sbox_add(sbx[a][b], cl); }
                }
            }
        }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < 3 * SAH_MAX_BINS; j += SBLK)
    {
        const uint32_t a = j / SAH_MAX_BINS, bb = j % SAH_MAX_BINS;
        if (ocnt[a][bb]) { atomicAdd(&A.ocnt[a][bb], ocnt[a][bb]); }
        if (cin[a][bb]) { atomicAdd(&A.cin[a][bb], cin[a][bb]); }
        if (cout[a][bb]) { atomicAdd(&A.cout[a][bb], cout[a][bb]); }
        sbox_merge_global(A.obox[a][bb], obox[a][bb]);
        sbox_merge_global(A.sbox[a][bb], sbx[a][bb]);
    }
}

// the candidate evaluation over the accumulated bins, one warp per node
__global__ void __launch_bounds__(32) k_wide_decide(const LvlNode* __restrict__ lv, Ctx C, const uint32_t* __restrict__ wl,
                                                    uint32_t nw, WideAcc* __restrict__ acc)
{
    const uint32_t k = blockIdx.x;
    if (k >= nw) { return; }
    const LvlNode nd = lv[wl[k]];
    const uint32_t n = nd.count;
    WideAcc& A = acc[k];
    const int nb = std_clampi((int)n / 4, (int)C.bins_min, (int)C.bins_max);
    box3 nbox;
    for (int a = 0; a < 3; a++) { nbox.mn[a] = nd.box[a]; nbox.mx[a] = nd.box[3 + a]; }
    const float parent_inv_area = 1.0f / box_half_area(nbox);
    Best B;
    B.cost = C.c_isect * (float)n;  // leaf cost, bvh_sah.cpp:32
    B.axis = -1; B.bin = -1; B.cmin = 0.f; B.scale = 0.f; B.spatial = 0; B.node_min = 0.f; B.sscale = 0.f;
    for (int a = 0; a < 3; a++)
    {
        float cmin, scale;
        wide_axis_scale(A, a, nb, C, cmin, scale);
        if (scale == 0.f) { continue; }
        warp_eval_object_axis(A.ocnt[a], A.obox[a], nb, a, cmin, scale, parent_inv_area, C, B);
    }
    if (threadIdx.x == 0) { A.o_axis = B.axis; A.o_bin = B.bin; A.o_cmin = B.cmin; A.o_scale = B.scale; }
    for (int a = 0; a < 3; a++)
    {
        const float node_min = nbox.mn[a], node_max = nbox.mx[a];
        if (node_max - node_min < C.spatial_eps) { continue; }
        const float sscale = (float)nb / (node_max - node_min);
        warp_eval_spatial_axis(A.cin[a], A.cout[a], A.sbox[a], nb, a, node_min, sscale, parent_inv_area, C, B);
    }
    if (threadIdx.x == 0) { A.B = B; }
}

// partition side counts of the chosen candidate
__global__ void __launch_bounds__(SBLK)
k_wide_counts(const LvlNode* __restrict__ lv, const uint32_t* __restrict__ refs, Ctx C, const uint32_t* __restrict__ wl,
              const uint32_t* __restrict__ wco, uint32_t nw, WideAcc* __restrict__ acc)
{
    __shared__ uint32_t sh[SBLK / 32 + 1];
    uint32_t c;
    const uint32_t k = wide_item(wco, nw, blockIdx.x, c);
    const LvlNode nd = lv[wl[k]];
    const uint32_t n = nd.count;
    const uint32_t* R = refs + nd.ref_off;
    WideAcc& A = acc[k];
    const Best B = A.B;
    if (B.axis == -1) { return; }
    uint32_t b0, e0;
    chunk_range(n, c, b0, e0);
    const int nb = std_clampi((int)n / 4, (int)C.bins_min, (int)C.bins_max);
    if (!B.spatial)
    {
        uint32_t l = 0;
        for (uint32_t i = b0 + threadIdx.x; i < e0; i += SBLK)
        {
            l += obj_bin(centroid(C, R[i], B.axis), B.cmin, B.scale, nb) < B.bin ? 1u : 0u;
        }
        l = block_sum<SBLK>(l, sh);
        if (threadIdx.x == 0 && l) { atomicAdd(&A.cnt[0], l); }
        return;
    }
    const float plane = B.node_min + (float)B.bin / B.sscale;
    const int axis = B.axis;
    const int oa = A.o_axis, ob = A.o_bin;
    const float oc = A.o_cmin, os = A.o_scale;
    uint32_t lo_ = 0, st_ = 0, ol = 0;
    for (uint32_t i = b0 + threadIdx.x; i < e0; i += SBLK)
    {
        const uint32_t t = R[i];
        if (tri_hi(C, t, axis) <= plane) { lo_++; }
        else if (tri_lo(C, t, axis) < plane) { st_++; }
        if (oa != -1) { ol += obj_bin(centroid(C, t, oa), oc, os, nb) < ob ? 1u : 0u; }
    }
    lo_ = block_sum<SBLK>(lo_, sh);
    st_ = block_sum<SBLK>(st_, sh);
    ol = block_sum<SBLK>(ol, sh);
    if (threadIdx.x == 0)
    {
        if (lo_) { atomicAdd(&A.cnt[0], lo_); }
        if (st_) { atomicAdd(&A.cnt[1], st_); }
        if (ol) { atomicAdd(&A.cnt[2], ol); }
    }
}

// the decision record, as the one-block path writes it (bvh_sah.cpp:249-394)
__global__ void k_wide_final(const LvlNode* __restrict__ lv, Ctx C, const uint32_t* __restrict__ wl, uint32_t nw,
                             const WideAcc* __restrict__ acc, Dec* __restrict__ dec)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nw) { return; }
    const uint32_t node = wl[k];
    const uint32_t n = lv[node].count;
    const WideAcc& A = acc[k];
    const Best B = A.B;
    Dec d;
    memset(&d, 0, sizeof(d));
    d.n = n;
    d.nb = std_clampi((int)n / 4, (int)C.bins_min, (int)C.bins_max);
    d.oaxis = A.o_axis; d.obin = A.o_bin; d.ocmin = A.o_cmin; d.oscale = A.o_scale;
    if (B.axis == -1)
    {
        d.kind = K_LEAF;
    }
    else if (!B.spatial)
    {
        const uint32_t l = A.cnt[0];
        d.kind = (l == 0 || l == n) ? K_LEAF : K_OBJECT;
        d.oleft = l;
        d.axis = B.axis; d.bin = B.bin; d.cmin = B.cmin; d.scale = B.scale;
    }
    else
    {
        const uint32_t lo_ = A.cnt[0], st_ = A.cnt[1], ol = A.cnt[2];
        const uint32_t ri = n - lo_ - st_;
        const int fb = (A.o_axis == -1 || ol == 0 || ol == n) ? K_LEAF : K_OBJECT;
        d.sp_axis = B.axis; d.plane = B.node_min + (float)B.bin / B.sscale; d.straddle = st_; d.right = ri; d.fb_kind = fb; d.oleft = ol;
        if ((lo_ + st_ == 0) || (st_ + ri == 0))
        {
            // the saved object split, applied after the spatial partitions (bvh_sah.cpp:331-333)
            d.kind = fb; d.pre_spatial = 1;
            d.axis = A.o_axis; d.bin = A.o_bin; d.cmin = A.o_cmin; d.scale = A.o_scale;
        }
        else
        {
            d.kind = K_SPATIAL;
            d.axis = B.axis;
        }
    }
    dec[node] = d;
}

// The spatial-split reference budget and the next level's layout, in three launches.
// Each scene of a batched build has its own budget (used[s] of cap[s]), as a bake of that
// scene alone would; the scene of level node i is that of its subtree root.
//   k_sah_need    sums every scene's requests (right + straddle references of each spatial
//                 candidate) over the level;
//   k_sah_grant   grants them all when every scene's requests fit, else walks the candidates
//                 in queue order (a refused request leaves the budget to later, smaller ones);
//   k_sah_offsets allocates child slots (2 per split node), next-level references and
//                 leaf-store space by a one-pass prefix scan.
// io: [1] spatial taken, [2] spatial refused, [3] next-level nodes, [4] next-level references,
//     [5] leaf-store entries of this level, [6] leaves, [10] largest next-level node,
//     [7] every spatial candidate of the level refused, [11] spatial candidates of the level,
//     [12] status (a bounded wait gave up), [13] / [14] the warp evaluations' node counters,
//     [15] the smallest request of the level
constexpr uint32_t MAX_BUDGET_SCENES = 1024;
constexpr int NEED_THREADS = 256;

__global__ void __launch_bounds__(NEED_THREADS)
k_sah_need(const Dec* __restrict__ dec, const LvlNode* __restrict__ lv, const SahRoot* __restrict__ roots, uint32_t n_lvl,
           uint32_t n_scenes, unsigned long long* __restrict__ need, uint32_t* __restrict__ io)
{
    __shared__ uint32_t sh[NEED_THREADS / 32 + 1];
    const uint32_t i = blockIdx.x * NEED_THREADS + threadIdx.x;
    uint32_t nd = 0, sp = 0, mn = 0xffffffffu;
    if (i < n_lvl && dec[i].kind == K_SPATIAL)
    {
        nd = dec[i].right + dec[i].straddle;
        mn = nd;
        sp = 1;
        if (n_scenes > 1)
        {
            atomicAdd(&need[min(roots[lv[i].root].scene, n_scenes - 1u)], (unsigned long long)nd);
            nd = 0;
        }
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    if ((threadIdx.x & 31) == 0 && mn != 0xffffffffu) { atomicMin(&io[15], mn); }
    // one scene: one addition per block (a level's references fit 32 bits)
    nd = block_sum<NEED_THREADS>(nd, sh);
    sp = block_sum<NEED_THREADS>(sp, sh);
    if (threadIdx.x == 0)
    {
        if (nd) { atomicAdd(&need[0], (unsigned long long)nd); }
        if (sp) { atomicAdd(&io[11], sp); }
    }
}

// One block. Afterwards need[], io[10], io[11] and the offset scan's descriptors and ticket
// (3 * n_tiles + 1 words) are zero for the next launches.
__global__ void __launch_bounds__(1024)
k_sah_grant(Dec* __restrict__ dec, const LvlNode* __restrict__ lv, const SahRoot* __restrict__ roots, uint32_t n_lvl,
            uint32_t n_scenes, uint32_t* __restrict__ used, const uint32_t* __restrict__ cap,
            unsigned long long* __restrict__ need, uint32_t* __restrict__ io, uint32_t* __restrict__ leaf_off,
            unsigned long long* __restrict__ desc, uint32_t n_tiles)
{
    __shared__ uint32_t sh[33];
    __shared__ int s_all;
    const int tid = threadIdx.x;
    if (tid == 0) { s_all = 1; io[7] = 0u; }
    __syncthreads();
    for (uint32_t k = tid; k < n_scenes; k += 1024)
    {
        if ((unsigned long long)used[k] + need[k] > (unsigned long long)cap[k]) { s_all = 0; }
    }
    __syncthreads();
    if (s_all)
    {
        for (uint32_t k = tid; k < n_scenes; k += 1024) { used[k] = (uint32_t)(used[k] + need[k]); }
        if (tid == 0) { io[1] += io[11]; }
    }
    else if (n_scenes == 1 && (unsigned long long)used[0] + io[15] > (unsigned long long)cap[0])
    {
        // not even the smallest request fits: k_sah_offsets refuses every candidate
        if (tid == 0) { io[7] = 1u; }
    }
    else
    {
        // The grants are sequential (a refused request leaves the budget to later, smaller
        // ones), so one thread walks the spatial candidates in queue order -- compacted first,
        // and with one scene it stops as soon as even the smallest request no longer fits;
        // the rest are refused in parallel. leaf_off serves as the candidate list here (it is
        // filled only further down).
        __shared__ uint32_t s_ns, s_stop, s_minneed;
        uint32_t ns = 0, mn = 0xffffffffu;
        for (uint32_t base = 0; base < n_lvl; base += 1024)
        {
            const uint32_t i = base + tid;
            uint32_t f = 0;
            if (i < n_lvl)
            {
                const Dec d = dec[i];
                if (d.kind == K_SPATIAL) { f = 1; mn = min(mn, d.right + d.straddle); }
            }
            uint32_t tot;
            const uint32_t e = block_excl_scan<1024>(f, sh, &tot);
            if (f) { leaf_off[ns + e] = i; }
            ns += tot;
        }
        for (int o = 16; o > 0; o >>= 1) { mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o)); }
        if (tid == 0) { s_minneed = 0xffffffffu; s_ns = ns; }
        __syncthreads();
        if ((tid & 31) == 0) { atomicMin(&s_minneed, mn); }
        __syncthreads();
        if (tid == 0)
        {
            const uint32_t min_need = s_minneed;
            uint32_t j = 0;
            for (; j < s_ns; j++)
            {
                if (n_scenes == 1 && (unsigned long long)used[0] + min_need > (unsigned long long)cap[0]) { break; }
                const uint32_t i = leaf_off[j];
                Dec d = dec[i];
                const uint32_t sc = min(roots[lv[i].root].scene, n_scenes - 1u);
                const uint32_t nd = d.right + d.straddle;
                if ((unsigned long long)used[sc] + nd > (unsigned long long)cap[sc])
                {
                    d.kind = d.fb_kind; d.pre_spatial = 1;
                    d.axis = d.oaxis; d.bin = d.obin; d.cmin = d.ocmin; d.scale = d.oscale;
                    dec[i] = d;
                    io[2]++;
                }
                else
                {
                    used[sc] += nd;
                    io[1]++;
                }
            }
            s_stop = j;
        }
        __syncthreads();
        uint32_t refused = 0;
        for (uint32_t j = s_stop + tid; j < s_ns; j += 1024)
        {
            const uint32_t i = leaf_off[j];
            Dec d = dec[i];
            d.kind = d.fb_kind; d.pre_spatial = 1;
            d.axis = d.oaxis; d.bin = d.obin; d.cmin = d.ocmin; d.scale = d.oscale;
            dec[i] = d;
            refused++;
        }
        refused = block_sum<1024>(refused, sh);
        if (tid == 0) { io[2] += refused; }
    }
    __syncthreads();
    for (uint32_t k = tid; k < n_scenes; k += 1024) { need[k] = 0ull; }
    for (uint32_t k = tid; k <= 3 * n_tiles; k += 1024) { desc[k] = 0ull; }
    if (tid == 0) { io[10] = 0u; io[11] = 0u; io[13] = 0u; io[14] = 0u; io[15] = 0xffffffffu; }
}

// Child slots, reference offsets and leaf offsets of a level: three exclusive scans in one pass
// with decoupled look-back (the scheme of the bake's slot scan: blocks take tiles in the order
// they start, warp a publishes array a's tile sum and walks its predecessors 32 at a time).
// Descriptor: flag in bits 62-63 (1 sum, 2 inclusive prefix), value in the low 32 bits;
// desc[3 * tile + a], the ticket in the word after the last tile's. Waits are bounded (io[12]).
constexpr unsigned long long SO_AGG = 1ull << 62, SO_PRE = 2ull << 62, SO_FLAGS = 3ull << 62;
constexpr uint32_t SO_SPIN_LIMIT = 1u << 22;
constexpr int SO_THREADS = 512, SO_ITEMS = 8, SO_TILE = SO_THREADS * SO_ITEMS;

__global__ void __launch_bounds__(SO_THREADS)
k_sah_offsets(Dec* __restrict__ dec, uint32_t n_lvl, unsigned long long* __restrict__ desc,
              uint32_t* __restrict__ ticket, uint32_t* __restrict__ io, uint32_t* __restrict__ child_slot,
              uint32_t* __restrict__ ref_off, uint32_t* __restrict__ leaf_off)
{
    __shared__ uint32_t sh[SO_THREADS / 32 + 1];
    __shared__ uint32_t s_tile, s_prev[3];
    if (threadIdx.x == 0) { s_tile = atomicAdd(ticket, 1u); }
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t i0 = tile * SO_TILE + threadIdx.x * SO_ITEMS;
    const bool refuse_all = io[7] != 0u;
    uint32_t v[3][SO_ITEMS], sum[3] = { 0, 0, 0 }, nleaf = 0, bmax = 0, refused = 0;
#pragma unroll
    for (int r = 0; r < SO_ITEMS; r++)
    {
        v[0][r] = v[1][r] = v[2][r] = 0;
        const uint32_t i = i0 + r;
        if (i < n_lvl)
        {
            int kind = dec[i].kind;
            if (refuse_all && kind == K_SPATIAL)
            {
                // the saved object split (or a leaf) in place of the refused spatial split
                Dec& d = dec[i];
                kind = d.fb_kind;
                d.kind = kind; d.pre_spatial = 1;
                d.axis = d.oaxis; d.bin = d.obin; d.cmin = d.ocmin; d.scale = d.oscale;
                refused++;
            }
            const uint32_t n = dec[i].n;
            if (kind == K_LEAF) { v[2][r] = n; nleaf++; }
            else if (kind == K_OBJECT)
            {
                const uint32_t l = dec[i].oleft;
                v[0][r] = 2;
                v[1][r] = n;
                bmax = max(bmax, max(l, n - l));
            }
            else
            {
                const uint32_t st = dec[i].straddle, ri = dec[i].right;
                v[0][r] = 2;
                v[1][r] = n + st;
                bmax = max(bmax, max(n - ri, ri + st));
            }
        }
        sum[0] += v[0][r]; sum[1] += v[1][r]; sum[2] += v[2][r];
    }
    uint32_t excl[3], tot[3];
#pragma unroll
    for (int a = 0; a < 3; a++) { excl[a] = block_excl_scan<SO_THREADS>(sum[a], sh, &tot[a]); }
    nleaf = block_sum<SO_THREADS>(nleaf, sh);
    if (refuse_all)
    {
        refused = block_sum<SO_THREADS>(refused, sh);
        if (threadIdx.x == 0 && refused) { atomicAdd(&io[2], refused); }
    }
    // the largest next-level node
    for (int o = 16; o > 0; o >>= 1) { bmax = max(bmax, __shfl_xor_sync(0xffffffffu, bmax, o)); }
    if ((threadIdx.x & 31) == 0 && bmax) { atomicMax(&io[10], bmax); }
    if (threadIdx.x == 0 && nleaf) { atomicAdd(&io[6], nleaf); }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < 3)
    {
        const int a = warp;
        if (lane == 0)
        {
            cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> mine(desc[3 * (size_t)tile + a]);
            mine.store((tile == 0 ? SO_PRE : SO_AGG) | tot[a], cuda::memory_order_relaxed);
        }
        uint32_t prev = 0;
        int64_t top = (int64_t)tile - 1;  // the window is tiles top - 31 .. top
        while (top >= 0)
        {
            const int64_t p = top - lane;
            unsigned long long w = SO_PRE;  // below tile 0: nothing to add
            if (p >= 0)
            {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> d(desc[3 * (size_t)p + a]);
                w = d.load(cuda::memory_order_relaxed);
                for (uint32_t spin = 0; (w & SO_FLAGS) == 0; spin++)
                {
                    if (spin > SO_SPIN_LIMIT) { atomicOr(&io[12], 1u); w = SO_PRE; break; }
                    w = d.load(cuda::memory_order_relaxed);
                }
            }
            const unsigned pre = __ballot_sync(0xffffffffu, (w & SO_FLAGS) == SO_PRE);
            const int stop = pre ? __ffs(pre) - 1 : 31;
            uint32_t add = (lane <= stop && p >= 0) ? (uint32_t)w : 0u;
            add = warp_sum(add);
            prev += add;
            if (pre) { break; }
            top -= 32;
        }
        if (lane == 0)
        {
            if (tile > 0)
            {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> mine(desc[3 * (size_t)tile + a]);
                mine.store(SO_PRE | (uint32_t)(prev + tot[a]), cuda::memory_order_relaxed);
            }
            s_prev[a] = prev;
            if (tile == gridDim.x - 1) { io[3 + a] = prev + tot[a]; }
        }
    }
    __syncthreads();
    uint32_t run[3] = { s_prev[0] + excl[0], s_prev[1] + excl[1], s_prev[2] + excl[2] };
#pragma unroll
    for (int r = 0; r < SO_ITEMS; r++)
    {
        const uint32_t i = i0 + r;
        if (i < n_lvl) { child_slot[i] = run[0]; ref_off[i] = run[1]; leaf_off[i] = run[2]; }
        run[0] += v[0][r]; run[1] += v[1][r]; run[2] += v[2][r];
    }
}

__device__ __forceinline__ void set_node(LvlNode& L, uint32_t off, uint32_t cnt, uint32_t out, uint32_t root,
                                         uint32_t root_first, const box3& b)
{
    L.ref_off = off; L.count = cnt; L.out = out; L.root = root; L.root_first = root_first; L.pad = 0;
    for (int k = 0; k < 3; k++) { L.box[k] = b.mn[k]; L.box[3 + k] = b.mx[k]; }
}

__device__ __forceinline__ void set_out_child(OutNode& o, const box3& b, uint32_t root)
{
    for (int k = 0; k < 3; k++) { o.box[k] = b.mn[k]; o.box[3 + k] = b.mx[k]; }
    o.root = root;
    o.is_leaf = 0; o.a = 0; o.b = 0; o.size = 0; o.refs = 0; o.pre = 0; o.toff = 0;
}

// One block per node: applies the decision -- the reference's partitions in its order, the
// children's reference lists and boxes (computeRangeAABB for object splits, the union of
// the triangles clipped to each side for spatial splits, bvh_sah.cpp:426-444).
// node_list: the level nodes this launch covers (the wide nodes, with BS = 1024), or nullptr
// for one block per level node, which then leaves out the wide nodes and those of fewer than
// min_refs references.
template <int BS>
__global__ void __launch_bounds__(BS)
k_sah_split(const LvlNode* __restrict__ lv, const uint32_t* __restrict__ refs, const Dec* __restrict__ dec,
            const uint32_t* __restrict__ child_slot, const uint32_t* __restrict__ ref_off,
            const uint32_t* __restrict__ leaf_off, Ctx C, uint32_t* __restrict__ tmp, uint32_t* __restrict__ pos,
            uint8_t* __restrict__ flags, LvlNode* __restrict__ lv_next, uint32_t* __restrict__ refs_next,
            OutNode* __restrict__ out, uint32_t out_base, uint32_t leaf_base, uint32_t* __restrict__ leaf_refs,
            const uint32_t* __restrict__ node_list, uint32_t min_refs)
{
    __shared__ uint32_t sh[BS / 32 + 1];
    __shared__ SBox sb[2];
    const uint32_t ni = node_list ? node_list[blockIdx.x] : blockIdx.x;
    const LvlNode nd = lv[ni];
    if (!node_list && (nd.count > WIDE_MIN || nd.count < min_refs)) { return; }
    const Dec d = dec[ni];
    const uint32_t n = nd.count;
    const uint32_t* R = refs + nd.ref_off;
    uint32_t* T = tmp + nd.ref_off;
    uint32_t* P = pos + nd.ref_off;
    uint8_t* F = flags + nd.ref_off;
    const int tid = threadIdx.x;
    const uint32_t* W = R;
    uint32_t left_end = 0, straddle_end = 0;
    if (d.pre_spatial || d.kind == K_SPATIAL)
    {
        const int ax = d.sp_axis;
        const float plane = d.plane;
        left_end = cta_partition<BS>(R, T, n, [&](uint32_t t) { return tri_hi(C, t, ax) <= plane; }, F, P, sh);
        straddle_end = left_end + cta_partition<BS>(T + left_end, T + left_end, n - left_end,
                                                [&](uint32_t t) { return tri_lo(C, t, ax) < plane; }, F + left_end,
                                                P + left_end, sh);
        W = T;
    }
    OutNode* o = &out[nd.out];
    if (d.kind == K_LEAF)
    {
        const uint32_t lo = leaf_base + leaf_off[ni];
        for (uint32_t i = tid; i < n; i += BS) { leaf_refs[lo + i] = W[i]; }
        if (tid == 0) { o->is_leaf = 1; o->a = lo; o->b = n; }
        return;
    }
    const uint32_t slot = child_slot[ni];
    const uint32_t roff = ref_off[ni];
    const uint32_t lid = out_base + slot, rid = lid + 1;
    uint32_t* Q = refs_next + roff;
    if (tid < 2) { sbox_clear(sb[tid]); }
    __syncthreads();
    uint32_t lsz, rsz;
    if (d.kind == K_OBJECT)
    {
        const int ax = d.axis, bin = d.bin, nb = d.nb;
        const float cmin = d.cmin, scale = d.scale;
        const uint32_t m = cta_partition<BS>(W, Q, n, [&](uint32_t t) { return obj_bin(centroid(C, t, ax), cmin, scale, nb) < bin; },
                                         F, P, sh);
        lsz = m; rsz = n - m;
        OBox ob[2];
        obox_clear(ob[0]); obox_clear(ob[1]);
        for (uint32_t i = tid; i < n; i += BS) { obox_add(ob[i < m ? 0 : 1], tri_box(C, Q[i])); }
        obox_flush_warp(ob[0], sb[0]);
        obox_flush_warp(ob[1], sb[1]);
    }
    else
    {
        const uint32_t st = straddle_end - left_end, rc = n - straddle_end;
        lsz = left_end + st;
        rsz = rc + st;
        for (uint32_t i = tid; i < lsz; i += BS) { Q[i] = W[i]; }
        for (uint32_t i = tid; i < rc; i += BS) { Q[lsz + i] = W[straddle_end + i]; }
        for (uint32_t i = tid; i < st; i += BS) { Q[lsz + rc + i] = W[left_end + i]; }
        const int ax = d.axis;
        box3 nbox;
        for (int k = 0; k < 3; k++) { nbox.mn[k] = nd.box[k]; nbox.mx[k] = nd.box[3 + k]; }
        box3 lclip = nbox, rclip = nbox;
        lclip.mx[ax] = d.plane;
        rclip.mn[ax] = d.plane;
        __syncthreads();
        OBox ob[2];
        obox_clear(ob[0]); obox_clear(ob[1]);
        for (uint32_t i = tid; i < lsz + rsz; i += BS)
        {
            f3 v0, v1, v2;
            tri_verts(C, Q[i], v0, v1, v2);
            const box3 cl = clip_triangle(v0, v1, v2, i < lsz ? lclip : rclip);
            if (box_valid(cl)) { obox_add(ob[i < lsz ? 0 : 1], cl); }
        }
        obox_flush_warp(ob[0], sb[0]);
        obox_flush_warp(ob[1], sb[1]);
    }
    __syncthreads();
    if (tid == 0)
    {
        const box3 lb = sbox_result(sb[0]), rb = sbox_result(sb[1]);
        LvlNode L, Rn;
        set_node(L, roff, lsz, lid, nd.root, nd.root_first, lb);
        set_node(Rn, roff + lsz, rsz, rid, nd.root, nd.root_first, rb);
        lv_next[slot] = L;
        lv_next[slot + 1] = Rn;
        set_out_child(out[lid], lb, nd.root);
        set_out_child(out[rid], rb, nd.root);
        o->is_leaf = 0; o->a = lid; o->b = rid;
    }
}

// ---- small nodes: one warp each, the references in registers ----
// Position p of a node's (at most 64) references lives in lane p & 31 of w[p >> 5].
__device__ __forceinline__ uint64_t low_bits(uint32_t k) { return k >= 64 ? ~0ull : (1ull << k) - 1ull; }

// Position of the k-th (from 0) set bit of m (which has more than k).
__device__ __forceinline__ uint32_t select_bit(uint64_t m, uint32_t k)
{
    uint32_t p = 0;
#pragma unroll
    for (int s = 32; s > 0; s >>= 1)
    {
        const uint32_t c = __popcll(m & low_bits((uint32_t)s));
        if (k >= c) { k -= c; m >>= s; p += (uint32_t)s; }
    }
    return p;
}

// cta_partition's Hoare scheme over positions [lo, hi) by the flags f (per position, false
// outside the range): the k-th failing element left of the split point trades places with the
// k-th satisfying one from the right end. Returns the number satisfying.
__device__ __forceinline__ uint32_t warp_partition64(uint32_t (&w)[2], const bool (&f)[2], uint32_t lo, uint32_t hi)
{
    const int lane = threadIdx.x & 31;
    const uint64_t range = low_bits(hi) & ~low_bits(lo);
    const uint64_t F = (((uint64_t)__ballot_sync(0xffffffffu, f[1]) << 32) | __ballot_sync(0xffffffffu, f[0])) & range;
    const uint32_t m = __popcll(F);
    const uint64_t below = low_bits(lo + m);
    const uint64_t fail_l = ~F & range & below, sat_r = F & ~below;
    const uint32_t tr = __popcll(sat_r);
    uint32_t nw[2];
#pragma unroll
    for (int h = 0; h < 2; h++)
    {
        const uint32_t p = (uint32_t)lane + 32u * h;
        const uint64_t bit = 1ull << p;
        uint32_t q = p;
        if (fail_l & bit) { q = select_bit(sat_r, tr - 1u - __popcll(fail_l & (bit - 1ull))); }
        else if (sat_r & bit) { q = select_bit(fail_l, tr - 1u - __popcll(sat_r & (bit - 1ull))); }
        const uint32_t a = __shfl_sync(0xffffffffu, w[0], q & 31), b = __shfl_sync(0xffffffffu, w[1], q & 31);
        nw[h] = q < 32 ? a : b;
    }
    w[0] = nw[0];
    w[1] = nw[1];
    return m;
}

// The union of the lanes' boxes; the empty box when none.
__device__ __forceinline__ box3 obox_warp_union(OBox o)
{
    for (int k = 0; k < 3; k++)
    {
        o.m[k] = __reduce_min_sync(0xffffffffu, o.m[k]);
        o.M[k] = __reduce_max_sync(0xffffffffu, o.M[k]);
    }
    box3 b = box_empty();
    if (o.m[0] != 0xffffffffu) { for (int k = 0; k < 3; k++) { b.mn[k] = ord2f(o.m[k]); b.mx[k] = ord2f(o.M[k]); } }
    return b;
}

// k_sah_split for the nodes of at most EVAL_STAGE references, one warp each: the same
// partitions, children and boxes.
constexpr int SPLIT_WPB = 8;
static_assert(EVAL_STAGE <= 64, "two register positions per lane");

__global__ void __launch_bounds__(SPLIT_WPB * 32)
k_sah_split_warp(const LvlNode* __restrict__ lv, const uint32_t* __restrict__ refs, const Dec* __restrict__ dec,
                 const uint32_t* __restrict__ child_slot, const uint32_t* __restrict__ ref_off,
                 const uint32_t* __restrict__ leaf_off, Ctx C, LvlNode* __restrict__ lv_next,
                 uint32_t* __restrict__ refs_next, OutNode* __restrict__ out, uint32_t out_base, uint32_t leaf_base,
                 uint32_t* __restrict__ leaf_refs, uint32_t n_lvl)
{
    const int lane = threadIdx.x & 31;
    const uint32_t ni = blockIdx.x * SPLIT_WPB + (threadIdx.x >> 5);
    if (ni >= n_lvl) { return; }
    const LvlNode nd = lv[ni];
    const uint32_t n = nd.count;
    if (n > EVAL_STAGE) { return; }  // k_sah_split applies this one
    const Dec d = dec[ni];
    const uint32_t* R = refs + nd.ref_off;
    uint32_t w[2];
    bool f[2];
#pragma unroll
    for (int h = 0; h < 2; h++)
    {
        const uint32_t p = (uint32_t)lane + 32u * h;
        w[h] = p < n ? R[p] : 0u;
    }
    uint32_t left_end = 0, straddle_end = 0;
    if (d.pre_spatial || d.kind == K_SPATIAL)
    {
        const int ax = d.sp_axis;
        const float plane = d.plane;
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const uint32_t p = (uint32_t)lane + 32u * h;
            f[h] = p < n && tri_hi(C, w[h], ax) <= plane;
        }
        left_end = warp_partition64(w, f, 0, n);
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const uint32_t p = (uint32_t)lane + 32u * h;
            f[h] = p >= left_end && p < n && tri_lo(C, w[h], ax) < plane;
        }
        straddle_end = left_end + warp_partition64(w, f, left_end, n);
    }
    OutNode* o = &out[nd.out];
    if (d.kind == K_LEAF)
    {
        const uint32_t lo = leaf_base + leaf_off[ni];
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const uint32_t p = (uint32_t)lane + 32u * h;
            if (p < n) { leaf_refs[lo + p] = w[h]; }
        }
        if (lane == 0) { o->is_leaf = 1; o->a = lo; o->b = n; }
        return;
    }
    const uint32_t slot = child_slot[ni];
    const uint32_t roff = ref_off[ni];
    const uint32_t lid = out_base + slot, rid = lid + 1;
    uint32_t* Q = refs_next + roff;
    uint32_t lsz, rsz;
    OBox ob[2];
    obox_clear(ob[0]);
    obox_clear(ob[1]);
    if (d.kind == K_OBJECT)
    {
        const int ax = d.axis, bin = d.bin, nb = d.nb;
        const float cmin = d.cmin, scale = d.scale;
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const uint32_t p = (uint32_t)lane + 32u * h;
            f[h] = p < n && obj_bin(centroid(C, w[h], ax), cmin, scale, nb) < bin;
        }
        const uint32_t m = warp_partition64(w, f, 0, n);
        lsz = m;
        rsz = n - m;
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const uint32_t p = (uint32_t)lane + 32u * h;
            if (p < n)
            {
                Q[p] = w[h];
                obox_add(ob[p < m ? 0 : 1], tri_box(C, w[h]));
            }
        }
    }
    else
    {
        // left child: positions [0, straddle_end); right child: [straddle_end, n), then the
        // straddling [left_end, straddle_end) again -- position p keeps index p of the list
        // and a straddling one is repeated at n + p - left_end
        const uint32_t st = straddle_end - left_end, rc = n - straddle_end;
        lsz = left_end + st;
        rsz = rc + st;
        const int ax = d.axis;
        box3 lclip, rclip;
        for (int k = 0; k < 3; k++) { lclip.mn[k] = rclip.mn[k] = nd.box[k]; lclip.mx[k] = rclip.mx[k] = nd.box[3 + k]; }
        lclip.mx[ax] = d.plane;
        rclip.mn[ax] = d.plane;
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const uint32_t p = (uint32_t)lane + 32u * h;
            if (p < n)
            {
                Q[p] = w[h];
                const bool straddles = p >= left_end && p < straddle_end;
                if (straddles) { Q[n + p - left_end] = w[h]; }
                f3 v0, v1, v2;
                tri_verts(C, w[h], v0, v1, v2);
                if (p < straddle_end)
                {
                    const box3 cl = clip_triangle(v0, v1, v2, lclip);
                    if (box_valid(cl)) { obox_add(ob[0], cl); }
                }
                if (p >= straddle_end || straddles)
                {
                    const box3 cl = clip_triangle(v0, v1, v2, rclip);
                    if (box_valid(cl)) { obox_add(ob[1], cl); }
                }
            }
        }
    }
    const box3 lb = obox_warp_union(ob[0]), rb = obox_warp_union(ob[1]);
    if (lane == 0)
    {
        LvlNode L, Rn;
        set_node(L, roff, lsz, lid, nd.root, nd.root_first, lb);
        set_node(Rn, roff + lsz, rsz, rid, nd.root, nd.root_first, rb);
        lv_next[slot] = L;
        lv_next[slot + 1] = Rn;
        set_out_child(out[lid], lb, nd.root);
        set_out_child(out[rid], rb, nd.root);
        o->is_leaf = 0; o->a = lid; o->b = rid;
    }
}

// ---- the wide path's partitions: the reference's std::partition (Hoare's scheme, see
// cta_partition) over many blocks. Pass 0 splits a spatial node's references by "box max <=
// plane" (R -> T), pass 1 the rest by "box min < plane" (T -> T2, the left part copied), pass 2
// an object split by "centroid bin < split bin" (R or T2 -> the next level's list). Per pass:
// flags and satisfied counts; per chunk the failing elements left of the split point and the
// satisfying ones right of it; their ranks from the chunk prefixes; the scatter, where the
// k-th failing element from the left and the k-th satisfying one from the right trade places.
// Each block owns WIDE_CH consecutive references, 16 per thread.
struct WideSplit
{
    const LvlNode*  lv;
    const Dec*      dec;
    const uint32_t* wl;
    const uint32_t* wco;
    uint32_t        nw;
    WideAcc*        acc;
    const uint32_t* refs;       // this level's references
    uint32_t*       tmp;        // T
    uint32_t*       tmp2;       // T2
    uint32_t*       posf;       // failing-left positions, ascending
    uint32_t*       poss;       // satisfying-right positions, ascending
    uint8_t*        flags;
    uint32_t*       chunk;      // per block: failing-left, satisfying-right counts
    uint32_t*       refs_next;  // next level's references
    const uint32_t* ref_off;    // next-level offset per level node
    const uint32_t* child_slot;
    const uint32_t* leaf_off;
    uint32_t*       leaf_refs;
    LvlNode*        lv_next;
    OutNode*        out;
    uint32_t        out_base, leaf_base;
};

__device__ __forceinline__ bool wp_applies(int pass, const Dec& d)
{
    return pass < 2 ? (d.pre_spatial || d.kind == K_SPATIAL) : d.kind == K_OBJECT;
}
__device__ __forceinline__ bool wp_pred(int pass, const Dec& d, const Ctx& C, uint32_t t)
{
    if (pass == 0) { return tri_hi(C, t, d.sp_axis) <= d.plane; }
    if (pass == 1) { return tri_lo(C, t, d.sp_axis) < d.plane; }
    return obj_bin(centroid(C, t, d.axis), d.cmin, d.scale, d.nb) < d.bin;
}
__device__ __forceinline__ const uint32_t* wp_in(int pass, const WideSplit& W, const LvlNode& nd, const Dec& d)
{
    if (pass == 0) { return W.refs + nd.ref_off; }
    if (pass == 1) { return W.tmp + nd.ref_off; }
    return (d.pre_spatial ? W.tmp2 : W.refs) + nd.ref_off;
}

// block and thread ranges of chunk c: the block's [c0, c1), this thread's [t0, t1)
struct WpItem
{
    uint32_t k, g, node, c0, c1, t0, t1, n;
};
__device__ __forceinline__ WpItem wp_item(const WideSplit& W)
{
    WpItem it;
    uint32_t c;
    it.k = wide_item(W.wco, W.nw, blockIdx.x, c);
    it.g = blockIdx.x;
    it.node = W.wl[it.k];
    it.n = W.lv[it.node].count;
    it.c0 = c * WIDE_CH;
    it.c1 = min(it.n, it.c0 + WIDE_CH);
    it.t0 = min(it.c1, it.c0 + threadIdx.x * 16u);
    it.t1 = min(it.c1, it.t0 + 16u);
    return it;
}

template <int PASS>
__global__ void __launch_bounds__(SBLK) k_wp_flags(WideSplit W, Ctx C)
{
    __shared__ uint32_t sh[SBLK / 32 + 1];
    const WpItem it = wp_item(W);
    const Dec d = W.dec[it.node];
    if (!wp_applies(PASS, d)) { return; }
    const LvlNode nd = W.lv[it.node];
    WideAcc& A = W.acc[it.k];
    const uint32_t b0 = PASS == 1 ? A.pm[0] : 0u;
    const uint32_t* in = wp_in(PASS, W, nd, d);
    uint8_t* F = W.flags + nd.ref_off;
    uint32_t cnt = 0;
    for (uint32_t i = max(it.t0, b0); i < it.t1; i++)
    {
        const uint8_t f = wp_pred(PASS, d, C, in[i]) ? 1 : 0;
        F[i] = f;
        cnt += f;
    }
    cnt = block_sum<SBLK>(cnt, sh);
    if (threadIdx.x == 0 && cnt) { atomicAdd(&A.pm[PASS], cnt); }
}

template <int PASS>
__global__ void __launch_bounds__(SBLK) k_wp_sides(WideSplit W)
{
    __shared__ uint32_t sh[SBLK / 32 + 1];
    const WpItem it = wp_item(W);
    const Dec d = W.dec[it.node];
    if (!wp_applies(PASS, d)) { return; }
    const LvlNode nd = W.lv[it.node];
    WideAcc& A = W.acc[it.k];
    const uint32_t b0 = PASS == 1 ? A.pm[0] : 0u;
    const uint32_t m = b0 + A.pm[PASS];  // the split point
    const uint8_t* F = W.flags + nd.ref_off;
    uint32_t fl = 0, sr = 0;
    for (uint32_t i = max(it.t0, b0); i < it.t1; i++)
    {
        if (i < m) { fl += F[i] ? 0u : 1u; } else { sr += F[i]; }
    }
    fl = block_sum<SBLK>(fl, sh);
    sr = block_sum<SBLK>(sr, sh);
    if (threadIdx.x == 0)
    {
        W.chunk[2 * it.g] = fl;
        W.chunk[2 * it.g + 1] = sr;
        if (fl) { atomicAdd(&A.ftot[PASS], fl); }
    }
}

// Ranks of this thread's failing-left / satisfying-right elements: the counts of the node's
// earlier chunks plus the block's exclusive scan.
template <int PASS>
__device__ __forceinline__ void wp_ranks(const WideSplit& W, const WpItem& it, const uint8_t* F, uint32_t b0, uint32_t m,
                                         uint32_t* sh, uint32_t& rf, uint32_t& rs)
{
    const uint32_t g0 = W.wco[it.k];
    uint32_t pf = 0, ps = 0;
    for (uint32_t g = g0 + threadIdx.x; g < it.g; g += SBLK) { pf += W.chunk[2 * g]; ps += W.chunk[2 * g + 1]; }
    pf = block_sum<SBLK>(pf, sh);
    ps = block_sum<SBLK>(ps, sh);
    uint32_t fl = 0, sr = 0;
    for (uint32_t i = max(it.t0, b0); i < it.t1; i++)
    {
        if (i < m) { fl += F[i] ? 0u : 1u; } else { sr += F[i]; }
    }
    rf = pf + block_excl_scan<SBLK>(fl, sh, nullptr);
    rs = ps + block_excl_scan<SBLK>(sr, sh, nullptr);
}

template <int PASS>
__global__ void __launch_bounds__(SBLK) k_wp_pos(WideSplit W)
{
    __shared__ uint32_t sh[SBLK / 32 + 1];
    const WpItem it = wp_item(W);
    const Dec d = W.dec[it.node];
    if (!wp_applies(PASS, d)) { return; }
    const LvlNode nd = W.lv[it.node];
    const WideAcc& A = W.acc[it.k];
    const uint32_t b0 = PASS == 1 ? A.pm[0] : 0u;
    const uint32_t m = b0 + A.pm[PASS];
    const uint8_t* F = W.flags + nd.ref_off;
    uint32_t rf, rs;
    wp_ranks<PASS>(W, it, F, b0, m, sh, rf, rs);
    uint32_t* PF = W.posf + nd.ref_off;
    uint32_t* PS = W.poss + nd.ref_off;
    for (uint32_t i = max(it.t0, b0); i < it.t1; i++)
    {
        if (i < m) { if (!F[i]) { PF[rf++] = i; } }
        else if (F[i]) { PS[rs++] = i; }
    }
}

template <int PASS>
__global__ void __launch_bounds__(SBLK) k_wp_scatter(WideSplit W)
{
    __shared__ uint32_t sh[SBLK / 32 + 1];
    const WpItem it = wp_item(W);
    const Dec d = W.dec[it.node];
    if (!wp_applies(PASS, d)) { return; }
    const LvlNode nd = W.lv[it.node];
    const WideAcc& A = W.acc[it.k];
    const uint32_t b0 = PASS == 1 ? A.pm[0] : 0u;
    const uint32_t m = b0 + A.pm[PASS];
    const uint32_t tot = A.ftot[PASS];
    const uint8_t* F = W.flags + nd.ref_off;
    uint32_t rf, rs;
    wp_ranks<PASS>(W, it, F, b0, m, sh, rf, rs);
    const uint32_t* in = wp_in(PASS, W, nd, d);
    uint32_t* out = PASS == 0 ? W.tmp + nd.ref_off : (PASS == 1 ? W.tmp2 + nd.ref_off : W.refs_next + W.ref_off[it.node]);
    const uint32_t* PF = W.posf + nd.ref_off;
    const uint32_t* PS = W.poss + nd.ref_off;
    if (PASS == 1)
    {
        for (uint32_t i = it.t0; i < min(it.t1, b0); i++) { out[i] = in[i]; }  // the left part, unchanged
    }
    for (uint32_t i = max(it.t0, b0); i < it.t1; i++)
    {
        uint32_t src = i;
        if (i < m) { if (!F[i]) { src = PS[tot - 1u - rf]; rf++; } }
        else if (F[i]) { src = PF[tot - 1u - rs]; rs++; }
        out[i] = in[src];
    }
}

// the node's references in their final places (leaf store, or the children's lists) and the
// children's boxes (computeRangeAABB for object splits, clipped triangles for spatial ones)
__global__ void __launch_bounds__(SBLK) k_wp_place(WideSplit W, Ctx C)
{
    const WpItem it = wp_item(W);
    const Dec d = W.dec[it.node];
    const LvlNode nd = W.lv[it.node];
    WideAcc& A = W.acc[it.k];
    const uint32_t n = it.n;
    const uint32_t* Wr = (d.pre_spatial || d.kind == K_SPATIAL ? W.tmp2 : W.refs) + nd.ref_off;
    if (d.kind == K_LEAF)
    {
        const uint32_t lo = W.leaf_base + W.leaf_off[it.node];
        for (uint32_t i = it.t0; i < it.t1; i++) { W.leaf_refs[lo + i] = Wr[i]; }
        return;
    }
    uint32_t* Q = W.refs_next + W.ref_off[it.node];
    OBox ob[2];
    obox_clear(ob[0]); obox_clear(ob[1]);
    if (d.kind == K_OBJECT)
    {
        const uint32_t m = A.pm[2];
        for (uint32_t i = it.t0; i < it.t1; i++) { obox_add(ob[i < m ? 0 : 1], tri_box(C, Q[i])); }
    }
    else
    {
        const uint32_t le = A.pm[0], se = le + A.pm[1];
        const uint32_t st = se - le, rc = n - se, lsz = le + st, tot = n + st;
        box3 nbox;
        for (int k = 0; k < 3; k++) { nbox.mn[k] = nd.box[k]; nbox.mx[k] = nd.box[3 + k]; }
        box3 lclip = nbox, rclip = nbox;
        lclip.mx[d.axis] = d.plane;
        rclip.mn[d.axis] = d.plane;
        // this block's destination slots: [c0, c1) and the duplicates' [n + c0, n + c1)
        for (int part = 0; part < 2; part++)
        {
            const uint32_t j0 = part ? n + it.t0 : it.t0, j1 = part ? min(n + it.t1, tot) : it.t1;
            for (uint32_t j = j0; j < j1; j++)
            {
                const uint32_t src = j < lsz ? j : (j < lsz + rc ? se + (j - lsz) : le + (j - lsz - rc));
                const uint32_t t = Wr[src];
                Q[j] = t;
                f3 v0, v1, v2;
                tri_verts(C, t, v0, v1, v2);
                const box3 cl = clip_triangle(v0, v1, v2, j < lsz ? lclip : rclip);
                if (box_valid(cl)) { obox_add(ob[j < lsz ? 0 : 1], cl); }
            }
        }
    }
    obox_flush_warp(ob[0], A.cb[0]);
    obox_flush_warp(ob[1], A.cb[1]);
}

// the children's records (the tail of k_sah_split), one thread per wide node
__global__ void k_wp_final(WideSplit W)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= W.nw) { return; }
    const uint32_t ni = W.wl[k];
    const LvlNode nd = W.lv[ni];
    const Dec d = W.dec[ni];
    const WideAcc& A = W.acc[k];
    const uint32_t n = nd.count;
    OutNode* o = &W.out[nd.out];
    if (d.kind == K_LEAF)
    {
        o->is_leaf = 1; o->a = W.leaf_base + W.leaf_off[ni]; o->b = n;
        return;
    }
    uint32_t lsz, rsz;
    if (d.kind == K_OBJECT) { lsz = A.pm[2]; rsz = n - lsz; }
    else
    {
        const uint32_t st = A.pm[1], rc = n - A.pm[0] - A.pm[1];
        lsz = A.pm[0] + st;
        rsz = rc + st;
    }
    const uint32_t slot = W.child_slot[ni];
    const uint32_t roff = W.ref_off[ni];
    const uint32_t lid = W.out_base + slot, rid = lid + 1;
    const box3 lb = sbox_result(A.cb[0]), rb = sbox_result(A.cb[1]);
    LvlNode L, Rn;
    set_node(L, roff, lsz, lid, nd.root, nd.root_first, lb);
    set_node(Rn, roff + lsz, rsz, rid, nd.root, nd.root_first, rb);
    W.lv_next[slot] = L;
    W.lv_next[slot + 1] = Rn;
    set_out_child(W.out[lid], lb, nd.root);
    set_out_child(W.out[rid], rb, nd.root);
    o->is_leaf = 0; o->a = lid; o->b = rid;
}

// ---- the subtree roots in the reference's queue order: by depth, then key position ----
// Key of root i: depth << fb | first (first < 2^fb, depth < 256), and the counts of every 8-bit
// digit of the sort's passes (hist, zeroed). grp[512] = the largest root, grp[513] = the
// deepest root (both zeroed).
constexpr uint32_t ROOT_MAX_DEPTH = 255;
constexpr int      ROOT_HIST_PASSES = 8;

__global__ void __launch_bounds__(SBLK)
k_root_keys(const SahRoot* __restrict__ roots, uint32_t nr, int fb, int passes, uint64_t* __restrict__ keys,
            uint32_t* __restrict__ hist, uint32_t* __restrict__ grp)
{
    __shared__ uint32_t sh[ROOT_HIST_PASSES][256];
    for (int k = threadIdx.x; k < ROOT_HIST_PASSES * 256; k += SBLK) { (&sh[0][0])[k] = 0u; }
    __syncthreads();
    const uint32_t i = blockIdx.x * SBLK + threadIdx.x;
    uint32_t cnt = 0, dep = 0;
    if (i < nr)
    {
        const SahRoot r = roots[i];
        cnt = r.count;
        dep = r.depth;
        const uint64_t key = ((uint64_t)min(dep, ROOT_MAX_DEPTH) << fb) | r.first;
        keys[i] = key;
        for (int p = 0; p < passes; p++) { atomicAdd(&sh[p][(key >> (8 * p)) & 255u], 1u); }
    }
    cnt = __reduce_max_sync(0xffffffffu, cnt);
    dep = __reduce_max_sync(0xffffffffu, dep);
    if ((threadIdx.x & 31) == 0)
    {
        atomicMax(&grp[512], cnt);
        atomicMax(&grp[513], dep);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < passes * 256; k += SBLK)
    {
        const uint32_t c = (&sh[0][0])[k];
        if (c) { atomicAdd(&hist[k], c); }
    }
}

// sorted[j] = roots[order[j]] (order: nullptr for the identity), and its triangle count.
__global__ void __launch_bounds__(SBLK)
k_root_gather(const SahRoot* __restrict__ roots, const uint32_t* __restrict__ order, uint32_t nr,
              SahRoot* __restrict__ sorted, uint32_t* __restrict__ cnt)
{
    const uint32_t j = blockIdx.x * SBLK + threadIdx.x;
    if (j >= nr) { return; }
    const SahRoot r = roots[order ? order[j] : j];
    sorted[j] = r;
    cnt[j] = r.count;
}

// Where each depth's run of sorted roots starts: grp[d] = its first index, grp[256 + d] = the
// triangles of all shallower roots (pre: the exclusive scan of the counts). grp[0..255] start
// at ~0: depths without roots keep it.
__global__ void __launch_bounds__(SBLK)
k_root_groups(const SahRoot* __restrict__ sorted, const uint32_t* __restrict__ pre, uint32_t nr, uint32_t* __restrict__ grp)
{
    const uint32_t j = blockIdx.x * SBLK + threadIdx.x;
    if (j >= nr) { return; }
    const uint32_t d = min(sorted[j].depth, ROOT_MAX_DEPTH);
    if (j == 0 || min(sorted[j - 1].depth, ROOT_MAX_DEPTH) != d)
    {
        grp[d] = j;
        grp[256 + d] = pre[j];
    }
}

constexpr uint32_t ROOT_CHUNK = 8192;  // references per block of k_sah_root_refs

// Copies the Morton-sorted triangles of new subtree roots into the level's reference list, at
// offsets pre[b] + delta (pre: the sorted roots' exclusive count scan), which it also stores
// in new_off for k_sah_merge.
__global__ void __launch_bounds__(SBLK)
k_sah_root_refs(const SahRoot* __restrict__ roots, const uint32_t* __restrict__ pre, uint32_t delta,
                uint32_t* __restrict__ new_off, const uint32_t* __restrict__ perm, uint32_t* __restrict__ refs,
                uint32_t* __restrict__ wtri, uint8_t* __restrict__ kpos)
{
    const SahRoot r = roots[blockIdx.x];
    const uint32_t off = pre[blockIdx.x] + delta;  // (modulo 2^32: delta may be "negative")
    if (threadIdx.x == 0 && blockIdx.y == 0) { new_off[blockIdx.x] = off; }
    // blockIdx.y: this block's ROOT_CHUNK references of the root
    const uint32_t e = min(r.count, (blockIdx.y + 1) * ROOT_CHUNK);
    for (uint32_t i = blockIdx.y * ROOT_CHUNK + threadIdx.x; i < e; i += SBLK)
    {
        refs[off + i] = perm[r.first + i];
        wtri[r.first + i] = 0u;  // these keys' triangles are counted and placed by the subtree
        kpos[r.first + i] = 0u;
    }
}

// Merges new roots (sorted by key position) into the continuing nodes (sorted by their
// root's key position): the reference's queue order at this level.
__global__ void __launch_bounds__(SBLK)
k_sah_merge(const LvlNode* __restrict__ cont, uint32_t n_cont, const SahRoot* __restrict__ roots, uint32_t r0, uint32_t m,
            const uint32_t* __restrict__ new_off, uint32_t out_base, LvlNode* __restrict__ merged, OutNode* __restrict__ out,
            uint32_t* __restrict__ root_out)
{
    const uint32_t i = blockIdx.x * SBLK + threadIdx.x;
    if (i < n_cont)
    {
        const LvlNode c = cont[i];
        uint32_t lo = 0, hi = m;  // new roots with first < c.root_first
        while (lo < hi)
        {
            const uint32_t mid = (lo + hi) >> 1;
            if (roots[r0 + mid].first < c.root_first) { lo = mid + 1; } else { hi = mid; }
        }
        merged[i + lo] = c;
    }
    else if (i < n_cont + m)
    {
        const uint32_t j = i - n_cont;
        const SahRoot r = roots[r0 + j];
        uint32_t lo = 0, hi = n_cont;  // continuing nodes whose root starts before this one
        while (lo < hi)
        {
            const uint32_t mid = (lo + hi) >> 1;
            if (cont[mid].root_first < r.first) { lo = mid + 1; } else { hi = mid; }
        }
        box3 b;
        for (int k = 0; k < 3; k++) { b.mn[k] = r.box[k]; b.mx[k] = r.box[3 + k]; }
        LvlNode L;
        set_node(L, new_off[j], r.count, out_base + j, r0 + j, r.first, b);
        merged[j + lo] = L;
        set_out_child(out[out_base + j], b, r0 + j);
        root_out[r0 + j] = out_base + j;
    }
}

__global__ void __launch_bounds__(SBLK) k_sah_up(OutNode* __restrict__ out, uint32_t b, uint32_t e)
{
    const uint32_t i = b + blockIdx.x * SBLK + threadIdx.x;
    if (i >= e) { return; }
    OutNode& o = out[i];
    if (o.is_leaf) { o.size = 1; o.refs = o.b; }
    else
    {
        o.size = 1 + out[o.a].size + out[o.b].size;
        o.refs = out[o.a].refs + out[o.b].refs;
    }
}

__global__ void __launch_bounds__(SBLK) k_sah_down(OutNode* __restrict__ out, uint32_t b, uint32_t e)
{
    const uint32_t i = b + blockIdx.x * SBLK + threadIdx.x;
    if (i >= e) { return; }
    const OutNode o = out[i];
    if (o.is_leaf) { return; }
    OutNode& l = out[o.a];
    OutNode& r = out[o.b];
    l.pre = o.pre + 1;
    l.toff = o.toff;
    r.pre = o.pre + 1 + l.size;
    r.toff = o.toff + l.refs;
}

__global__ void __launch_bounds__(SBLK)
k_sah_root_weights(const SahRoot* __restrict__ roots, uint32_t n_roots, const uint32_t* __restrict__ root_out,
                   const OutNode* __restrict__ out, uint32_t* __restrict__ wnode, uint32_t* __restrict__ wtri)
{
    const uint32_t r = blockIdx.x * SBLK + threadIdx.x;
    if (r >= n_roots) { return; }
    const OutNode& o = out[root_out[r]];
    wnode[roots[r].first] = roots[r].rank + o.size;
    wtri[roots[r].first] = o.refs;
}

__global__ void __launch_bounds__(SBLK)
k_sah_emit(const OutNode* __restrict__ out, uint32_t n_out, const SahRoot* __restrict__ roots,
           const uint32_t* __restrict__ snode, const uint32_t* __restrict__ stri, const uint32_t* __restrict__ leaf_refs,
           const rt_triangle* __restrict__ tris, rt_bvh_node* __restrict__ nodes, rt_triangle* __restrict__ otris,
           uint32_t* __restrict__ prim, uint32_t max_nodes, uint32_t max_tris, uint32_t* __restrict__ status)
{
    const uint32_t i = blockIdx.x * SBLK + threadIdx.x;
    if (i >= n_out) { return; }
    const OutNode o = out[i];
    const SahRoot r = roots[o.root];
    const uint32_t base = snode[r.first] + r.rank;
    box3 b;
    for (int k = 0; k < 3; k++) { b.mn[k] = o.box[k]; b.mx[k] = o.box[3 + k]; }
    if (base + o.pre >= max_nodes) { atomicOr(status, ST_CAPACITY); return; }
    if (o.is_leaf)
    {
        const uint32_t t0 = stri[r.first] + o.toff;
        if ((uint64_t)t0 + o.b > max_tris) { atomicOr(status, ST_CAPACITY); return; }
        write_node(nodes, base + o.pre, b, 1, t0, o.b);
        for (uint32_t k = 0; k < o.b; k++)
        {
            const uint32_t t = leaf_refs[o.a + k];
            otris[t0 + k] = tris[t];
            prim[t0 + k] = t;
        }
    }
    else
    {
        write_node(nodes, base + o.pre, b, 0, base + out[o.a].pre, base + out[o.b].pre);
    }
}

inline uint32_t nblk(uint64_t n) { return (uint32_t)((n + SBLK - 1) / SBLK); }

} // namespace

int sah_build(rt_bvh* B, const rt_build_cfg& cfg, const SahInput& in, cudaStream_t st, SahResult* res)
{
    BuildScratch& S = B->s;
    const uint32_t cap = in.cap;
    const uint32_t nr = in.n_roots;

    if (S.sah_roots_lvl.ensure((size_t)nr * sizeof(SahRoot)) || S.sah_lvl_a.ensure((size_t)cap * sizeof(LvlNode)) ||
        S.sah_lvl_b.ensure((size_t)cap * sizeof(LvlNode)) || S.sah_node_ids.ensure((size_t)cap * sizeof(LvlNode)) ||
        S.sah_refs_a.ensure((size_t)cap * 4) || S.sah_refs_b.ensure((size_t)cap * 4) || S.sah_tmp.ensure((size_t)cap * 4) ||
        S.sah_pos.ensure((size_t)cap * 4) || S.sah_scan_in.ensure((size_t)cap) || S.sah_dec.ensure((size_t)cap * sizeof(Dec)) ||
        S.sah_out.ensure((size_t)2 * cap * sizeof(OutNode)) || S.sah_leaf_refs.ensure((size_t)cap * 4) ||
        S.sah_scan_out.ensure((size_t)3 * cap * 4 + (size_t)2 * nr * 4 + 64))
    {
        return RT_E_CUDA;
    }
    SahRoot* d_roots = S.sah_roots_lvl.as<SahRoot>();
    // subtree roots in the reference's queue order -- by depth, then key position -- sorted on
    // the device; the host reads back where each depth's run starts
    int fb = 1;
    while (fb < 32 && (1ull << fb) < (uint64_t)in.n) { fb++; }
    const int key_bits = fb + 8, passes = sort_passes(key_bits);
    const size_t o_vals = (size_t)nr * 8, o_cnt = o_vals + (size_t)nr * 4, o_pre = o_cnt + (size_t)nr * 4,
                 o_hist = o_pre + (size_t)nr * 4, o_grp = o_hist + (size_t)ROOT_HIST_PASSES * 256 * 4;
    if (S.sah_root_ord.ensure(o_grp + 520 * 4)) { return RT_E_CUDA; }
    uint8_t* ob = S.sah_root_ord.as<uint8_t>();
    uint64_t* rkeys = reinterpret_cast<uint64_t*>(ob);
    uint32_t* rvals = reinterpret_cast<uint32_t*>(ob + o_vals);
    uint32_t* rcnt = reinterpret_cast<uint32_t*>(ob + o_cnt);
    uint32_t* rpre = reinterpret_cast<uint32_t*>(ob + o_pre);
    uint32_t* rhist = reinterpret_cast<uint32_t*>(ob + o_hist);
    uint32_t* rgrp = reinterpret_cast<uint32_t*>(ob + o_grp);
    RT_CUDA(cudaMemsetAsync(rhist, 0, (size_t)ROOT_HIST_PASSES * 256 * 4, st));
    RT_CUDA(cudaMemsetAsync(rgrp, 0xff, 256 * 4, st));
    RT_CUDA(cudaMemsetAsync(rgrp + 256, 0, 264 * 4, st));
    const uint32_t* order = nullptr;
    if (nr > 1)
    {
        k_root_keys<<<nblk(nr), SBLK, 0, st>>>(in.roots, nr, fb, passes, rkeys, rhist, rgrp);
        count_launch();
        uint64_t* kout = nullptr;
        uint32_t* vout = nullptr;
        if (int e = radix_sort_pairs<uint64_t>(rkeys, rvals, true, nr, key_bits, rhist, nullptr, S.root_sort, in.status, st,
                                               &kout, &vout))
        {
            return e;
        }
        order = vout;
    }
    else
    {
        k_root_keys<<<1, SBLK, 0, st>>>(in.roots, nr, fb, 0, rkeys, rhist, rgrp);
        count_launch();
    }
    k_root_gather<<<nblk(nr), SBLK, 0, st>>>(in.roots, order, nr, d_roots, rcnt);
    count_launch();
    if (int e = exclusive_scan_u32(rcnt, rpre, nr, rgrp + 514, S.scan, st)) { return e; }
    k_root_groups<<<nblk(nr), SBLK, 0, st>>>(d_roots, rpre, nr, rgrp);
    count_launch();
    if (int e = check_launch("sah roots")) { return e; }
    uint32_t grp[520];
    RT_CUDA(cudaMemcpyAsync(grp, rgrp, sizeof(grp), cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    if (grp[513] > ROOT_MAX_DEPTH) { return fail(RT_E_CAPACITY, "SAH builder: subtree roots deeper than 255 levels"); }
    // runs of roots per depth: {depth, first index, triangles of the shallower roots}
    struct Run { uint32_t depth, start, pre; };
    std::vector<Run> runs;
    for (uint32_t d = 0; d <= ROOT_MAX_DEPTH; d++)
    {
        if (grp[d] != 0xffffffffu) { runs.push_back({ d, grp[d], grp[256 + d] }); }
    }
    if (runs.empty() || runs[0].start != 0) { return fail(RT_E_CAPACITY, "SAH builder: root runs out of order"); }
    const uint32_t root_total = grp[514], root_max = grp[512];
    uint32_t* child_slot = S.sah_scan_out.as<uint32_t>();
    uint32_t* ref_offs = child_slot + cap;
    uint32_t* leaf_offs = ref_offs + cap;
    uint32_t* root_out = leaf_offs + cap;
    uint32_t* new_off = root_out + nr;
    uint32_t* io = new_off + nr;
    uint32_t io_h[16] = { in.n, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0xffffffffu };
    RT_CUDA(cudaMemcpyAsync(io, io_h, 64, cudaMemcpyHostToDevice, st));
    // wide-node scratch: at most cap / WIDE_MIN nodes of a level have more than WIDE_MIN references
    const uint32_t max_wide = cap / WIDE_MIN + 2;
    const uint32_t max_chunks = cap / WIDE_CH + max_wide + 1;
    if (S.sah_wide.ensure((size_t)max_wide * sizeof(WideAcc) + (size_t)(2 * max_wide + 2) * 4 + (size_t)max_chunks * 8) ||
        S.sah_tmp2.ensure((size_t)cap * 4) || S.sah_pos2.ensure((size_t)cap * 4))
    {
        return RT_E_CUDA;
    }
    WideAcc* wacc = S.sah_wide.as<WideAcc>();
    uint32_t* wl = reinterpret_cast<uint32_t*>(wacc + max_wide);
    uint32_t* wco = wl + max_wide;
    uint32_t* wchunk = wco + max_wide + 2;
    uint32_t next_bound = 0;  // upper bound of the largest node of the coming level
    const uint32_t n_budget = (uint32_t)in.budget_used.size();
    if (n_budget == 0 || n_budget > MAX_BUDGET_SCENES || in.budget_cap.size() != n_budget)
    {
        return fail(RT_E_INVALID, "SAH builder: bad spatial-split budget");
    }
    // budget scratch: need (n_budget words of 64 bits), the offset scan's descriptors and ticket
    // (3 * max_tiles + 1), then used and cap (n_budget words of 32 bits each)
    std::vector<uint32_t> budget(in.budget_used);
    budget.insert(budget.end(), in.budget_cap.begin(), in.budget_cap.end());
    const uint32_t max_tiles = (cap + SO_TILE - 1) / SO_TILE + 1;
    const size_t n_zero64 = (size_t)n_budget + 3 * (size_t)max_tiles + 1;
    if (S.sah_budget.ensure(n_zero64 * 8 + (size_t)budget.size() * 4)) { return RT_E_CUDA; }
    unsigned long long* d_need = S.sah_budget.as<unsigned long long>();
    unsigned long long* d_desc = d_need + n_budget;
    uint32_t* d_used = reinterpret_cast<uint32_t*>(d_need + n_zero64);
    RT_CUDA(cudaMemsetAsync(d_need, 0, n_zero64 * 8, st));
    RT_CUDA(cudaMemcpyAsync(d_used, budget.data(), budget.size() * 4, cudaMemcpyHostToDevice, st));

    Ctx C;
    C.verts = in.verts; C.tris = in.tris; C.lo = in.lo; C.hi = in.hi; C.cz = in.cz;
    C.max_leaf = cfg.max_leaf; C.bins_min = cfg.bins_min; C.bins_max = cfg.bins_max;
    C.c_trav = cfg.c_trav; C.c_isect = cfg.c_isect; C.centroid_eps = cfg.centroid_eps; C.spatial_eps = cfg.spatial_eps;

    LvlNode* lv_cur = S.sah_lvl_a.as<LvlNode>();
    LvlNode* lv_next = S.sah_lvl_b.as<LvlNode>();
    LvlNode* lv_tmp = S.sah_node_ids.as<LvlNode>();
    uint32_t* refs_cur = S.sah_refs_a.as<uint32_t>();
    uint32_t* refs_next = S.sah_refs_b.as<uint32_t>();
    OutNode* out = S.sah_out.as<OutNode>();

    std::vector<std::pair<uint32_t, uint32_t>> levels;
    uint32_t out_total = 0, n_cur = 0, r_cur = 0, leaf_total = 0, ri = 0;
    size_t run = 0;
    uint32_t depth = runs[0].depth;
    for (int guard = 0; guard < 100000; guard++)
    {
        // subtree roots entering at this depth
        uint32_t m = 0, add = 0, delta = 0;
        if (run < runs.size() && runs[run].depth == depth)
        {
            const uint32_t end = run + 1 < runs.size() ? runs[run + 1].start : nr;
            const uint32_t pend = run + 1 < runs.size() ? runs[run + 1].pre : root_total;
            if (runs[run].start != ri || end < ri) { return fail(RT_E_CAPACITY, "SAH builder: root runs out of order"); }
            m = end - ri;
            add = pend - runs[run].pre;
            delta = r_cur - runs[run].pre;
            next_bound = std::max(next_bound, root_max);
            run++;
        }
        const uint32_t lvl_begin = out_total - n_cur;
        if (m > 0)
        {
            if ((uint64_t)r_cur + add > cap || (uint64_t)n_cur + m > cap || (uint64_t)out_total + m > 2ull * cap)
            {
                return fail(RT_E_CAPACITY, "SAH builder: level capacity exceeded");
            }
            const dim3 rgrid(m, (root_max + ROOT_CHUNK - 1) / ROOT_CHUNK);
            k_sah_root_refs<<<rgrid, SBLK, 0, st>>>(d_roots + ri, rpre + ri, delta, new_off + ri, in.perm, refs_cur, in.wtri,
                                                    in.kpos);
            k_sah_merge<<<nblk(n_cur + m), SBLK, 0, st>>>(lv_cur, n_cur, d_roots, ri, m, new_off + ri, out_total, lv_tmp,
                                                          out, root_out);
            count_launch(2);
            std::swap(lv_cur, lv_tmp);
            out_total += m;
            n_cur += m;
            r_cur += add;
            ri += m;
        }
        if (n_cur == 0)
        {
            if (run >= runs.size()) { break; }
            depth = runs[run].depth;
            continue;
        }
        levels.emplace_back(lvl_begin, out_total);
        const uint32_t level_bound = next_bound;  // no node of this level has more references
        uint32_t nw = 0, nch = 0;
        if (next_bound > WIDE_MIN)
        {
            k_wide_list<<<1, 1024, 0, st>>>(lv_cur, n_cur, wl, wco, max_wide, io);
            count_launch();
            RT_CUDA(cudaMemcpyAsync(io_h + 8, io + 8, 8, cudaMemcpyDeviceToHost, st));
            RT_CUDA(cudaStreamSynchronize(st));
            nw = io_h[8];
            nch = io_h[9];
            if (nw > max_wide) { return fail(RT_E_CAPACITY, "SAH builder: too many wide nodes"); }
        }
        const uint32_t eval_blocks = std::min<uint32_t>((n_cur + EVAL_WPB - 1) / EVAL_WPB, 8u * (uint32_t)device_sm_count());
        k_sah_eval_warp<true><<<eval_blocks, EVAL_WPB * 32, 0, st>>>(lv_cur, refs_cur, C, S.sah_dec.as<Dec>(), n_cur, io + 13);
        count_launch();
        if (next_bound > EVAL_STAGE)
        {
            k_sah_eval_warp<false><<<eval_blocks, EVAL_WPB * 32, 0, st>>>(lv_cur, refs_cur, C, S.sah_dec.as<Dec>(), n_cur,
                                                                           io + 14);
            count_launch();
        }
        if (next_bound > WARP_MAX)
        {
            k_sah_eval<<<n_cur, SBLK, 0, st>>>(lv_cur, refs_cur, C, S.sah_dec.as<Dec>());
            count_launch();
        }
        if (nw > 0)
        {
            k_wide_init<<<nw, SBLK, 0, st>>>(wacc);
            k_wide_bounds<<<nch, SBLK, 0, st>>>(lv_cur, refs_cur, C, wl, wco, nw, wacc);
            k_wide_bins<<<nch, SBLK, 0, st>>>(lv_cur, refs_cur, C, wl, wco, nw, wacc);
            k_wide_decide<<<nw, 32, 0, st>>>(lv_cur, C, wl, nw, wacc);
            k_wide_counts<<<nch, SBLK, 0, st>>>(lv_cur, refs_cur, C, wl, wco, nw, wacc);
            k_wide_final<<<(nw + 31) / 32, 32, 0, st>>>(lv_cur, C, wl, nw, wacc, S.sah_dec.as<Dec>());
            count_launch(6);
        }
        const uint32_t n_tiles = (n_cur + SO_TILE - 1) / SO_TILE;
        k_sah_need<<<(n_cur + NEED_THREADS - 1) / NEED_THREADS, NEED_THREADS, 0, st>>>(S.sah_dec.as<Dec>(), lv_cur, d_roots,
                                                                                        n_cur, n_budget, d_need, io);
        k_sah_grant<<<1, 1024, 0, st>>>(S.sah_dec.as<Dec>(), lv_cur, d_roots, n_cur, n_budget, d_used, d_used + n_budget,
                                        d_need, io, leaf_offs, d_desc, n_tiles);
        k_sah_offsets<<<n_tiles, SO_THREADS, 0, st>>>(S.sah_dec.as<Dec>(), n_cur, d_desc,
                                                      reinterpret_cast<uint32_t*>(d_desc + 3 * (size_t)n_tiles), io,
                                                      child_slot, ref_offs, leaf_offs);
        count_launch(3);
        if (int e = check_launch("sah eval")) { return e; }
        RT_CUDA(cudaMemcpyAsync(io_h, io, 64, cudaMemcpyDeviceToHost, st));
        RT_CUDA(cudaStreamSynchronize(st));
        if (io_h[12]) { return fail(RT_E_TIMEOUT, "a bounded device wait gave up (SAH level offsets)"); }
        const uint32_t n_next = io_h[3], r_next = io_h[4], leaf_lvl = io_h[5];
        if (n_next > cap || r_next > cap || (uint64_t)out_total + n_next > 2ull * cap || (uint64_t)leaf_total + leaf_lvl > cap)
        {
            return fail(RT_E_CAPACITY, "SAH builder: capacity exceeded");
        }
        // nodes of at most EVAL_STAGE references (all of them in the reference's default hybrid
        // bake, which hands ranges of at most 64 triangles to the SAH) split by one warp each
        k_sah_split_warp<<<(n_cur + SPLIT_WPB - 1) / SPLIT_WPB, SPLIT_WPB * 32, 0, st>>>(
            lv_cur, refs_cur, S.sah_dec.as<Dec>(), child_slot, ref_offs, leaf_offs, C, lv_next, refs_next, out, out_total,
            leaf_total, S.sah_leaf_refs.as<uint32_t>(), n_cur);
        count_launch();
        if (level_bound > EVAL_STAGE)
        {
            k_sah_split<SBLK><<<n_cur, SBLK, 0, st>>>(lv_cur, refs_cur, S.sah_dec.as<Dec>(), child_slot, ref_offs, leaf_offs, C,
                                                      S.sah_tmp.as<uint32_t>(), S.sah_pos.as<uint32_t>(),
                                                      S.sah_scan_in.as<uint8_t>(), lv_next, refs_next, out, out_total, leaf_total,
                                                      S.sah_leaf_refs.as<uint32_t>(), nullptr, EVAL_STAGE + 1);
            count_launch();
        }
        if (nw > 0)
        {
            WideSplit W;
            W.lv = lv_cur; W.dec = S.sah_dec.as<Dec>(); W.wl = wl; W.wco = wco; W.nw = nw; W.acc = wacc;
            W.refs = refs_cur; W.tmp = S.sah_tmp.as<uint32_t>(); W.tmp2 = S.sah_tmp2.as<uint32_t>();
            W.posf = S.sah_pos.as<uint32_t>(); W.poss = S.sah_pos2.as<uint32_t>(); W.flags = S.sah_scan_in.as<uint8_t>();
            W.chunk = wchunk; W.refs_next = refs_next; W.ref_off = ref_offs; W.child_slot = child_slot;
            W.leaf_off = leaf_offs; W.leaf_refs = S.sah_leaf_refs.as<uint32_t>(); W.lv_next = lv_next; W.out = out;
            W.out_base = out_total; W.leaf_base = leaf_total;
            k_wp_flags<0><<<nch, SBLK, 0, st>>>(W, C);
            k_wp_sides<0><<<nch, SBLK, 0, st>>>(W);
            k_wp_pos<0><<<nch, SBLK, 0, st>>>(W);
            k_wp_scatter<0><<<nch, SBLK, 0, st>>>(W);
            k_wp_flags<1><<<nch, SBLK, 0, st>>>(W, C);
            k_wp_sides<1><<<nch, SBLK, 0, st>>>(W);
            k_wp_pos<1><<<nch, SBLK, 0, st>>>(W);
            k_wp_scatter<1><<<nch, SBLK, 0, st>>>(W);
            k_wp_flags<2><<<nch, SBLK, 0, st>>>(W, C);
            k_wp_sides<2><<<nch, SBLK, 0, st>>>(W);
            k_wp_pos<2><<<nch, SBLK, 0, st>>>(W);
            k_wp_scatter<2><<<nch, SBLK, 0, st>>>(W);
            k_wp_place<<<nch, SBLK, 0, st>>>(W, C);
            k_wp_final<<<(nw + 31) / 32, 32, 0, st>>>(W);
            count_launch(14);
        }
        next_bound = io_h[10];
        if (int e = check_launch("sah split")) { return e; }
        out_total += n_next;
        leaf_total += leaf_lvl;
        std::swap(lv_cur, lv_next);
        std::swap(refs_cur, refs_next);
        n_cur = n_next;
        r_cur = r_next;
        depth++;
    }
    // subtree sizes bottom-up, then pre-order slots and triangle offsets top-down
    for (size_t l = levels.size(); l-- > 0;)
    {
        const auto& L = levels[l];
        if (L.second > L.first) { k_sah_up<<<nblk(L.second - L.first), SBLK, 0, st>>>(out, L.first, L.second); count_launch(); }
    }
    for (const auto& L : levels)
    {
        if (L.second > L.first) { k_sah_down<<<nblk(L.second - L.first), SBLK, 0, st>>>(out, L.first, L.second); count_launch(); }
    }
    k_sah_root_weights<<<nblk(nr), SBLK, 0, st>>>(d_roots, nr, root_out, out, in.wnode, in.wtri);
    count_launch();
    if (int e = check_launch("sah finish")) { return e; }
    RT_CUDA(cudaMemcpyAsync(io_h, io, 32, cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    res->spatial_taken = io_h[1];
    res->spatial_refused = io_h[2];
    res->leaves = io_h[6];
    res->nodes = out_total;
    res->levels = (uint32_t)levels.size();
    res->sorted_roots = d_roots;
    return RT_OK;
}

int sah_emit(rt_bvh* B, uint32_t n_roots, const uint32_t* snode, const uint32_t* stri, const rt_triangle* tris,
             cudaStream_t st, const SahResult& res, uint32_t max_nodes, uint32_t max_tris, uint32_t* status)
{
    (void)n_roots;
    BuildScratch& S = B->s;
    if (res.nodes == 0) { return RT_OK; }
    k_sah_emit<<<nblk(res.nodes), SBLK, 0, st>>>(S.sah_out.as<OutNode>(), res.nodes, res.sorted_roots, snode, stri,
                                                  S.sah_leaf_refs.as<uint32_t>(), tris, B->nodes.as<rt_bvh_node>(),
                                                  B->tris.as<rt_triangle>(), B->prim.as<uint32_t>(), max_nodes,
                                                  max_tris, status);
    count_launch();
    return check_launch("sah emit");
}

} // namespace rtb
