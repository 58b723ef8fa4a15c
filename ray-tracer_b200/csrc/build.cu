// build.cu -- the GPU bake: the reference's bvh::bakeBVH (src/bvh/bvh_bake.cpp:180-194) as a
// handful of data-parallel kernels producing the identical tree.
//
//  k_vertices   normal renormalisation of initGeos (src/bvh/bvh_IO.cpp:102-118)
//  k_tri_prep   index check (bvh_IO.cpp:88-99), per-triangle box and centroid
//               (bvh_morton.cpp:88-90, bvh_bake.cpp:50-54), scene box (bvh_morton.cpp:49-59)
//  k_morton     quantisation + 3-way bit interleave (bvh_morton.cpp:19-36,61-101), and the
//               digit histograms of every radix pass
//  radix sort   stable onesweep LSD sort (radix_sort.cu; bvh_morton.cpp:109-159)
//  k_karras     the binary radix tree over the sorted codes (Karras, HPG 2012), every node
//               found independently, and a hierarchy of block boxes over the sorted keys. Its
//               split of a range whose first and last codes differ is the reference's Morton
//               split (the first index where the highest differing bit flips,
//               bvh_bfs.cpp:35-48,98-109); a node's range box, the reference's computeRangeAABB
//               (bvh_bfs.cpp:14-28), is a union of at most 15 hierarchy blocks per level and end
//  k_boundary   the reference stops splitting at <= BVH_MAX_LEAF_SIZE triangles and hands ranges
//               of <= BVH_LBVH_THRESHOLD triangles or of identical codes to the binned SAH
//               (bvh_bfs.cpp:30-33,79-107); this kernel finds those boundary nodes, marks their
//               positions, registers SAH roots and the left-spine ranks of the kept nodes
//  sah.cu       the binned SAH / spatial-split subtrees (bvh_sah.cpp:24-460)
//  k_emit*      the DFS pre-order re-layout of reorderNodes / reorderTriangles
//               (bvh_bake.cpp:75-149): a node's pre-order index is the number of nodes whose
//               key range starts before its own plus its depth on its left spine, so every
//               node finds its output slot from two prefix sums without a tree walk.
#include <atomic>
#include "rt_internal.h"
#include "device_math.cuh"
#include "cta_utils.cuh"
#include "sah.cuh"
#include "layout.cuh"
#include "trace_core.cuh"

#include <algorithm>
#include <cstring>
#include <mutex>

#include <cuda/atomic>

namespace rtb
{
using namespace rtd;

namespace
{

constexpr int BLK = 256;
constexpr uint32_t NONE = 0xffffffffu;
// A Karras tree over n distinct (key, index) pairs is at most key bits + 32 deep.
constexpr uint32_t MAX_DEPTH = 128;

inline uint32_t blocks_for(uint64_t n, int per = BLK) { return (uint32_t)((n + per - 1) / per); }

// Three-argument hypot by scaling with the largest magnitude -- the evaluation the
// reference's std::hypot(float, float, float) performs (pinned bit-exactly by the tests).
__device__ __forceinline__ float hypot3f(float x, float y, float z)
{
    x = fabsf(x); y = fabsf(y); z = fabsf(z);
    const float a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a == 0.0f) { return 0.0f; }
    const float xa = x / a, ya = y / a, za = z / a;
    return a * sqrtf(xa * xa + ya * ya + za * za);
}

// Spreads the low 21 bits of v so that bit i lands on bit 3i (the standard
// shift-and-mask interleave for 3-D Morton codes).
__device__ __forceinline__ uint64_t spread3(uint32_t v)
{
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// Batched builds (rt_build_batch): scene s owns input triangles [toff[s], toff[s+1]) whose
// vertex indices are local to vertices [voff[s], voff[s+1]). Every scene gets its own box for
// its Morton codes, and its id is placed above the code bits of the sort key (shift `sshift`),
// so the radix tree first separates the scenes and each scene's subtree is the tree of that
// scene alone. S = 0: a single scene (no offsets; sshift = 63 never sees a set bit).
struct Batch
{
    uint32_t        S;
    const uint32_t* toff;
    const uint32_t* voff;
    uint32_t        sshift;
    const uint32_t* h_toff;  // host copy of toff
};
constexpr uint32_t MAX_BATCH_SCENES = 1024;

// Key bits that hold a scene id below S.
inline uint32_t scene_bits(uint32_t S)
{
    uint32_t b = 0;
    while ((1u << b) < S) { b++; }
    return b;
}

// Scene of input triangle i: the last s with toff[s] <= i (toff in shared memory).
__device__ __forceinline__ uint32_t scene_of(const uint32_t* toff, uint32_t S, uint32_t i)
{
    uint32_t lo = 0, hi = S;  // toff[lo] <= i < toff[hi]
    while (hi - lo > 1)
    {
        const uint32_t mid = (lo + hi) >> 1;
        if (toff[mid] <= i) { lo = mid; } else { hi = mid; }
    }
    return lo;
}

__global__ void k_init(uint32_t* scene, uint32_t* hist, uint32_t* counters, uint32_t* status)
{
    const int t = threadIdx.x;
    if (t < 3) { scene[t] = 0xffffffffu; scene[3 + t] = 0u; }
    for (int i = t; i < 8 * 256; i += blockDim.x) { hist[i] = 0u; }
    if (t < 16) { counters[t] = 0u; }
    if (t == 0) { *status = 0u; }
}

__global__ void __launch_bounds__(BLK) k_vertices(const rt_vertex* __restrict__ in, rt_vertex* __restrict__ out, uint32_t V)
{
    const uint32_t i = blockIdx.x * BLK + threadIdx.x;
    if (i >= V) { return; }
    rt_vertex v = in[i];
    const float len = hypot3f(v.nx, v.ny, v.nz);
    if (len > 1e-6f) { v.nx /= len; v.ny /= len; v.nz /= len; }
    else { v.nx = 0.f; v.ny = 1.f; v.nz = 0.f; }
    out[i] = v;
}

__device__ __forceinline__ f3 vpos(const rt_vertex* v, uint32_t i)
{
    const rt_vertex& p = v[i];
    return mk3(p.x, p.y, p.z);
}

// Per triangle: index check, box (lo.xyz/hi.xyz) with the centroid in lo.w, hi.w, cz.
// Block-reduces the scene box into `scene` (order-preserving uint encoding). In a batched
// build the triangle's scene box is scene[6 s ..] and its vertex indices are rebased to the
// concatenated vertex array (written to gtris).
template <bool BATCH>
__global__ void __launch_bounds__(BLK)
k_tri_prep(const rt_triangle* __restrict__ tris, uint32_t N, const rt_vertex* __restrict__ verts, uint32_t V,
           float4* __restrict__ lo, float4* __restrict__ hi, float* __restrict__ cz, uint32_t* __restrict__ scene,
           uint32_t* __restrict__ status, Batch bt, rt_triangle* __restrict__ gtris, float4* __restrict__ tpin)
{
    const uint32_t i = blockIdx.x * BLK + threadIdx.x;
    __shared__ uint32_t soff[BATCH ? MAX_BATCH_SCENES + 1 : 1];
    if (BATCH)
    {
        for (uint32_t k = threadIdx.x; k <= bt.S; k += BLK) { soff[k] = bt.toff[k]; }
        __syncthreads();
    }
    uint32_t om[3] = { 0xffffffffu, 0xffffffffu, 0xffffffffu }, oM[3] = { 0u, 0u, 0u };
    uint32_t sc = 0;
    if (i < N)
    {
        uint32_t a = tris[i].v[0], b = tris[i].v[1], c = tris[i].v[2];
        uint32_t vb = 0, vn = V;
        if (BATCH)
        {
            sc = scene_of(soff, bt.S, i);
            vb = bt.voff[sc];
            vn = bt.voff[sc + 1] - vb;
        }
        if (a >= vn || b >= vn || c >= vn) { atomicOr(status, ST_INDEX); a = b = c = 0; }
        a += vb; b += vb; c += vb;
        if (BATCH) { gtris[i] = rt_triangle{ { a, b, c } }; }
        const f3 p0 = vpos(verts, a), p1 = vpos(verts, b), p2 = vpos(verts, c);
        box3 bx = box_empty();
        box_pt(bx, p0); box_pt(bx, p1); box_pt(bx, p2);
        const float cx = (p0.x + p1.x + p2.x) / 3.0f;
        const float cy = (p0.y + p1.y + p2.y) / 3.0f;
        const float czv = (p0.z + p1.z + p2.z) / 3.0f;
        lo[i] = make_float4(bx.mn[0], bx.mn[1], bx.mn[2], cx);
        hi[i] = make_float4(bx.mx[0], bx.mx[1], bx.mx[2], cy);
        cz[i] = czv;
        if (tpin)
        {
            // the triangle's positions and vertex indices in one 48-byte record (input order), so
            // that the sorted passes gather one record per triangle
            tpin[3 * (size_t)i + 0] = make_float4(p0.x, p0.y, p0.z, p1.x);
            tpin[3 * (size_t)i + 1] = make_float4(p1.y, p1.z, p2.x, p2.y);
            tpin[3 * (size_t)i + 2] = make_float4(p2.z, __uint_as_float(a), __uint_as_float(b), __uint_as_float(c));
        }
        for (int k = 0; k < 3; k++) { om[k] = f2ord(bx.mn[k]); oM[k] = f2ord(bx.mx[k]); }
    }
    if (BATCH)
    {
        // warps inside one scene reduce first; a warp across a scene boundary adds per lane
        const uint32_t s0 = __shfl_sync(0xffffffffu, sc, 0);
        const bool uniform = __all_sync(0xffffffffu, i >= N || sc == s0);
        for (int k = 0; k < 3; k++)
        {
            uint32_t m = om[k], M = oM[k];
            if (uniform)
            {
                for (int o = 16; o > 0; o >>= 1)
                {
                    m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
                    M = max(M, __shfl_xor_sync(0xffffffffu, M, o));
                }
                if ((threadIdx.x & 31) == 0 && m != 0xffffffffu) { atomicMin(&scene[6 * s0 + k], m); atomicMax(&scene[6 * s0 + 3 + k], M); }
            }
            else if (i < N) { atomicMin(&scene[6 * sc + k], m); atomicMax(&scene[6 * sc + 3 + k], M); }
        }
        return;
    }
    __shared__ uint32_t s[6];
    if (threadIdx.x < 3) { s[threadIdx.x] = 0xffffffffu; s[3 + threadIdx.x] = 0u; }
    __syncthreads();
    for (int k = 0; k < 3; k++)
    {
        uint32_t m = om[k], M = oM[k];
        for (int o = 16; o > 0; o >>= 1)
        {
            m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
            M = max(M, __shfl_xor_sync(0xffffffffu, M, o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&s[k], m); atomicMax(&s[3 + k], M); }
    }
    __syncthreads();
    if (threadIdx.x < 3)
    {
        atomicMin(&scene[threadIdx.x], s[threadIdx.x]);
        atomicMax(&scene[3 + threadIdx.x], s[3 + threadIdx.x]);
    }
}

// Morton code per triangle (input order) and the 8-bit digit histograms of all sort passes
// (hist[256 p + d], digit d of bits 8p .. 8p+7); with msd_shift >= 0 also the histogram of
// bits msd_shift .. msd_shift+7 (the key's top digit) in hist[8 * 256 + d].
template <typename K, bool BATCH = false>
__global__ void __launch_bounds__(BLK)
k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, const float* __restrict__ cz, uint32_t N,
         const uint32_t* __restrict__ scene, uint32_t bits, int passes, K* __restrict__ keys, uint32_t* __restrict__ hist,
         int msd_shift = -1, Batch bt = Batch{ 0u, nullptr, nullptr, 63u, nullptr })
{
    // grid-stride: the block histograms are flushed to global memory once per block, so the
    // launch uses a few blocks per SM rather than one block per 256 triangles
    __shared__ uint32_t h[9 * 256];
    __shared__ uint32_t soff[BATCH ? MAX_BATCH_SCENES + 1 : 1];
    for (int t = threadIdx.x; t < 9 * 256; t += BLK) { h[t] = 0u; }
    if (BATCH)
    {
        for (uint32_t k = threadIdx.x; k <= bt.S; k += BLK) { soff[k] = bt.toff[k]; }
    }
    __syncthreads();
    float mn[3], size[3];
    uint32_t cur = 0xffffffffu;  // scene whose box is in mn/size
    const uint32_t qmax = (1u << bits) - 1u;
    const float fmax = (float)qmax;
    for (uint32_t i = blockIdx.x * BLK + threadIdx.x; i < N; i += gridDim.x * BLK)
    {
        const uint32_t sc = BATCH ? scene_of(soff, bt.S, i) : 0u;
        if (sc != cur)
        {
            cur = sc;
            for (int k = 0; k < 3; k++)
            {
                mn[k] = ord2f(scene[6 * sc + k]);
                size[k] = ord2f(scene[6 * sc + 3 + k]) - mn[k];
                if (size[k] == 0.f) { size[k] = 1.f; }
            }
        }
        const float c[3] = { lo[i].w, hi[i].w, cz[i] };
        uint32_t q[3];
        for (int k = 0; k < 3; k++)
        {
            const uint32_t v = x86_f2u((c[k] - mn[k]) * fmax / size[k]);
            q[k] = v > qmax ? qmax : v;
        }
        uint64_t code = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
        if (BATCH) { code |= (uint64_t)sc << bt.sshift; }
        keys[i] = (K)code;
        for (int p = 0; p < passes; p++) { atomicAdd(&h[p * 256 + (uint32_t)((code >> (8 * p)) & 255u)], 1u); }
        if (msd_shift >= 0) { atomicAdd(&h[8 * 256 + (uint32_t)((code >> msd_shift) & 255u)], 1u); }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 9 * 256; t += BLK)
    {
        const bool used = t < passes * 256 || (msd_shift >= 0 && t >= 8 * 256);  // hist may hold 8 x 256 words only
        if (used && h[t]) { atomicAdd(&hist[t], h[t]); }
    }
}

// Node ids of the binary radix tree: inner 0..n-2, leaf k -> n-1+k; knode = {first, last,
// left, right} (built by k_karras below).
template <typename K>
__device__ __forceinline__ void krange(const uint4* __restrict__ knode, uint32_t n, uint32_t x, uint32_t& f, uint32_t& l)
{
    if (x < n - 1) { const uint4 k = knode[x]; f = k.x; l = k.y; }
    else { f = l = x - (n - 1); }
}

__device__ __forceinline__ void store_box(float4* kbox, uint32_t x, const box3& b)
{
    __stcg(&kbox[2 * x], make_float4(b.mn[0], b.mn[1], b.mn[2], 0.f));
    __stcg(&kbox[2 * x + 1], make_float4(b.mx[0], b.mx[1], b.mx[2], 0.f));
}
__device__ __forceinline__ box3 load_box(const float4* kbox, uint32_t x)
{
    const float4 a = __ldcg(&kbox[2 * x]), c = __ldcg(&kbox[2 * x + 1]);
    box3 b;
    b.mn[0] = a.x; b.mn[1] = a.y; b.mn[2] = a.z; b.mx[0] = c.x; b.mx[1] = c.y; b.mx[2] = c.z;
    return b;
}

// ---- the binary radix tree (Karras, "Maximizing Parallelism in the Construction of BVHs,
// Octrees, and k-d Trees", HPG 2012) and the boxes of key ranges ----
//
// Inner node i (0 <= i < n - 1) of the tree over the sorted keys, each extended by its index so
// that equal codes still differ, covers a key range with one end at i: its direction and other
// end come from an exponential and a binary search on the length of the common prefix, its
// split from one more binary search. Every node is found independently (no climb, no atomics).
// The split of a range whose first and last codes differ is the reference's Morton split (the
// first index where the highest differing bit flips, bvh_bfs.cpp:35-48,98-109).
//
// A node's box is the reference's computeRangeAABB (bvh_bfs.cpp:14-28): the union of the boxes
// of the triangles in its key range. Level 0 of a hierarchy is the sorted keys, level k + 1 has
// one element per 16 elements of level k (its box: their union, `blk`), and every element of
// levels 0 .. top - 1 also has the union from the start of its group of 16 up to itself (`pre`)
// and from itself to the end of the group (`suf`). A range whose ends lie in different groups
// is then `suf` of its first element, `pre` of its last, and the same two entries one level up
// for the groups strictly between, until both ends share a group: at most 2 loads per level plus
// 14 at the top, all independent of one another (range_box). k_karras builds levels 0 and 1,
// k_box_levels level 2 and, in its last block, the levels above.
constexpr uint32_t LV_FAN = 16;
constexpr int LV_MAX = 8;  // 16^8 = 2^32 keys

// Elements of level k over n keys, and the number of levels below the first one-element level.
__host__ __device__ __forceinline__ uint64_t lv_count(uint32_t n, int k) { return ((uint64_t)n + (1ull << (4 * k)) - 1) >> (4 * k); }
inline int lv_top(uint32_t n)
{
    int k = 0;
    while (k < LV_MAX && lv_count(n, k) > 1) { k++; }
    return k;
}
// Offset (in boxes) of level k in the pre / suf arrays (levels 0 ..) and in the blk array
// (levels 1 ..): the counts of the levels before it.
__host__ __device__ __forceinline__ uint64_t lv_off(uint32_t n, int k, int first)
{
    uint64_t o = 0;
    for (int j = first; j < k; j++) { o += lv_count(n, j); }
    return o;
}

struct BoxLevels
{
    float4* pre;  // 2 float4 (min, max) per element of levels 0 .. top - 1
    float4* suf;
    float4* blk;  // levels 1 .. top
    uint32_t n;
    int top;
};

__device__ __forceinline__ void box_union(box3& b, float4 mn, float4 mx)
{
    b.mn[0] = sse_min(b.mn[0], mn.x); b.mn[1] = sse_min(b.mn[1], mn.y); b.mn[2] = sse_min(b.mn[2], mn.z);
    b.mx[0] = sse_max(b.mx[0], mx.x); b.mx[1] = sse_max(b.mx[1], mx.y); b.mx[2] = sse_max(b.mx[2], mx.z);
}
__device__ __forceinline__ void box_union_at(box3& b, const float4* __restrict__ a, uint64_t e)
{
    box_union(b, __ldcg(&a[2 * e]), __ldcg(&a[2 * e + 1]));
}
__device__ __forceinline__ void put_box(float4* __restrict__ a, uint64_t e, float4 mn, float4 mx)
{
    __stcg(&a[2 * e], mn);
    __stcg(&a[2 * e + 1], mx);
}

// Box of the triangles of sorted keys [f, l] (inclusive).
__device__ box3 range_box(const uint32_t* __restrict__ perm, const float4* __restrict__ lo, const float4* __restrict__ hi,
                          const BoxLevels& V, uint32_t f, uint32_t l)
{
    box3 b = box_empty();
    if ((f >> 4) == (l >> 4))  // one group of 16 keys: its triangles' boxes
    {
#pragma unroll
        for (uint32_t q = 0; q < LV_FAN; q++)
        {
            if (f + q <= l) { const uint32_t t = perm[f + q]; box_union(b, lo[t], hi[t]); }
        }
        return b;
    }
    box_union_at(b, V.suf, f);
    box_union_at(b, V.pre, l);
    uint64_t a = f >> 4, c = l >> 4, off_ps = V.n, off_blk = 0;
#pragma unroll
    for (int k = 1; k < LV_MAX; k++)
    {
        // elements a + 1 .. c - 1 of level k are still to be covered
        if (a + 1 >= c) { break; }
        if ((a >> 4) == (c >> 4))
        {
#pragma unroll
            for (uint32_t q = 1; q < LV_FAN - 1; q++)
            {
                if (a + q < c) { box_union_at(b, V.blk, off_blk + a + q); }
            }
            break;
        }
        if ((a & 15u) != 15u) { box_union_at(b, V.suf, off_ps + a + 1); }
        if ((c & 15u) != 0u) { box_union_at(b, V.pre, off_ps + c - 1); }
        off_ps += lv_count(V.n, k);
        off_blk += lv_count(V.n, k);
        a >>= 4;
        c >>= 4;
    }
    return b;
}

// Prefix and suffix unions over each group of 16 lanes of a full warp (lane 0 of a group ends
// with the group's total as its suffix).
__device__ __forceinline__ void group_scans(float4 mn, float4 mx, float4& pmn, float4& pmx, float4& smn, float4& smx)
{
    const uint32_t g = threadIdx.x & 15u;
    pmn = mn; pmx = mx; smn = mn; smx = mx;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1)
    {
        const float ax = __shfl_up_sync(0xffffffffu, pmn.x, o, 16), ay = __shfl_up_sync(0xffffffffu, pmn.y, o, 16);
        const float az = __shfl_up_sync(0xffffffffu, pmn.z, o, 16);
        const float bx = __shfl_up_sync(0xffffffffu, pmx.x, o, 16), by = __shfl_up_sync(0xffffffffu, pmx.y, o, 16);
        const float bz = __shfl_up_sync(0xffffffffu, pmx.z, o, 16);
        const float cx = __shfl_down_sync(0xffffffffu, smn.x, o, 16), cy = __shfl_down_sync(0xffffffffu, smn.y, o, 16);
        const float cz = __shfl_down_sync(0xffffffffu, smn.z, o, 16);
        const float dx = __shfl_down_sync(0xffffffffu, smx.x, o, 16), dy = __shfl_down_sync(0xffffffffu, smx.y, o, 16);
        const float dz = __shfl_down_sync(0xffffffffu, smx.z, o, 16);
        if (g >= (uint32_t)o)
        {
            pmn.x = sse_min(pmn.x, ax); pmn.y = sse_min(pmn.y, ay); pmn.z = sse_min(pmn.z, az);
            pmx.x = sse_max(pmx.x, bx); pmx.y = sse_max(pmx.y, by); pmx.z = sse_max(pmx.z, bz);
        }
        if (g + (uint32_t)o < 16u)
        {
            smn.x = sse_min(smn.x, cx); smn.y = sse_min(smn.y, cy); smn.z = sse_min(smn.z, cz);
            smx.x = sse_max(smx.x, dx); smx.y = sse_max(smx.y, dy); smx.z = sse_max(smx.z, dz);
        }
    }
}

__device__ __forceinline__ void empty_box4(float4& mn, float4& mx)
{
    const float inf = bits2f(0x7f800000u), ninf = bits2f(0xff800000u);
    mn = make_float4(inf, inf, inf, 0.f);
    mx = make_float4(ninf, ninf, ninf, 0.f);
}

// One level of the hierarchy from level k's element boxes, called by whole warps (element e,
// 16-aligned groups; lanes with valid = false carry an empty box and write nothing): pre / suf
// of every element and the blk box of every group (level k + 1).
__device__ __forceinline__ void level_from(const BoxLevels& V, int k, uint64_t e, bool valid, float4 mn, float4 mx)
{
    float4 pmn, pmx, smn, smx;
    group_scans(mn, mx, pmn, pmx, smn, smx);
    if (!valid || e >= lv_count(V.n, k)) { return; }
    const uint64_t o = lv_off(V.n, k, 0);
    put_box(V.pre, o + e, pmn, pmx);
    put_box(V.suf, o + e, smn, smx);
    // the group's union is its first lane's suffix
    if ((e & 15u) == 0) { put_box(V.blk, lv_off(V.n, k + 1, 1) + (e >> 4), smn, smx); }
}

// Length of the common prefix of sorted keys a and b extended by their indices; -1 when b is
// outside the keys.
template <typename K>
__device__ __forceinline__ int prefix_len(const K* __restrict__ keys, uint32_t n, uint32_t a, int64_t b)
{
    if (b < 0 || b >= (int64_t)n) { return -1; }
    const K x = keys[a] ^ keys[(uint32_t)b];
    constexpr int W = 8 * (int)sizeof(K);
    if (x == 0) { return W + __clz(a ^ (uint32_t)b); }
    return sizeof(K) == 8 ? __clzll((unsigned long long)x) : __clz((unsigned int)x);
}

// Bucket table of the sorted keys: tab[b] = the first index whose top `tb` key bits are >= b,
// for b = 0 .. 2^tb (tab[2^tb] = n). One thread per key writes the entries between its
// predecessor's bucket and its own; thread n the entries past the last key. msd_flag (or
// nullptr): the sort's MSD flag when its per-bucket pass writes the table; it is built here
// only when that pass did not run (the flag is set).
template <typename K>
__global__ void __launch_bounds__(BLK)
k_bucket_table(const K* __restrict__ keys, uint32_t n, int kshift, uint32_t tb_size, uint32_t* __restrict__ tab,
               const uint32_t* __restrict__ abort_flag, const uint32_t* __restrict__ msd_flag)
{
    if (*abort_flag) { return; }
    if (msd_flag && *msd_flag == 0u) { return; }  // the sort's per-bucket pass wrote the table
    // grid-stride (a small grid, so that the usual early return costs little)
    for (uint32_t i = blockIdx.x * BLK + threadIdx.x; i <= n; i += gridDim.x * BLK)
    {
        const uint64_t b = i < n ? (uint64_t)(keys[i] >> kshift) : (uint64_t)tb_size;
        const uint64_t b0 = i == 0 ? 0 : (uint64_t)(keys[i - 1] >> kshift) + 1u;
        for (uint64_t q = b0; q <= b; q++) { tab[q] = i; }
    }
}

// The reference splits a node by Morton code (it is "Morton-split") if it has more triangles
// than the leaf size and the SAH threshold and its codes are not all equal, or if it spans
// scenes of a batched build (bvh_bfs.cpp:79-107).
template <typename K>
__device__ __forceinline__ bool morton_split_keys(K kf, K kl, uint32_t size, uint32_t tm, uint32_t sshift)
{
    const uint64_t x = (uint64_t)(kf ^ kl);
    return (size > tm && x != 0) || (x >> sshift) != 0;
}

// Per node flags written by the node's parent (the root's by thread 0): bit 0 kept (the parent
// is Morton-split, or it is the root), bit 1 the node itself is Morton-split.
constexpr uint8_t KF_KEPT = 1u, KF_MSPLIT = 2u;

// One thread per sorted key i: level 0 (key i's triangle box) and level 1 of the box hierarchy;
// inner node i ({first, last, left, right}; leaf k has id n - 1 + k), the parent of its two
// children and their flags. The node's range is all keys sharing one more leading bit with key i
// than its neighbour on the other side does; with the bucket table over the top `tb` key bits
// (key_bits in all) the range, and then the split, are table lookups when that prefix is at most
// tb bits long, and short binary searches inside one bucket otherwise; runs of equal keys
// (split by the index bits) take the general exponential and binary searches.
template <typename K>
__global__ void __launch_bounds__(BLK)
k_karras(const K* __restrict__ keys, const uint32_t* __restrict__ perm, uint32_t n, const float4* __restrict__ lo,
         const float4* __restrict__ hi, uint4* __restrict__ knode, uint32_t* __restrict__ parent,
         uint8_t* __restrict__ kflag, const uint32_t* __restrict__ tab, int key_bits, int tb, uint32_t tm,
         uint32_t sshift, BoxLevels V, const float4* __restrict__ tpin,
         rt_triangle* __restrict__ out_tris, uint32_t* __restrict__ prim, float4* __restrict__ tp,
         uint32_t* __restrict__ status, const uint32_t* __restrict__ abort_flag)
{
    static_assert(BLK == LV_FAN * LV_FAN, "one block of threads covers one level-2 element");
    __shared__ float4 s_mn[LV_FAN], s_mx[LV_FAN];
    if (*abort_flag) { return; }  // (uniform over the grid)
    const uint32_t i = blockIdx.x * BLK + threadIdx.x;
    float4 mn, mx;
    empty_box4(mn, mx);
    if (i < n)
    {
        // key i's triangle: positions and vertex indices from its 48-byte record; its box as
        // k_tri_prep forms it (the same min / max sequence over the three vertices)
        const uint32_t t = perm[i];
        const float4 r0 = tpin[3 * (size_t)t], r1 = tpin[3 * (size_t)t + 1], r2 = tpin[3 * (size_t)t + 2];
        box3 bx = box_empty();
        box_pt(bx, mk3(r0.x, r0.y, r0.z));
        box_pt(bx, mk3(r0.w, r1.x, r1.y));
        box_pt(bx, mk3(r1.z, r1.w, r2.x));
        mn = make_float4(bx.mn[0], bx.mn[1], bx.mn[2], 0.f);
        mx = make_float4(bx.mx[0], bx.mx[1], bx.mx[2], 0.f);
        if (out_tris)
        {
            // the baked triangle at position i when the tree has no SAH subtrees (then every key is
            // in a Morton leaf, in key order): the .bvh triangle, its input index and its
            // traversal position record
            out_tris[i] = rt_triangle{ { __float_as_uint(r2.y), __float_as_uint(r2.z), __float_as_uint(r2.w) } };
            prim[i] = t;
            tp[3 * (size_t)i + 0] = r0;
            tp[3 * (size_t)i + 1] = r1;
            tp[3 * (size_t)i + 2] = make_float4(r2.x, 0.f, 0.f, 0.f);
        }
    }
    {
        float4 pmn, pmx, smn, smx;
        group_scans(mn, mx, pmn, pmx, smn, smx);
        if (i < n) { put_box(V.pre, i, pmn, pmx); put_box(V.suf, i, smn, smx); }
        if ((threadIdx.x & 15u) == 0) { s_mn[threadIdx.x >> 4] = smn; s_mx[threadIdx.x >> 4] = smx; }
    }
    if (n >= 2 && i < n - 1)
    {
        constexpr int W = 8 * (int)sizeof(K);
        const int lead = W - key_bits;  // leading bits every key has zero
        const K ki = keys[i];
        const int dR = prefix_len<K>(keys, n, i, (int64_t)i + 1), dL = prefix_len<K>(keys, n, i, (int64_t)i - 1);
        const int d = dR > dL ? 1 : -1;
        const int dmin = d > 0 ? dL : dR;
        uint32_t f, l;
        const int p = dmin + 1 - lead;  // key bits the range shares
        if (dmin < W && p <= 0) { f = 0; l = n - 1; }
        else if (dmin < W && p <= tb)
        {
            const uint64_t P = (uint64_t)(ki >> (key_bits - p));
            f = tab[P << (tb - p)];
            l = tab[(P + 1) << (tb - p)] - 1u;
        }
        else if (dmin < W)
        {
            // the range lies inside key i's bucket: the farthest key in direction d that still
            // shares dmin + 1 bits with key i
            const uint64_t b = (uint64_t)(ki >> (key_bits - tb));
            const uint32_t lim = d > 0 ? tab[b + 1] - 1u - i : i - tab[b];
            uint32_t len = 0;
            for (uint32_t t = lim ? 1u << (31 - __clz(lim)) : 0u; t >= 1; t >>= 1)
            {
                if (len + t <= lim && prefix_len<K>(keys, n, i, (int64_t)i + (int64_t)(len + t) * d) > dmin) { len += t; }
            }
            const int64_t j = (int64_t)i + (int64_t)len * d;
            f = (uint32_t)min((int64_t)i, j);
            l = (uint32_t)max((int64_t)i, j);
        }
        else
        {
            uint64_t lmax = 2;
            while (prefix_len<K>(keys, n, i, (int64_t)i + (int64_t)lmax * d) > dmin) { lmax <<= 1; }
            uint64_t len = 0;
            for (uint64_t t = lmax >> 1; t >= 1; t >>= 1)
            {
                if (prefix_len<K>(keys, n, i, (int64_t)i + (int64_t)(len + t) * d) > dmin) { len += t; }
            }
            const int64_t j = (int64_t)i + (int64_t)len * d;
            f = (uint32_t)min((int64_t)i, j);
            l = (uint32_t)max((int64_t)i, j);
        }
        // the split: the last key before the highest bit in which the range's ends differ flips
        const K kf = keys[f], kl = keys[l];
        uint32_t g;
        if (kf == kl)
        {
            const int hb = 31 - __clz(f ^ l);  // a run of equal keys splits by the index bits
            g = ((l >> hb) << hb) - 1u;
        }
        else
        {
            const int dn = prefix_len<K>(keys, n, f, (int64_t)l);
            const int pn = dn - lead;  // key bits the whole range shares
            if (pn + 1 <= tb)
            {
                const uint64_t P = pn == 0 ? 0ull : (uint64_t)(kf >> (key_bits - pn));
                g = tab[((P << 1) | 1ull) << (tb - pn - 1)] - 1u;
            }
            else
            {
                uint32_t s = 0;
                const uint32_t lim = l - f - 1u;
                for (uint32_t t = lim ? 1u << (31 - __clz(lim)) : 0u; t >= 1; t >>= 1)
                {
                    if (s + t <= lim && prefix_len<K>(keys, n, f, (int64_t)f + s + t) > dn) { s += t; }
                }
                g = f + s;
            }
        }
        if (g < f || g >= l || (d > 0 ? f != i : l != i)) { atomicOr(status, ST_CAPACITY); }
        else
        {
            const uint32_t left = g == f ? n - 1 + g : g;
            const uint32_t right = g + 1 == l ? n + g : g + 1;
            knode[i] = make_uint4(f, l, left, right);
            parent[left] = i;
            parent[right] = i;
            const bool ms = morton_split_keys<K>(kf, kl, l - f + 1u, tm, sshift);
            const K kg = keys[g], kg1 = keys[g + 1];
            const uint8_t kept = ms ? KF_KEPT : 0u;
            kflag[left] = kept | (g > f && morton_split_keys<K>(kf, kg, g - f + 1u, tm, sshift) ? KF_MSPLIT : 0u);
            kflag[right] = kept | (g + 1 < l && morton_split_keys<K>(kg1, kl, l - g, tm, sshift) ? KF_MSPLIT : 0u);
            if (i == 0) { kflag[0] = KF_KEPT | (ms ? KF_MSPLIT : 0u); }  // the root (its range is all keys)
        }
    }
    // level 1: the block's 16 groups of keys, in the first warp (its upper half idle)
    __syncthreads();
    if (threadIdx.x < 32 && V.top >= 1)
    {
        const bool mine = threadIdx.x < LV_FAN;
        const uint64_t e = (uint64_t)blockIdx.x * LV_FAN + (threadIdx.x & 15u);
        const bool valid = mine && e < lv_count(n, 1);
        float4 a, c;
        empty_box4(a, c);
        if (valid)
        {
            a = s_mn[threadIdx.x];
            c = s_mx[threadIdx.x];
            put_box(V.blk, e, a, c);  // level 1 starts the blk array
        }
        if (V.top >= 2) { level_from(V, 1, e, valid, a, c); }
    }
}

// Level 2 from level 1 (one thread per level-1 group), then, in the last block to finish, the
// levels above.
__global__ void __launch_bounds__(BLK) k_box_levels(BoxLevels V, uint32_t* __restrict__ ticket,
                                                    const uint32_t* __restrict__ abort_flag)
{
    __shared__ uint32_t s_last;
    if (*abort_flag) { return; }  // (uniform over the grid)
    if (V.top >= 3)
    {
        const uint64_t e = (uint64_t)blockIdx.x * BLK + threadIdx.x;  // level-2 element
        float4 mn, mx;
        empty_box4(mn, mx);
        if (e < lv_count(V.n, 2))
        {
            const uint64_t o = lv_off(V.n, 2, 1) + e;
            mn = __ldcg(&V.blk[2 * o]);
            mx = __ldcg(&V.blk[2 * o + 1]);
        }
        level_from(V, 2, e, true, mn, mx);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) { s_last = atomicAdd(ticket, 1u) == gridDim.x - 1u ? 1u : 0u; }
    __syncthreads();
    if (!s_last) { return; }
    __threadfence();
    for (int k = 3; k < V.top; k++)
    {
        const uint64_t cnt = lv_count(V.n, k);
        for (uint64_t e0 = 0; e0 < cnt; e0 += BLK)
        {
            const uint64_t e = e0 + threadIdx.x;
            float4 mn, mx;
            empty_box4(mn, mx);
            if (e < cnt)
            {
                const uint64_t o = lv_off(V.n, k, 1) + e;
                mn = __ldcg(&V.blk[2 * o]);
                mx = __ldcg(&V.blk[2 * o + 1]);
            }
            level_from(V, k, e, true, mn, mx);
        }
        __threadfence_block();
        __syncthreads();
    }
}

// One thread per Karras node. Kept nodes (Morton-split nodes and the boundary nodes right
// below them) record their left-spine rank and their range box; boundary nodes also mark their
// positions and register SAH roots.
template <typename K>
__global__ void __launch_bounds__(BLK)
k_boundary(const K* __restrict__ keys, const uint32_t* __restrict__ perm, uint32_t n, const uint4* __restrict__ knode,
           const uint32_t* __restrict__ parent, const float4* __restrict__ lo, const float4* __restrict__ hi,
           BoxLevels V,
           uint32_t tm, uint32_t max_leaf, uint32_t sshift, float4* __restrict__ kbox, uint32_t* __restrict__ rank,
           uint32_t* __restrict__ wnode, uint32_t* __restrict__ wtri,
           uint8_t* __restrict__ kpos, SahRoot* __restrict__ roots, uint32_t* __restrict__ counters,
           const uint8_t* __restrict__ kflag, uint32_t* __restrict__ status, const uint32_t* __restrict__ abort_flag)
{
    const uint32_t x = blockIdx.x * BLK + threadIdx.x;
    if (x >= 2 * n - 1 || *abort_flag) { return; }
    const uint8_t fl = kflag[x];
    if (!(fl & KF_KEPT)) { return; }
    const bool is_m = (fl & KF_MSPLIT) != 0;
    uint32_t f, l;
    krange<K>(knode, n, x, f, l);
    const uint32_t par = parent[x];

    // left-spine rank: consecutive steps up while this chain is a left child
    uint32_t r = 0, cur = x, p = par;
    while (p != NONE && knode[p].z == cur)
    {
        r++; cur = p; p = parent[p];
        if (r > MAX_DEPTH) { atomicOr(status, ST_CAPACITY); return; }
    }
    rank[x] = r;
    // the exact range box (computeRangeAABB): from the box hierarchy for an inner node, the
    // triangle's own box for a single-key leaf
    box3 b;
    if (x < n - 1)
    {
        b = range_box(perm, lo, hi, V, f, l);
        store_box(kbox, x, b);
    }
    if (is_m) { return; }

    const uint32_t size = l - f + 1u;
    if (x >= n - 1)
    {
        const uint32_t t = perm[f];
        const float4 a = lo[t], c = hi[t];
        b.mn[0] = a.x; b.mn[1] = a.y; b.mn[2] = a.z; b.mx[0] = c.x; b.mx[1] = c.y; b.mx[2] = c.z;
        store_box(kbox, x, b);
    }
    if (size <= max_leaf)
    {
        wnode[f] = r + 1u;  // its keys' wtri and kpos are 1 from k_clear
    }
    else
    {
        // an SAH subtree root: the SAH builder clears its keys' wtri / kpos, then counts and places
        // their triangles
        uint32_t depth = 0;
        for (uint32_t q = par; q != NONE; q = parent[q])
        {
            if (++depth > MAX_DEPTH) { atomicOr(status, ST_CAPACITY); return; }
        }
        // one atomic per warp for the roots of its lanes
        const unsigned m = __activemask();
        const int lane = (int)(threadIdx.x & 31u), leader = __ffs(m) - 1;
        uint32_t base = 0;
        if (lane == leader) { base = atomicAdd(&counters[0], (uint32_t)__popc(m)); }
        base = __shfl_sync(m, base, leader);
        const uint32_t slot = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
        SahRoot sr;
        sr.kid = x; sr.first = f; sr.count = size; sr.depth = depth; sr.rank = r;
        sr.scene = (uint32_t)((uint64_t)keys[f] >> sshift);
        for (int k = 0; k < 3; k++) { sr.box[k] = b.mn[k]; sr.box[3 + k] = b.mx[k]; }
        roots[slot] = sr;
    }
}

// Output slots of the kept Karras nodes: pre-order index = snode[first] + rank.
// In a batched build, the node covering exactly one scene's keys is that scene's root; it
// records {root node, subtree node count, first triangle, triangle count} in info[4 s ..].
template <typename K>
__global__ void __launch_bounds__(BLK)
k_emit(const K* __restrict__ keys, uint32_t n, const uint4* __restrict__ knode, const uint32_t* __restrict__ parent,
       uint32_t tm, uint32_t max_leaf, uint32_t sshift, const float4* __restrict__ kbox, const uint32_t* __restrict__ rank,
       const uint32_t* __restrict__ snode, const uint32_t* __restrict__ stri, rt_bvh_node* __restrict__ out,
       uint32_t max_nodes, uint32_t* __restrict__ info, const uint8_t* __restrict__ kflag, float* __restrict__ gn,
       TraceRoot* __restrict__ root, uint32_t* __restrict__ status,
       const uint32_t* __restrict__ abort_flag)
{
    const uint32_t x = blockIdx.x * BLK + threadIdx.x;
    if (x >= 2 * n - 1 || *abort_flag) { return; }
    const uint8_t fl = kflag[x];
    if (!(fl & KF_KEPT)) { return; }
    const bool is_m = (fl & KF_MSPLIT) != 0;
    uint32_t f, l;
    krange<K>(knode, n, x, f, l);
    const uint32_t pre = snode[f] + rank[x];
    if (info)
    {
        const uint64_t sf = (uint64_t)keys[f] >> sshift, sl = (uint64_t)keys[l] >> sshift;
        if (sf == sl && (f == 0 || ((uint64_t)keys[f - 1] >> sshift) != sf) &&
            (l == n - 1 || ((uint64_t)keys[l + 1] >> sshift) != sl))
        {
            uint32_t* o = info + 4 * (size_t)sf;
            const uint32_t tf = stri ? stri[f] : f, tl = stri ? stri[l + 1] : l + 1u;
            o[0] = pre; o[1] = snode[l + 1] - pre; o[2] = tf; o[3] = tl - tf;
        }
    }
    if (!is_m && l - f + 1u > max_leaf) { return; }  // SAH subtree root: emitted by the SAH builder
    if (pre >= max_nodes) { atomicOr(status, ST_CAPACITY); return; }
    const box3 b = load_box(kbox, x);
    if (is_m)
    {
        const uint32_t r = knode[x].w;
        uint32_t rf, rl;
        krange<K>(knode, n, r, rf, rl);
        write_node(out, pre, b, 0, pre + 1u, snode[rf]);
    }
    else
    {
        write_node(out, pre, b, 1, stri ? stri[f] : f, l - f + 1u);
    }
    if (gn)
    {
        // the traversal layout (a tree without SAH subtrees): this node's box, reference and
        // count in its parent's 64-byte record -- the left child's half is floats 0-5 and words
        // 12 / 14, the right child's floats 6-11 and words 13 / 15 -- or the entry record (the root)
        const uint32_t ref = is_m ? pre : (stri ? stri[f] : f);
        const uint32_t cnt = is_m ? 0u : (LEAF_BIT | (l - f + 1u));
        const uint32_t par = parent[x];
        if (par == NONE)
        {
            TraceRoot r;
            for (int k = 0; k < 3; k++) { r.box[k] = b.mn[k]; r.box[3 + k] = b.mx[k]; }
            r.ref = is_m ? 0u : ref;
            r.cnt = cnt;
            *root = r;
            return;
        }
        const uint4 pk = knode[par];
        const bool left = pk.z == x;
        // a left child follows its parent in pre-order; a right child's parent is found by its own slot
        const uint32_t ppre = left ? pre - 1u : snode[pk.x] + rank[par];
        float* g = gn + 16 * (size_t)ppre;
        uint32_t* gu = reinterpret_cast<uint32_t*>(g);
        if (left)
        {
            g[0] = b.mn[0]; g[1] = b.mn[1]; g[2] = b.mn[2]; g[3] = b.mx[0]; g[4] = b.mx[1]; g[5] = b.mx[2];
            gu[12] = ref; gu[14] = cnt;
        }
        else
        {
            g[6] = b.mn[0]; g[7] = b.mn[1]; g[8] = b.mn[2]; g[9] = b.mx[0]; g[10] = b.mx[1]; g[11] = b.mx[2];
            gu[13] = ref; gu[15] = cnt;
        }
    }
}

// Triangles of the Morton leaves, in sorted order at their output offsets.
__global__ void __launch_bounds__(BLK)
k_emit_tris(const uint32_t* __restrict__ perm, const uint8_t* __restrict__ kpos, const uint32_t* __restrict__ stri,
            uint32_t n, const rt_triangle* __restrict__ tris, rt_triangle* __restrict__ out, uint32_t* __restrict__ prim,
            uint32_t max_tris, const rt_vertex* __restrict__ verts, float4* __restrict__ tp, uint32_t* __restrict__ status)
{
    const uint32_t k = blockIdx.x * BLK + threadIdx.x;
    if (k >= n || !kpos[k]) { return; }
    const uint32_t t = perm[k], at = stri[k];
    if (at >= max_tris) { atomicOr(status, ST_CAPACITY); return; }
    const rt_triangle tr = tris[t];
    out[at] = tr;
    prim[at] = t;
    if (tp)  // the traversal layout's position record of the baked triangle (k_make_tripos)
    {
        const rt_vertex& a = verts[tr.v[0]];
        const rt_vertex& b = verts[tr.v[1]];
        const rt_vertex& c = verts[tr.v[2]];
        tp[3 * at + 0] = make_float4(a.x, a.y, a.z, b.x);
        tp[3 * at + 1] = make_float4(b.y, b.z, c.x, c.y);
        tp[3 * at + 2] = make_float4(c.z, 0.f, 0.f, 0.f);
    }
}

// ---- device-wide exclusive scan (reduce, scan of partials, apply) ----
constexpr int SCAN_TILE = 2048;  // 256 threads x 8

__global__ void __launch_bounds__(256) k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ part)
{
    __shared__ uint32_t sh[9];
    const uint32_t base = blockIdx.x * SCAN_TILE;
    uint32_t s = 0;
    for (int j = 0; j < 8; j++)
    {
        const uint32_t i = base + j * 256 + threadIdx.x;
        if (i < n) { s += in[i]; }
    }
    const uint32_t t = block_sum<256>(s, sh);
    if (threadIdx.x == 0) { part[blockIdx.x] = t; }
}

__global__ void __launch_bounds__(1024) k_scan_partials(uint32_t* __restrict__ part, uint32_t np, uint32_t* __restrict__ total)
{
    __shared__ uint32_t sh[33];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < np; base += 1024)
    {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < np ? part[i] : 0u;
        uint32_t tot;
        const uint32_t e = block_excl_scan<1024>(v, sh, &tot);
        if (i < np) { part[i] = carry + e; }
        carry += tot;
    }
    if (threadIdx.x == 0 && total) { *total = carry; }
}

__global__ void __launch_bounds__(256)
k_scan_apply(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* __restrict__ part, uint32_t* __restrict__ out)
{
    __shared__ uint32_t sh[9];
    const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * 8;
    uint32_t v[8];
    uint32_t s = 0;
    for (int j = 0; j < 8; j++)
    {
        const uint32_t i = base + j;
        v[j] = i < n ? in[i] : 0u;
        s += v[j];
    }
    uint32_t run = part[blockIdx.x] + block_excl_scan<256>(s, sh, nullptr);
    for (int j = 0; j < 8; j++)
    {
        const uint32_t i = base + j;
        if (i < n) { out[i] = run; }
        run += v[j];
    }
}

// Exclusive scans of two arrays at once (the pre-order slot and triangle-offset weights).
struct Scan2
{
    const uint32_t* in[2];
    uint32_t*       out[2];
    uint32_t*       total[2];
};

// Both scans in one pass with decoupled look-back (Merrill and Garland, "Single-pass Parallel
// Prefix Scan with Decoupled Look-back", 2016): blocks take tiles of SCAN_TILE elements in the
// order they start (a ticket), publish each array's tile sum, then sum their predecessors'
// published values back to the nearest inclusive prefix and publish their own. A descriptor is
// one 64-bit word: flag in bits 62-63 (1 sum, 2 inclusive prefix), value in the low 32 bits.
// desc (2 per tile) and the ticket after them start zeroed. Waits are bounded (ST_TIMEOUT).
constexpr unsigned long long SC_AGG = 1ull << 62, SC_PRE = 2ull << 62, SC_FLAGS = 3ull << 62;
constexpr uint32_t SC_SPIN_LIMIT = 1u << 22;
// Large tiles: with every tile resident at once, a tile's look-back mostly finds sums, not
// prefixes, so its walk is as long as the number of tiles before it (in windows of 32).
constexpr int SC1_THREADS = 512, SC1_ITEMS = 16, SC1_TILE = SC1_THREADS * SC1_ITEMS;

// NA = 1: the first array only; the second is then the identity (every key places one
// triangle: a tree without SAH subtrees), whose total n - 1 the last tile writes.
template <int NA>
__global__ void __launch_bounds__(SC1_THREADS)
k_scan2_onepass(Scan2 S, uint32_t n, unsigned long long* __restrict__ desc, uint32_t* __restrict__ ticket,
                uint32_t* __restrict__ status, const uint32_t* __restrict__ abort_flag)
{
    __shared__ uint32_t sh[SC1_THREADS / 32 + 1];
    __shared__ uint32_t s_tile, s_prev[2];
    if (*abort_flag) { return; }  // (uniform over the grid)
    if (threadIdx.x == 0) { s_tile = atomicAdd(ticket, 1u); }
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * SC1_TILE + threadIdx.x * SC1_ITEMS;
    uint32_t v[2][SC1_ITEMS], excl[2], tot[2];
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        uint32_t sum = 0;
        if (base + SC1_ITEMS <= n)
        {
            const uint4* q = reinterpret_cast<const uint4*>(S.in[a] + base);
#pragma unroll
            for (int j = 0; j < SC1_ITEMS / 4; j++)
            {
                const uint4 w = q[j];
                v[a][4 * j] = w.x; v[a][4 * j + 1] = w.y; v[a][4 * j + 2] = w.z; v[a][4 * j + 3] = w.w;
            }
        }
        else
        {
#pragma unroll
            for (int j = 0; j < SC1_ITEMS; j++) { v[a][j] = base + j < n ? S.in[a][base + j] : 0u; }
        }
#pragma unroll
        for (int j = 0; j < SC1_ITEMS; j++) { sum += v[a][j]; }
        excl[a] = block_excl_scan<SC1_THREADS>(sum, sh, &tot[a]);
    }
    // warp a (0, 1) publishes and looks back for array a, 32 predecessors at a time
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < NA)
    {
        const int a = warp;
        if (lane == 0)
        {
            cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> mine(desc[2 * (size_t)tile + a]);
            mine.store((tile == 0 ? SC_PRE : SC_AGG) | tot[a], cuda::memory_order_relaxed);
        }
        uint32_t prev = 0;
        int64_t top = (int64_t)tile - 1;  // the window is tiles top - 31 .. top
        while (top >= 0)
        {
            const int64_t p = top - lane;
            unsigned long long w = SC_PRE;  // below tile 0: nothing to add
            if (p >= 0)
            {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> d(desc[2 * (size_t)p + a]);
                w = d.load(cuda::memory_order_relaxed);
                for (uint32_t spin = 0; (w & SC_FLAGS) == 0; spin++)
                {
                    if (spin > SC_SPIN_LIMIT) { atomicOr(status, ST_TIMEOUT); w = SC_PRE; break; }
                    w = d.load(cuda::memory_order_relaxed);
                }
            }
            // the nearest inclusive prefix in the window ends the walk: lanes up to it add in
            const unsigned pre = __ballot_sync(0xffffffffu, (w & SC_FLAGS) == SC_PRE);
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
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> mine(desc[2 * (size_t)tile + a]);
                mine.store(SC_PRE | (uint32_t)(prev + tot[a]), cuda::memory_order_relaxed);
            }
            s_prev[a] = prev;
            if (tile == gridDim.x - 1)
            {
                *S.total[a] = prev + tot[a];
                if (NA == 1) { *S.total[1] = n - 1u; }
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        uint32_t run = s_prev[a] + excl[a];
#pragma unroll
        for (int j = 0; j < SC1_ITEMS; j++)
        {
            const uint32_t i = base + j;
            if (i < n) { S.out[a][i] = run; }
            run += v[a][j];
        }
    }
}


// All per-build initialisation in one launch: block 0 also does k_init's work.
__global__ void __launch_bounds__(BLK)
k_clear(uint32_t n, uint32_t* __restrict__ parent, uint8_t* __restrict__ kflag, uint32_t* __restrict__ wnode,
        uint32_t* __restrict__ wtri, uint8_t* __restrict__ kpos, uint32_t* __restrict__ scene, uint32_t n_scene_boxes,
        uint32_t* __restrict__ hist, uint32_t* __restrict__ counters, uint32_t* __restrict__ status,
        uint32_t* __restrict__ lookback, uint32_t n_lookback, uint32_t* __restrict__ tile_counters)
{
    const uint32_t i = blockIdx.x * BLK + threadIdx.x;
    if (i < n_lookback) { lookback[i] = 0u; }  // the radix sort's look-back words (all its passes)
    if (i < 64) { tile_counters[i] = 0u; }
    if (i == 0) { parent[0] = NONE; }  // the root (inner node 0, or the single leaf); k_karras sets the rest
    if (i == 0 && n == 1) { kflag[0] = KF_KEPT; }  // a single triangle: the root leaf (no k_karras)
    // every key starts in a Morton leaf (k_boundary clears the keys of SAH subtree roots)
    if (i < n) { kpos[i] = 1u; }
    if (i <= n) { wnode[i] = 0u; wtri[i] = i < n ? 1u : 0u; }
    if (i < 6 * n_scene_boxes) { scene[i] = (i % 6) < 3 ? 0xffffffffu : 0u; }
    if (blockIdx.x == 0)
    {
        const int t = threadIdx.x;
        for (int k = t; k < 9 * 256; k += BLK) { hist[k] = 0u; }
        if (t < 16) { counters[t] = 0u; }
        if (t == 0) { *status = 0u; }
    }
}

template <typename K>
int build_typed(rt_bvh* B, const rt_vertex* d_verts, uint32_t V, const rt_triangle* d_tris, uint32_t N,
                const rt_build_cfg& cfg, cudaStream_t st, uint32_t cap, const Batch& bt)
{
    BuildScratch& S = B->s;
    const bool batch = bt.S > 0;
    const uint32_t n_boxes = batch ? bt.S : 1u;
    const int key_bits = batch ? (int)bt.sshift + (int)scene_bits(bt.S) : 3 * (int)cfg.morton_bits;
    const uint32_t sshift = batch ? bt.sshift : 63u;
    const int passes = sort_passes(key_bits);
    const int msd_shift = key_bits > 8 ? key_bits - 8 : -1;  // top digit, for the sort's MSD path
    const uint32_t nk = 2 * N - 1;  // Karras nodes
    // the box hierarchy: pre / suf of levels 0 .. top - 1, blk of levels 1 .. top
    const int lv_top_level = lv_top(N);
    const uint64_t n_ps = lv_off(N, lv_top_level, 0), n_blk = lv_off(N, lv_top_level + 1, 1);
    if (S.tri_lo.ensure((size_t)N * 16) || S.tri_hi.ensure((size_t)N * 16) || S.tri_cz.ensure((size_t)N * 4) ||
        S.tpin.ensure((size_t)N * 48) ||
        S.keys.ensure((size_t)N * sizeof(K)) || S.vals.ensure((size_t)N * 4) || S.hist.ensure(9 * 256 * 4) ||
        S.scene.ensure((size_t)n_boxes * 24 + 64) || S.status.ensure(64) || S.counters.ensure(64) ||
        (batch && (S.gtris.ensure((size_t)N * sizeof(rt_triangle)) || B->scene_info.ensure((size_t)bt.S * 16) ||
                   B->scene_roots.ensure((size_t)bt.S * 32))) ||
        S.knode.ensure((size_t)std::max<uint32_t>(N - 1, 1) * 16) || S.parent.ensure((size_t)nk * 4) ||
        S.kbox.ensure((size_t)nk * 32) || S.lvbox.ensure((size_t)(2 * n_ps + n_blk) * 32 + 32) ||
        S.kflag.ensure((size_t)nk + 16) || S.ktab.ensure(((size_t)1 << 16) * 4 + 16) || S.rank.ensure((size_t)nk * 4) ||
        S.wnode.ensure((size_t)(N + 1) * 4) || S.wtri.ensure((size_t)(N + 1) * 4) ||
        S.snode.ensure((size_t)(N + 1) * 4) || S.stri.ensure((size_t)(N + 1) * 4) || S.bnd.ensure((size_t)N) ||
        S.sah_roots.ensure((size_t)N * sizeof(SahRoot)))
    {
        return RT_E_CUDA;
    }
    uint32_t* counters = S.counters.as<uint32_t>();
    uint32_t* status = counters + 15;  // read back with the counters in one copy
    BoxLevels bl;
    bl.pre = S.lvbox.as<float4>();
    bl.suf = bl.pre + 2 * n_ps;
    bl.blk = bl.suf + 2 * n_ps;
    bl.n = N;
    bl.top = lv_top_level;
    // the sort's scratch, zeroed by k_clear below (radix_sort_pairs then skips its memsets)
    const size_t n_lookback = sort_lookback_words(N, passes);
    if (S.sort.lookback.ensure(n_lookback * 4) || S.sort.tile_counters.ensure((64 + 260) * 4)) { return RT_E_CUDA; }

    K* skeys = nullptr;
    uint32_t* perm = nullptr;
    const uint32_t tm = std::max(cfg.max_leaf, cfg.lbvh_threshold);
    // a captured bake leaves the sort's LSD fallback out and reports in counters[14] whether it
    // was needed (a top-digit bucket over one block); such a bake is then done again plainly
    bool msd_only = false;
    // When the SAH threshold does not exceed the leaf size (the LBVH presets), subtrees for the
    // binned SAH only come from runs of identical Morton codes; the layout is emitted at once
    // and redone in the rare case such runs exist, which saves a host round trip.
    const bool expect_sah = cfg.lbvh_threshold > cfg.max_leaf;
    bool tris_fused = false;  // k_karras wrote the baked triangles (a build with no SAH subtree expected)
    // everything up to the boundary nodes, enqueued on st
    auto front = [&]() -> int {
        prof_mark(B, 0, st);
        k_clear<<<blocks_for(std::max<uint32_t>(std::max<uint32_t>(N + 1, 6 * n_boxes), (uint32_t)n_lookback)), BLK, 0, st>>>(
            N, S.parent.as<uint32_t>(), S.kflag.as<uint8_t>(), S.wnode.as<uint32_t>(), S.wtri.as<uint32_t>(),
            S.bnd.as<uint8_t>(), S.scene.as<uint32_t>(), n_boxes, S.hist.as<uint32_t>(), counters, status,
            S.sort.lookback.as<uint32_t>(), (uint32_t)n_lookback, S.sort.tile_counters.as<uint32_t>());
        count_launch();
        k_vertices<<<blocks_for(V), BLK, 0, st>>>(d_verts, B->verts.as<rt_vertex>(), V);
        count_launch();
        const uint32_t morton_blocks = std::min<uint32_t>(blocks_for(N), 4u * (uint32_t)device_sm_count());
        if (batch)
        {
            k_tri_prep<true><<<blocks_for(N), BLK, 0, st>>>(d_tris, N, d_verts, V, S.tri_lo.as<float4>(), S.tri_hi.as<float4>(),
                                                             S.tri_cz.as<float>(), S.scene.as<uint32_t>(), status, bt,
                                                             S.gtris.as<rt_triangle>(), S.tpin.as<float4>());
            d_tris = S.gtris.as<rt_triangle>();  // vertex indices of the concatenated array from here on
            k_morton<K, true><<<morton_blocks, BLK, 0, st>>>(S.tri_lo.as<float4>(), S.tri_hi.as<float4>(), S.tri_cz.as<float>(),
                                                             N, S.scene.as<uint32_t>(), cfg.morton_bits, passes,
                                                             S.keys.as<K>(), S.hist.as<uint32_t>(), msd_shift, bt);
        }
        else
        {
            k_tri_prep<false><<<blocks_for(N), BLK, 0, st>>>(d_tris, N, d_verts, V, S.tri_lo.as<float4>(), S.tri_hi.as<float4>(),
                                                              S.tri_cz.as<float>(), S.scene.as<uint32_t>(), status, bt,
                                                              nullptr, S.tpin.as<float4>());
            k_morton<K><<<morton_blocks, BLK, 0, st>>>(S.tri_lo.as<float4>(), S.tri_hi.as<float4>(), S.tri_cz.as<float>(), N,
                                                       S.scene.as<uint32_t>(), cfg.morton_bits, passes, S.keys.as<K>(),
                                                       S.hist.as<uint32_t>(), msd_shift);
        }
        count_launch(2);
        if (int e = check_launch("morton")) { return e; }

        prof_mark(B, 1, st);
        const uint32_t* table_flag = nullptr;
        if (int e = radix_sort_pairs<K>(S.keys.as<K>(), S.vals.as<uint32_t>(), true, N, key_bits, S.hist.as<uint32_t>(),
                                        msd_shift >= 0 ? S.hist.as<uint32_t>() + 8 * 256 : nullptr, S.sort, status, st,
                                        &skeys, &perm, true, msd_only ? counters + 14 : nullptr,
                                        N >= 2 && key_bits > 16 ? S.ktab.as<uint32_t>() : nullptr, &table_flag))
        {
            return e;
        }
        prof_mark(B, 2, st);
        if (N >= 2)
        {
            const int tb = std::min(16, key_bits);
            const uint32_t table_blocks = std::min<uint32_t>(blocks_for((uint64_t)N + 1), 4u * (uint32_t)device_sm_count());
            k_bucket_table<K><<<table_blocks, BLK, 0, st>>>(skeys, N, key_bits - tb, 1u << tb,
                                                                         S.ktab.as<uint32_t>(), counters + 14, table_flag);
            // without expected SAH subtrees the baked triangles are written here (in key order); a
            // bake that finds runs of equal codes after all writes them again in its second emit
            const bool fuse = !expect_sah;
            k_karras<K><<<blocks_for(N), BLK, 0, st>>>(skeys, perm, N, S.tri_lo.as<float4>(), S.tri_hi.as<float4>(),
                                                       S.knode.as<uint4>(), S.parent.as<uint32_t>(), S.kflag.as<uint8_t>(),
                                                       S.ktab.as<uint32_t>(), key_bits, tb, tm, sshift, bl, S.tpin.as<float4>(),
                                                       fuse ? B->tris.as<rt_triangle>() : nullptr, B->prim.as<uint32_t>(),
                                                       B->tripos.as<float4>(), status, counters + 14);
            tris_fused = fuse;
            count_launch();
            // counters[8]: the ticket that elects the last block to build the upper levels
            k_box_levels<<<blocks_for(lv_count(N, 2)), BLK, 0, st>>>(bl, counters + 8, counters + 14);
            count_launch(2);
        }
        k_boundary<K><<<blocks_for(nk), BLK, 0, st>>>(skeys, perm, N, S.knode.as<uint4>(), S.parent.as<uint32_t>(),
                                                      S.tri_lo.as<float4>(), S.tri_hi.as<float4>(), bl,
                                                      tm, cfg.max_leaf, sshift,
                                                      S.kbox.as<float4>(), S.rank.as<uint32_t>(),
                                                      S.wnode.as<uint32_t>(), S.wtri.as<uint32_t>(), S.bnd.as<uint8_t>(),
                                                      S.sah_roots.as<SahRoot>(), counters, S.kflag.as<uint8_t>(), status,
                                                      counters + 14);
        count_launch();
        if (int e = check_launch("boundary")) { return e; }
        prof_mark(B, 3, st);
        return RT_OK;
    };

    SahResult sah;
    uint32_t n_roots = 0;
    auto run_sah = [&]() -> int {
        SahInput in;
        in.verts = B->verts.as<rt_vertex>();
        in.tris = d_tris;
        in.lo = S.tri_lo.as<float4>();
        in.hi = S.tri_hi.as<float4>();
        in.cz = S.tri_cz.as<float>();
        in.perm = perm;
        in.n = N;
        in.cap = cap;
        in.roots = S.sah_roots.as<SahRoot>();
        in.n_roots = n_roots;
        in.wnode = S.wnode.as<uint32_t>();
        in.wtri = S.wtri.as<uint32_t>();
        in.kpos = S.bnd.as<uint8_t>();
        in.status = status;
        if (batch)
        {
            for (uint32_t k = 0; k < bt.S; k++)
            {
                const uint32_t ns = bt.h_toff[k + 1] - bt.h_toff[k];
                const uint32_t c = (uint32_t)((float)ns * cfg.spatial_mult);  // bvh_morton.cpp:46-47, per scene
                in.budget_used.push_back(ns);
                in.budget_cap.push_back(std::max(c, ns));
            }
        }
        else
        {
            in.budget_used.push_back(N);
            in.budget_cap.push_back(cap);
        }
        return sah_build(B, cfg, in, st, &sah);
    };
    // pre-order node slots and triangle offsets per start key, then the nodes and triangles
    auto emit_all = [&]() -> int {
        // without SAH subtrees every key places its own triangle at its own position, so the
        // triangle offsets are the identity and only the node slots are scanned
        const bool tri_identity = !expect_sah && n_roots == 0 && tris_fused;
        {
            const uint32_t n1 = N + 1, np = (n1 + SC1_TILE - 1) / SC1_TILE;
            // look-back descriptors (2 per tile) and the tile ticket, zeroed for every scan
            if (S.scan.partials.ensure(((size_t)2 * np + 1) * 8)) { return RT_E_CUDA; }
            unsigned long long* desc = S.scan.partials.as<unsigned long long>();
            RT_CUDA(cudaMemsetAsync(desc, 0, ((size_t)2 * np + 1) * 8, st));
            Scan2 sc;
            sc.in[0] = S.wnode.as<uint32_t>(); sc.out[0] = S.snode.as<uint32_t>(); sc.total[0] = counters + 4;
            sc.in[1] = S.wtri.as<uint32_t>(); sc.out[1] = S.stri.as<uint32_t>(); sc.total[1] = counters + 5;
            if (tri_identity)
            {
                k_scan2_onepass<1><<<np, SC1_THREADS, 0, st>>>(sc, n1, desc, reinterpret_cast<uint32_t*>(desc + 2 * (size_t)np),
                                                               status, counters + 14);
            }
            else
            {
                k_scan2_onepass<2><<<np, SC1_THREADS, 0, st>>>(sc, n1, desc, reinterpret_cast<uint32_t*>(desc + 2 * (size_t)np),
                                                               status, counters + 14);
            }
            count_launch();
        }
        k_emit<K><<<blocks_for(nk), BLK, 0, st>>>(skeys, N, S.knode.as<uint4>(), S.parent.as<uint32_t>(), tm, cfg.max_leaf,
                                                  sshift, S.kbox.as<float4>(), S.rank.as<uint32_t>(), S.snode.as<uint32_t>(),
                                                  tri_identity ? nullptr : S.stri.as<uint32_t>(), B->nodes.as<rt_bvh_node>(), 2 * cap - 1,
                                                  batch ? B->scene_info.as<uint32_t>() : nullptr, S.kflag.as<uint8_t>(),
                                                  n_roots == 0 ? B->gnodes.as<float>() : nullptr,
                                                  B->rootbuf.as<TraceRoot>(), status, counters + 14);
        count_launch();
        // without SAH subtrees every triangle passes here: its traversal record is written too
        // (input positions: the renormalisation changes only normals); k_karras wrote them already
        // when no SAH subtree was expected and none came
        if (!(tris_fused && n_roots == 0))
        {
            k_emit_tris<<<blocks_for(N), BLK, 0, st>>>(perm, S.bnd.as<uint8_t>(), S.stri.as<uint32_t>(), N, d_tris,
                                                        B->tris.as<rt_triangle>(), B->prim.as<uint32_t>(), cap, d_verts,
                                                        n_roots == 0 ? B->tripos.as<float4>() : nullptr, status);
            count_launch();
        }
        if (n_roots > 0)
        {
            if (int e = sah_emit(B, n_roots, S.snode.as<uint32_t>(), S.stri.as<uint32_t>(), d_tris, st, sah, 2 * cap - 1,
                                 cap, status))
            {
                return e;
            }
        }
        return check_launch("emit");
    };

    // emit and traversal layout, after the SAH subtrees if any
    auto tail = [&]() -> int {
        prof_mark(B, 4, st);
        if (int e = emit_all()) { return e; }
        prof_mark(B, 5, st);
        // traversal layout from the device-side counts: the build's only host round trip follows
        // without SAH subtrees k_emit wrote the traversal nodes and k_karras / k_emit_tris the
        // triangle records
        if (int e = launch_traversal_layout(B, st, 2 * cap - 1, cap, counters + 4, status, n_roots == 0, n_roots == 0))
        {
            return e;
        }
        if (batch)
        {
            if (int e = launch_scene_roots(B, bt.S, counters + 4, status, st)) { return e; }
            B->scene_info_host.resize((size_t)4 * bt.S);
            RT_CUDA(cudaMemcpyAsync(B->scene_info_host.data(), B->scene_info.p, (size_t)bt.S * 16, cudaMemcpyDeviceToHost, st));
        }
        prof_mark(B, 6, st);
        return RT_OK;
    };
    // An LBVH bake (no SAH subtrees expected, one scene, no stage events) replays its launch
    // sequence from a CUDA graph: captured on the second call with the same key -- sizes,
    // settings, inputs and the address of every buffer the launches use, as the previous plain
    // bake left them -- and replayed on the handle's own stream between two events on the
    // caller's. The host work between the launches, and the launches themselves, then cost one
    // graph launch.
    const bool graph_path = !batch && !B->prof && !expect_sah;
    auto bake_key = [&]() {
        const void* bufs[] = { S.tri_lo.p, S.tri_hi.p, S.tri_cz.p, S.keys.p, S.vals.p, S.hist.p, S.scene.p, S.counters.p,
                               S.knode.p, S.parent.p, S.kbox.p, S.lvbox.p, S.kflag.p, S.ktab.p, S.tpin.p, S.rank.p, S.wnode.p, S.wtri.p, S.snode.p,
                               S.stri.p, S.bnd.p, S.sah_roots.p, S.sort.keys_alt.p, S.sort.vals_alt.p, S.sort.lookback.p,
                               S.sort.tile_counters.p, S.scan.partials.p, B->nodes.p, B->tris.p, B->prim.p, B->verts.p,
                               B->gnodes.p, B->tripos.p, B->rootbuf.p, d_verts, d_tris };
        const uint64_t kv[2] = { ((uint64_t)N << 32) | V, sizeof(K) };
        std::vector<unsigned char> key(sizeof(rt_build_cfg) + sizeof(kv) + sizeof(bufs));
        std::memcpy(key.data(), &cfg, sizeof(rt_build_cfg));
        std::memcpy(key.data() + sizeof(rt_build_cfg), kv, sizeof(kv));
        std::memcpy(key.data() + sizeof(rt_build_cfg) + sizeof(kv), bufs, sizeof(bufs));
        return key;
    };
    bool enq0 = false;  // attempt 0's launches are in flight already
    if (graph_path)
    {
        const std::vector<unsigned char> key = bake_key();
        const bool replay = B->bake_exec && key == B->bake_key;
        if (replay || key == B->bake_seen)
        {
            if (!B->bake_stream)
            {
                RT_CUDA(cudaStreamCreateWithFlags(&B->bake_stream, cudaStreamNonBlocking));
                for (cudaEvent_t& e : B->bake_ev) { RT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)); }
            }
            const cudaStream_t caller = st;
            RT_CUDA(cudaEventRecord(B->bake_ev[0], caller));
            RT_CUDA(cudaStreamWaitEvent(B->bake_stream, B->bake_ev[0], 0));
            if (!replay)
            {
                if (B->bake_exec) { cudaGraphExecDestroy(B->bake_exec); B->bake_exec = nullptr; }
                st = B->bake_stream;  // the lambdas enqueue on st
                RT_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                const uint64_t l0 = thread_launches();
                msd_only = true;
                int e = front();
                if (!e) { e = tail(); }
                msd_only = false;
                cudaGraph_t g = nullptr;
                const cudaError_t ce = cudaStreamEndCapture(st, &g);
                st = caller;
                if (!e && ce != cudaSuccess) { e = fail(RT_E_CUDA, std::string("bake capture: ") + cudaGetErrorString(ce)); }
                if (!e && cudaGraphInstantiate(&B->bake_exec, g, 0) != cudaSuccess)
                {
                    B->bake_exec = nullptr;
                    e = fail(RT_E_CUDA, "bake graph instantiation");
                }
                if (g) { cudaGraphDestroy(g); }
                if (e) { return e; }
                B->bake_kernels = thread_launches() - l0;
                B->bake_key = key;
                B->bake_skeys = skeys;
                B->bake_perm = perm;
            }
            else
            {
                skeys = static_cast<K*>(B->bake_skeys);
                perm = B->bake_perm;
                count_launch(B->bake_kernels);
            }
            RT_CUDA(cudaGraphLaunch(B->bake_exec, B->bake_stream));
            RT_CUDA(cudaEventRecord(B->bake_ev[1], B->bake_stream));
            RT_CUDA(cudaStreamWaitEvent(caller, B->bake_ev[1], 0));
            enq0 = true;
        }
    }
    if (!enq0)
    {
        if (int e = front()) { return e; }
    }
    if (batch) { RT_CUDA(cudaMemsetAsync(B->scene_info.p, 0xff, (size_t)bt.S * 16, st)); }
    uint32_t res[16];  // counters[0..15]; [15] is the status word
    uint32_t stat = 0;
    for (int attempt = 0; attempt < 2; attempt++)
    {
        if (expect_sah || attempt == 1)
        {
            if (attempt == 0)
            {
                RT_CUDA(cudaMemcpyAsync(res, counters, 8, cudaMemcpyDeviceToHost, st));
                RT_CUDA(cudaStreamSynchronize(st));
                n_roots = res[0];
            }
            if (n_roots > 0)
            {
                if (int e = run_sah()) { return e; }
            }
        }
        if (!(attempt == 0 && enq0))
        {
            if (int e = tail()) { return e; }
        }
        RT_CUDA(cudaMemcpyAsync(res, counters, 64, cudaMemcpyDeviceToHost, st));
        RT_CUDA(cudaStreamSynchronize(st));
        if (attempt == 0 && enq0 && res[14] != 0u)
        {
            // the replayed launches have no LSD fallback and a bucket overflowed: bake plainly
            enq0 = false;
            if (int e = front()) { return e; }
            if (int e = tail()) { return e; }
            RT_CUDA(cudaMemcpyAsync(res, counters, 64, cudaMemcpyDeviceToHost, st));
            RT_CUDA(cudaStreamSynchronize(st));
        }
        stat = res[15];
        if (graph_path && attempt == 0 && !enq0) { B->bake_seen = bake_key(); }  // with this bake's buffers
        if (expect_sah || res[0] == 0) { break; }
        n_roots = res[0];  // identical-code runs found: build their SAH subtrees and emit again
    }
    B->stats[0] = sah.spatial_taken;
    B->stats[1] = sah.spatial_refused;
    B->stats[2] = n_roots;
    if (stat & ST_INDEX) { return fail(RT_E_INDEX, "triangle has an out-of-bounds vertex index"); }
    if (stat & ST_TIMEOUT) { return fail(RT_E_TIMEOUT, "a bounded device wait gave up (radix sort look-back)"); }
    if (stat & ST_CAPACITY) { return fail(RT_E_CAPACITY, "internal capacity exceeded during the build"); }
    if (res[4] > 2 * cap - 1 || res[5] > cap) { return fail(RT_E_CAPACITY, "build produced more nodes than its bound"); }
    B->n_nodes = res[4];
    B->n_tris = res[5];
    B->n_scenes = bt.S;
    for (uint32_t k = 0; k < bt.S; k++)
    {
        const uint32_t* in = &B->scene_info_host[4 * (size_t)k];
        if (in[0] >= B->n_nodes || (uint64_t)in[0] + in[1] > B->n_nodes || (uint64_t)in[2] + in[3] > B->n_tris)
        {
            return fail(RT_E_CAPACITY, "batched build: a scene's root record is out of range");
        }
    }
    B->stats[4] = (B->n_nodes + 1u) / 2u;  // a full binary tree: one leaf more than inner nodes
    B->stats[3] = B->n_nodes - B->stats[4];
    B->trace_ww = prefer_while_while(B->n_tris, B->stats[4]);
    return RT_OK;
}

} // namespace

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* d_total, ScanScratch& s, cudaStream_t st)
{
    const uint32_t np = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (s.partials.ensure((size_t)std::max<uint32_t>(np, 1) * 4)) { return RT_E_CUDA; }
    k_scan_reduce<<<np, 256, 0, st>>>(in, n, s.partials.as<uint32_t>());
    k_scan_partials<<<1, 1024, 0, st>>>(s.partials.as<uint32_t>(), np, d_total);
    k_scan_apply<<<np, 256, 0, st>>>(in, n, s.partials.as<uint32_t>(), out);
    count_launch(3);
    return check_launch("scan");
}

int build_bvh(rt_bvh* B, const rt_vertex* d_verts, uint32_t V, const rt_triangle* d_tris, uint32_t N,
              const rt_build_cfg& cfg, cudaStream_t st)
{
    return build_bvh_batch(B, d_verts, V, d_tris, N, cfg, st, 0, nullptr, nullptr, nullptr);
}

int build_bvh_batch(rt_bvh* B, const rt_vertex* d_verts, uint32_t V, const rt_triangle* d_tris, uint32_t N,
                    const rt_build_cfg& cfg, cudaStream_t st, uint32_t n_scenes, const uint32_t* d_toff,
                    const uint32_t* d_voff, const uint32_t* h_toff)
{
    if (V == 0 || N == 0) { return fail(RT_E_EMPTY, "no vertices or no triangles"); }
    if (cfg.morton_bits < 1 || cfg.morton_bits > 21) { return fail(RT_E_INVALID, "morton_bits must be in 1..21"); }
    if (cfg.bins_min < 1 || cfg.bins_max > SAH_MAX_BINS || cfg.bins_min > cfg.bins_max)
    {
        return fail(RT_E_INVALID, "bins must satisfy 1 <= bins_min <= bins_max <= 32");
    }
    if (cfg.max_leaf < 1) { return fail(RT_E_INVALID, "max_leaf must be >= 1"); }
    if (N > (1u << 29)) { return fail(RT_E_CAPACITY, "more than 2^29 triangles"); }
    uint32_t cap = (uint32_t)((float)N * cfg.spatial_mult);  // bvh_morton.cpp:46-47
    if (cap < N) { cap = N; }
    const size_t max_nodes = (size_t)cap * 2 - 1;  // bvh_bfs.cpp:58
    if (B->tripos.ensure((size_t)cap * 48) ||  // written by k_emit_tris in builds without SAH subtrees
        B->gnodes.ensure(max_nodes * sizeof(rt_gnode)) || B->rootbuf.ensure(sizeof(TraceRoot)) ||  // and by k_emit
        B->nodes.ensure(max_nodes * sizeof(rt_bvh_node)) || B->tris.ensure((size_t)cap * sizeof(rt_triangle)) ||
        B->prim.ensure((size_t)cap * 4) || B->verts.ensure((size_t)V * sizeof(rt_vertex)))
    {
        return RT_E_CUDA;
    }
    B->n_verts = V;
    B->has_prim = true;
    B->n_scenes = 0;
    Batch bt{ n_scenes, d_toff, d_voff, 3 * cfg.morton_bits, h_toff };
    if (n_scenes > MAX_BATCH_SCENES) { return fail(RT_E_CAPACITY, "more than 1024 scenes in one batched build"); }
    const uint32_t key_bits = 3 * cfg.morton_bits + (n_scenes ? scene_bits(n_scenes) : 0u);
    if (key_bits > 64)
    {
        return fail(RT_E_INVALID, "batched build: 3 * morton_bits + ceil(log2(n_scenes)) must not exceed 64 "
                                  "(use 30-bit codes, morton_bits = 10, for more than 2 scenes)");
    }
    int e = (key_bits > 32) ? build_typed<uint64_t>(B, d_verts, V, d_tris, N, cfg, st, cap, bt)
                            : build_typed<uint32_t>(B, d_verts, V, d_tris, N, cfg, st, cap, bt);
    if (e) { return e; }
    if (B->prof)
    {
        RT_CUDA(cudaEventSynchronize(B->ev[6]));
        for (int i = 0; i < 6; i++) { cudaEventElapsedTime(&B->stage_ms[i], B->ev[i], B->ev[i + 1]); }
        cudaEventElapsedTime(&B->stage_ms[6], B->ev[0], B->ev[6]);
    }
    return RT_OK;
}

} // namespace rtb

// ---------------------------------------------------------------------------------------------
// Allocation-free Morton order (rt_morton_order_noalloc). Its scratch is one file-scope device
// array, shared by every call on a device and kept from call to call; each call clears what
// must start at zero. Host code reaches the array only through the device address that
// cudaGetSymbolAddress returns (the symbol itself is a host-side stand-in).
namespace
{

constexpr uint32_t NA_MAX_TRIS = RT_NOALLOC_MAX_TRIS;
constexpr uint32_t NA_TILES = (NA_MAX_TRIS + rtb::RS_SMALL_TILE_KEYS - 1) / rtb::RS_SMALL_TILE_KEYS;  // onesweep tiles
constexpr size_t NA_OFF_LO = 0;
constexpr size_t NA_OFF_HI = NA_OFF_LO + 16ull * NA_MAX_TRIS;
constexpr size_t NA_OFF_CZ = NA_OFF_HI + 16ull * NA_MAX_TRIS;
constexpr size_t NA_OFF_KEYS = NA_OFF_CZ + 4ull * NA_MAX_TRIS;
constexpr size_t NA_OFF_KALT = NA_OFF_KEYS + 8ull * NA_MAX_TRIS;
constexpr size_t NA_OFF_VALT = NA_OFF_KALT + 8ull * NA_MAX_TRIS;
constexpr size_t NA_OFF_HIST = NA_OFF_VALT + 4ull * NA_MAX_TRIS;
constexpr size_t NA_OFF_LB = NA_OFF_HIST + 8ull * 256 * 4;
constexpr size_t NA_OFF_TILE = NA_OFF_LB + 8ull * NA_TILES * 256 * 4;
constexpr size_t NA_OFF_SMALL = NA_OFF_TILE + 64 * 4;  // scene box, counters, status
constexpr size_t NA_BYTES = NA_OFF_SMALL + 256;
static_assert(NA_MAX_TRIS <= rtb::RS_SMALL_MAX_KEYS, "the fixed-scratch sort takes at most RS_SMALL_MAX_KEYS keys");
static_assert(NA_OFF_TILE - NA_OFF_LB >= 4 * rtb::sort_raw_lookback_words(NA_MAX_TRIS, 8),
              "look-back region too small for the sort's tiles");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

std::mutex g_na_mu;
unsigned char* g_na_dev[64];  // device address of g_noalloc_scratch, per device

template <typename K>
int morton_order_noalloc_typed(unsigned char* base, const rt_vertex* verts, uint32_t V, const rt_triangle* tris,
                               uint32_t N, uint32_t bits, uint32_t* perm_out, cudaStream_t st)
{
    using namespace rtb;
    float4* lo = reinterpret_cast<float4*>(base + NA_OFF_LO);
    float4* hi = reinterpret_cast<float4*>(base + NA_OFF_HI);
    float* cz = reinterpret_cast<float*>(base + NA_OFF_CZ);
    K* keys = reinterpret_cast<K*>(base + NA_OFF_KEYS);
    K* kalt = reinterpret_cast<K*>(base + NA_OFF_KALT);
    uint32_t* valt = reinterpret_cast<uint32_t*>(base + NA_OFF_VALT);
    uint32_t* hist = reinterpret_cast<uint32_t*>(base + NA_OFF_HIST);
    uint32_t* lookback = reinterpret_cast<uint32_t*>(base + NA_OFF_LB);
    uint32_t* tiles = reinterpret_cast<uint32_t*>(base + NA_OFF_TILE);
    uint32_t* scene = reinterpret_cast<uint32_t*>(base + NA_OFF_SMALL);
    uint32_t* counters = scene + 16;
    uint32_t* status = scene + 48;
    const int key_bits = 3 * (int)bits;
    k_init<<<1, 256, 0, st>>>(scene, hist, counters, status);
    k_tri_prep<false><<<blocks_for(N), BLK, 0, st>>>(tris, N, verts, V, lo, hi, cz, scene, status,
                                                      Batch{ 0u, nullptr, nullptr, 63u, nullptr }, nullptr, nullptr);
    k_morton<K><<<blocks_for(N), BLK, 0, st>>>(lo, hi, cz, N, scene, bits, sort_passes(key_bits), keys, hist);
    count_launch(3);
    if (int e = check_launch("morton (no-alloc)")) { return e; }
    K* kout = nullptr;
    uint32_t* vout = nullptr;
    if (int e = radix_sort_pairs_raw<K>(keys, perm_out, N, key_bits, hist, kalt, valt, lookback, tiles, status, st, &kout,
                                        &vout))
    {
        return e;
    }
    if (vout != perm_out)
    {
        RT_CUDA(cudaMemcpyAsync(perm_out, vout, (size_t)N * 4, cudaMemcpyDeviceToDevice, st));
    }
    uint32_t stat = 0;
    RT_CUDA(cudaMemcpyAsync(&stat, status, 4, cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    if (stat & ST_INDEX) { return fail(RT_E_INDEX, "triangle has an out-of-bounds vertex index"); }
    if (stat & ST_TIMEOUT) { return fail(RT_E_TIMEOUT, "a bounded device wait gave up (radix sort look-back)"); }
    if (stat & ST_CAPACITY) { return fail(RT_E_CAPACITY, "internal capacity exceeded in the sort"); }
    return RT_OK;
}

} // namespace

extern "C" int rt_morton_order_noalloc(const rt_vertex* verts, uint32_t n_verts, const rt_triangle* tris, uint32_t n_tris,
                                       uint32_t morton_bits, uint32_t* perm_out, void* stream)
{
    using namespace rtb;
    if (!verts || !tris || !perm_out) { return fail(RT_E_INVALID, "null pointer"); }
    if (n_verts == 0 || n_tris == 0) { return fail(RT_E_EMPTY, "no vertices or no triangles"); }
    if (n_tris > NA_MAX_TRIS)
    {
        return fail(RT_E_CAPACITY, "rt_morton_order_noalloc takes at most " + std::to_string(NA_MAX_TRIS) +
                                       " triangles (its fixed scratch); use rt_build for larger meshes");
    }
    if (morton_bits < 1 || morton_bits > 21) { return fail(RT_E_INVALID, "morton_bits must be in 1..21"); }
    int dev = 0;
    RT_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { return fail(RT_E_INVALID, "device index out of range"); }
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!g_na_dev[dev])
        {
            void* p = nullptr;
            RT_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_na_dev[dev] = static_cast<unsigned char*>(p);
        }
        base = g_na_dev[dev];
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : default_stream();
    return (3 * morton_bits > 32) ? morton_order_noalloc_typed<uint64_t>(base, verts, n_verts, tris, n_tris, morton_bits,
                                                                         perm_out, st)
                                  : morton_order_noalloc_typed<uint32_t>(base, verts, n_verts, tris, n_tris, morton_bits,
                                                                         perm_out, st);
}
