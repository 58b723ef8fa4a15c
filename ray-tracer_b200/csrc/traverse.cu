// traverse.cu -- closest-hit / any-hit ray traversal: bvh::trace (src/bvh/bvh_traverse.cpp:91-246)
// for batches of rays on the GPU.
//
// Layout: the .bvh node array is re-laid as 64-byte two-child nodes (rt_gnode: both children's
// boxes and references, four 128-bit loads per visited inner node) and a 48-byte triangle
// position record per baked triangle (three 128-bit loads per triangle test). Node indices are
// those of the .bvh array, so the traversal visits exactly the reference's nodes.
//
// Equivalence with the reference loop: the reference pops a node and re-tests its box against
// the current best t (bvh_traverse.cpp:104-110); here the stack keeps the entry distance tNear
// computed when the node was pushed. The slab interval's far end depends on the best t only
// through min(tFar, bestT), so "rayAABB(node, bestT) >= bestT" holds exactly when
// tNear >= bestT (also with the NaN slabs of axis-parallel rays: tNear, and whether tFar is NaN,
// do not depend on bestT). Children are tested and pushed in the reference's order (far child
// first, the left child first on ties, :143-174) and triangles are tested in leaf order with the
// strict "t < bestT" update (:112-142), so the first triangle at the minimal distance wins as
// in the reference and hits carry identical triangle indices (trace_core.cuh).
//
// The kernel is persistent: each warp claims 32 rays at a time from a global counter until
// the batch is exhausted, so long incoherent rays do not leave SMs idle at the tail.
#include "trace_core.cuh"

#include <mutex>
#include <vector>

namespace rtb
{

namespace
{

constexpr int TBLK = 128;

// Also validates the structure before any traversal may run on it: children of node i have
// larger indices (DFS pre-order, so no cycles) inside the array, leaf ranges inside the
// triangle array. A violation sets ST_CAPACITY and the handle is refused.
// d_counts (optional) holds {nodes, triangles} on the device (a build that has not synchronised);
// thread 0 also writes the traversal entry record of node 0.
__global__ void k_make_gnodes(const rt_bvh_node* __restrict__ nodes, uint32_t n_nodes, uint32_t n_tris,
                              const uint32_t* __restrict__ d_counts, rt_gnode* __restrict__ gn, TraceRoot* __restrict__ root,
                              uint32_t* __restrict__ status)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_counts) { n_nodes = d_counts[0]; n_tris = d_counts[1]; }
    if (i >= n_nodes) { return; }
    const rt_bvh_node nd = nodes[i];
    if (i == 0)
    {
        TraceRoot r;
        for (int k = 0; k < 3; k++) { r.box[k] = nd.bmin[k]; r.box[3 + k] = nd.bmax[k]; }
        r.ref = nd.is_leaf ? nd.a : 0u;
        r.cnt = nd.is_leaf ? (LEAF_BIT | nd.b) : 0u;
        *root = r;
    }
    if (nd.is_leaf)
    {
        if ((uint64_t)nd.a + nd.b > n_tris) { atomicOr(status, ST_CAPACITY); }
        return;
    }
    if (nd.a <= i || nd.b <= i || nd.a >= n_nodes || nd.b >= n_nodes)
    {
        atomicOr(status, ST_CAPACITY);
        gn[i] = rt_gnode{ make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f),
                          make_uint4(0u, 0u, LEAF_BIT, LEAF_BIT) };
        return;
    }
    const rt_bvh_node l = nodes[nd.a], r = nodes[nd.b];
    rt_gnode g;
    g.a = make_float4(l.bmin[0], l.bmin[1], l.bmin[2], l.bmax[0]);
    g.b = make_float4(l.bmax[1], l.bmax[2], r.bmin[0], r.bmin[1]);
    g.c = make_float4(r.bmin[2], r.bmax[0], r.bmax[1], r.bmax[2]);
    g.d = make_uint4(l.is_leaf ? l.a : nd.a, r.is_leaf ? r.a : nd.b, l.is_leaf ? (LEAF_BIT | l.b) : 0u,
                     r.is_leaf ? (LEAF_BIT | r.b) : 0u);
    gn[i] = g;
}

__global__ void k_make_tripos(const rt_triangle* __restrict__ tris, uint32_t n, const uint32_t* __restrict__ d_counts,
                              const rt_vertex* __restrict__ v, float4* __restrict__ tp)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_counts) { n = d_counts[1]; }
    if (i >= n) { return; }
    const rt_triangle t = tris[i];
    const rt_vertex a = v[t.v[0]], b = v[t.v[1]], c = v[t.v[2]];
    tp[3 * i + 0] = make_float4(a.x, a.y, a.z, b.x);
    tp[3 * i + 1] = make_float4(b.y, b.z, c.x, c.y);
    tp[3 * i + 2] = make_float4(c.z, 0.f, 0.f, 0.f);
}

// Entry record of each scene root of a batched build; d_counts[0] = node count. A root
// outside the node array (a record the build did not write) sets ST_CAPACITY.
__global__ void k_scene_roots(const rt_bvh_node* __restrict__ nodes, const uint32_t* __restrict__ info, uint32_t S,
                              const uint32_t* __restrict__ d_counts, TraceRoot* __restrict__ out,
                              uint32_t* __restrict__ status)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) { return; }
    if (info[4 * s] >= d_counts[0])
    {
        atomicOr(status, ST_CAPACITY);
        out[s] = TraceRoot{ { 0.f, 0.f, 0.f, 0.f, 0.f, 0.f }, 0u, LEAF_BIT };
        return;
    }
    const rt_bvh_node nd = nodes[info[4 * s]];
    TraceRoot r;
    for (int k = 0; k < 3; k++) { r.box[k] = nd.bmin[k]; r.box[3 + k] = nd.bmax[k]; }
    r.ref = nd.is_leaf ? nd.a : info[4 * s];
    r.cnt = nd.is_leaf ? (LEAF_BIT | nd.b) : 0u;
    out[s] = r;
}

// Tree depth: parent links (children of node i have larger indices), then every leaf counts
// its ancestors (bounded by the node count).
__global__ void k_parents(const rt_bvh_node* __restrict__ nodes, uint32_t n, uint32_t* __restrict__ par)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    if (i == 0) { par[0] = 0xffffffffu; }
    const rt_bvh_node nd = nodes[i];
    if (!nd.is_leaf && nd.a < n && nd.b < n) { par[nd.a] = i; par[nd.b] = i; }
}
__global__ void k_depth(const rt_bvh_node* __restrict__ nodes, uint32_t n, const uint32_t* __restrict__ par,
                        uint32_t* __restrict__ depth)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !nodes[i].is_leaf) { return; }
    uint32_t d = 0;
    for (uint32_t p = par[i]; p != 0xffffffffu && d < n; p = par[p]) { d++; }
    atomicMax(depth, d);
}

// rt_ray records in, rt_hit records out (two 128-bit accesses each). n_dev, when set, holds
// the ray count on the device (the wavefront path tracer's queue length). ROOTS: ray i
// traces the subtree roots[rscene[i]] (a scene of a batched build).
template <int MODE, int STK, bool ROOTS, bool WIDE = false>
__global__ void __launch_bounds__(256)
k_trace(TraceCtx T, const float4* __restrict__ rays, float4* __restrict__ hits, uint64_t n, const uint32_t* __restrict__ n_dev,
        unsigned long long* __restrict__ counter, uint32_t* __restrict__ status, const TraceRoot* __restrict__ roots,
        const uint32_t* __restrict__ rscene)
{
    const int lane = threadIdx.x & 31;
    if (n_dev) { n = *n_dev; }
    TraceRoot R0;
    if (!ROOTS) { R0 = *T.root; }
    for (;;)
    {
        unsigned long long base = 0;
        if (lane == 0) { base = atomicAdd(counter, 32ull); }
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) { return; }
        const uint64_t ri = base + (uint64_t)lane;
        if (ri >= n) { continue; }
        const float4 r0 = rays[2 * ri], r1 = rays[2 * ri + 1];
        const TraceRoot& R = ROOTS ? roots[rscene[ri]] : R0;
        const f3 o = mk3(r0.x, r0.y, r0.z), d = mk3(r1.x, r1.y, r1.z);
        THit H;
        if constexpr (WIDE) { H = trace_ray_wide<MODE, STK>(T, R, o, d, r0.w, r1.w); }  // one entry per wide level
        else { H = trace_ray<MODE, STK>(T, R, o, d, r0.w, r1.w); }
        float4 h0 = make_float4(0.f, 0.f, 0.f, 0.f), h1 = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t flags = 0;
        if (H.hit)
        {
            const f3 nrm = hit_normal(T, H.tri, H.u, H.v);
            h0 = make_float4(H.t, H.u, H.v, __uint_as_float(H.tri));
            h1 = make_float4(nrm.x, nrm.y, nrm.z, 0.f);
            flags = RT_HIT_FLAG_HIT;
        }
        if (H.overflow) { flags |= RT_HIT_FLAG_OVERFLOW; atomicOr(status, ST_STACK); }
        h1.w = __uint_as_float(flags);
        hits[2 * ri] = h0;
        hits[2 * ri + 1] = h1;
    }
}

using TraceFn = void (*)(TraceCtx, const float4*, float4*, uint64_t, const uint32_t*, unsigned long long*, uint32_t*,
                         const TraceRoot*, const uint32_t*);

TraceFn trace_fn(uint32_t flags, int stack, bool roots, bool wide)
{
    if (wide)
    {
        if (roots) { return (flags & 3u) == 0 ? k_trace<0, STACK, true, true> : nullptr; }
        switch (flags & 3u)
        {
        case 0: return k_trace<0, STACK, false, true>;
        case 1: return k_trace<1, STACK, false, true>;
        case 2: return k_trace<2, STACK, false, true>;
        default: return k_trace<3, STACK, false, true>;
        }
    }
    if (stack <= 32)
    {
        if (roots) { return k_trace<0, 32, true>; }
        return (flags & 3u) == 0 ? k_trace<0, 32, false> : nullptr;
    }
    if (roots) { return k_trace<0, STACK, true>; }
    switch (flags & 3u)
    {
    case 0: return k_trace<0, STACK, false>;
    case 1: return k_trace<1, STACK, false>;
    case 2: return k_trace<2, STACK, false>;
    default: return k_trace<3, STACK, false>;
    }
}

// Resident blocks per SM, per kernel variant and block size.
std::mutex g_occ_mu;
struct OccKey { TraceFn fn; int block; int v; };
std::vector<OccKey> g_occ;

int blocks_per_sm(TraceFn fn, int block)
{
    std::lock_guard<std::mutex> lk(g_occ_mu);
    for (const OccKey& k : g_occ)
    {
        if (k.fn == fn && k.block == block) { return k.v; }
    }
    int v = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, fn, block, 0) != cudaSuccess) { cudaGetLastError(); v = 1; }
    if (v < 1) { v = 1; }
    g_occ.push_back(OccKey{ fn, block, v });
    return v;
}

} // namespace

TraceCtx make_trace_ctx(const rt_bvh* B)
{
    TraceCtx T;
    T.gn = B->gnodes.as<rt_gnode>();
    T.tp = B->tripos.as<float4>();
    T.tris = B->tris.as<rt_triangle>();
    T.verts = B->verts.as<rt_vertex>();
    T.root = B->rootbuf.as<TraceRoot>();
    T.ww = B->trace_ww ? 1u : 0u;
    T.wn = B->wnodes.as<rt_wnode>();
    T.wid = B->wid.as<uint32_t>();
    return T;
}

int launch_traversal_layout(rt_bvh* B, cudaStream_t st, uint32_t max_nodes, uint32_t max_tris, const uint32_t* d_counts,
                            uint32_t* vstatus, bool tripos_ready, bool gnodes_ready)
{
    if (B->gnodes.ensure((size_t)max_nodes * sizeof(rt_gnode)) || B->tripos.ensure((size_t)(max_tris ? max_tris : 1) * 48) ||
        B->rootbuf.ensure(sizeof(TraceRoot)))
    {
        return RT_E_CUDA;
    }
    if (!gnodes_ready)
    {
        k_make_gnodes<<<(max_nodes + 255) / 256, 256, 0, st>>>(B->nodes.as<rt_bvh_node>(), max_nodes, max_tris, d_counts,
                                                               B->gnodes.as<rt_gnode>(), B->rootbuf.as<TraceRoot>(), vstatus);
        count_launch();
    }
    if (max_tris && !tripos_ready)
    {
        k_make_tripos<<<(max_tris + 255) / 256, 256, 0, st>>>(B->tris.as<rt_triangle>(), max_tris, d_counts,
                                                              B->verts.as<rt_vertex>(), B->tripos.as<float4>());
        count_launch();
    }
    return check_launch("traversal layout");
}

int make_traversal_layout(rt_bvh* B, cudaStream_t st)
{
    if (B->n_nodes == 0) { return fail(RT_E_EMPTY, "empty BVH"); }
    if (B->trace_status.ensure(64)) { return RT_E_CUDA; }
    uint32_t* vstatus = B->trace_status.as<uint32_t>() + 12;
    RT_CUDA(cudaMemsetAsync(vstatus, 0, 4, st));
    if (int e = launch_traversal_layout(B, st, B->n_nodes, B->n_tris, nullptr, vstatus)) { return e; }
    uint32_t vs = 0;
    RT_CUDA(cudaMemcpyAsync(&vs, vstatus, 4, cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    if (vs) { return fail(RT_E_FORMAT, "BVH structure check failed (child or triangle index out of range)"); }
    return RT_OK;
}

int trace_launch(const rt_bvh* B, const void* d_rays, void* d_hits, uint64_t n, const uint32_t* n_dev, uint32_t flags,
                 cudaStream_t st, uint32_t* d_status, unsigned long long* d_counter, const TraceLaunch& opt)
{
    const TraceFn fn = trace_fn(flags, opt.stack, opt.roots != nullptr, B->trace_wide);
    if (!fn) { return fail(RT_E_INVALID, "no trace kernel for this mode and stack depth"); }
    const int block = opt.block > 0 ? opt.block : TBLK;
    if (block % 32 || block > 256) { return fail(RT_E_INVALID, "trace block must be a multiple of 32, at most 256"); }
    uint64_t grid = (uint64_t)device_sm_count() * (uint64_t)blocks_per_sm(fn, block);
    if (!n_dev)
    {
        const uint64_t want = (n + block - 1) / block;
        if (grid > want) { grid = want; }
    }
    if (grid == 0) { return RT_OK; }
    const TraceCtx T = make_trace_ctx(B);
    fn<<<(uint32_t)grid, block, 0, st>>>(T, static_cast<const float4*>(d_rays), static_cast<float4*>(d_hits), n, n_dev,
                                         d_counter, d_status, opt.roots, opt.rscene);
    count_launch();
    return check_launch("trace");
}

int launch_scene_roots(rt_bvh* B, uint32_t S, const uint32_t* d_counts, uint32_t* status, cudaStream_t st)
{
    k_scene_roots<<<(S + 127) / 128, 128, 0, st>>>(B->nodes.as<rt_bvh_node>(), B->scene_info.as<uint32_t>(), S, d_counts,
                                                   B->scene_roots.as<TraceRoot>(), status);
    count_launch();
    return check_launch("scene roots");
}

int tree_depth(rt_bvh* B, cudaStream_t st, uint32_t* depth)
{
    if (B->depth) { *depth = B->depth; return RT_OK; }
    const uint32_t n = B->n_nodes;
    DevBuf tmp;
    if (tmp.ensure((size_t)n * 4 + 16)) { return RT_E_CUDA; }
    uint32_t* par = tmp.as<uint32_t>();
    uint32_t* d = par + n;
    int e = RT_OK;
    if (cudaMemsetAsync(d, 0, 4, st) != cudaSuccess) { e = fail(RT_E_CUDA, "memset"); }
    if (!e)
    {
        k_parents<<<(n + 255) / 256, 256, 0, st>>>(B->nodes.as<rt_bvh_node>(), n, par);
        k_depth<<<(n + 255) / 256, 256, 0, st>>>(B->nodes.as<rt_bvh_node>(), n, par, d);
        count_launch(2);
        e = check_launch("depth");
    }
    uint32_t v = 0;
    if (!e && (cudaMemcpyAsync(&v, d, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess))
    {
        e = fail(RT_E_CUDA, "depth readback");
    }
    tmp.release();
    if (e) { return e; }
    B->depth = v;
    *depth = v;
    return RT_OK;
}

int trace(const rt_bvh* B, const rt_ray* d_rays, rt_hit* d_hits, uint64_t n, uint32_t flags, cudaStream_t st,
          uint32_t* d_status)
{
    if (n == 0) { return RT_OK; }
    if (((uintptr_t)d_rays & 15) || ((uintptr_t)d_hits & 15)) { return fail(RT_E_INVALID, "rays/hits must be 16-byte aligned"); }
    rt_bvh* Bm = const_cast<rt_bvh*>(B);
    if (Bm->trace_status.ensure(64)) { return RT_E_CUDA; }
    unsigned long long* counter = Bm->trace_status.as<unsigned long long>();
    RT_CUDA(cudaMemsetAsync(counter, 0, 8, st));
    return trace_launch(B, d_rays, d_hits, n, nullptr, flags, st, d_status, counter, TraceLaunch{});
}

} // namespace rtb
