// wide.cu -- the 8-wide traversal layout: the baked binary tree collapsed into 128-byte nodes
// of up to eight children with child boxes quantised to 8 bits per plane against the union of
// the children's boxes, children placed in octant slots (after the compressed wide BVH of
// Ylitie, Karras and Laine, HPG 2017, in a simpler form: explicit child references, a greedy
// slot assignment).
//
// Which binary nodes become wide nodes: the root, every inner node whose depth is a multiple
// of three, and every scene root of a batched build. A wide node's children are found by
// replacing, in the list {node}, every inner node that is not itself a wide node by its two
// children until only leaves and wide nodes remain -- at most eight, since wide nodes recur
// at least every third level. Wide nodes are numbered in the binary array's (pre-)order, so
// the root is wide node 0 and a subtree's wide nodes sit together.
//
// Quantisation is conservative: a child's decoded box (origin + q * 2^e, in the same float
// operations the traversal uses) contains its exact box, so the traversal tests every
// triangle the exact boxes would let it test, and possibly a few more.
#include "rt_internal.h"
#include "device_math.cuh"

#include <algorithm>

namespace rtb
{

namespace
{

constexpr uint32_t WNONE = 0xffffffffu;
constexpr uint32_t WMAX_DEPTH = 1u << 12;  // bound of the depth walk (the tree is checked acyclic)

__global__ void k_wide_parents(const rt_bvh_node* __restrict__ nodes, uint32_t n, uint32_t* __restrict__ par)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    if (i == 0) { par[0] = WNONE; }
    const rt_bvh_node nd = nodes[i];
    if (!nd.is_leaf && nd.a < n && nd.b < n) { par[nd.a] = i; par[nd.b] = i; }
}

// flag[i] = 1 for the wide nodes (see the file comment).
__global__ void k_wide_flags(const rt_bvh_node* __restrict__ nodes, uint32_t n, const uint32_t* __restrict__ par,
                             uint32_t* __restrict__ flag)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    if (nodes[i].is_leaf) { flag[i] = 0u; return; }
    uint32_t d = 0;
    for (uint32_t p = par[i]; p != WNONE && d < WMAX_DEPTH; p = par[p]) { d++; }
    flag[i] = (d % 3u == 0u) ? 1u : 0u;
}

// Scene roots of a batched build are wide nodes too (their subtrees are traced on their own).
__global__ void k_wide_scene_flags(const uint32_t* __restrict__ info, uint32_t S, const rt_bvh_node* __restrict__ nodes,
                                   uint32_t n, uint32_t* __restrict__ flag)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) { return; }
    const uint32_t r = info[4 * s];
    if (r < n && !nodes[r].is_leaf) { flag[r] = 1u; }
}

// The float operations of the traversal's decode: origin + q * 2^e.
__device__ __forceinline__ float wdecode(float p, uint32_t q, float s) { return __fadd_rn(p, __fmul_rn((float)q, s)); }

// Scale 2^e (e a normal exponent) with 255 * 2^e reaching hi from p in decoded form.
__device__ __forceinline__ uint32_t wexponent(float p, float hi)
{
    const double ext = (double)hi - (double)p;
    int k = 0;
    if (ext > 0.0) { (void)frexp(ext / 255.0, &k); }  // ext / 255 < 2^k
    int e = k + 127;
    e = e < 1 ? 1 : (e > 254 ? 254 : e);
    while (e < 254 && wdecode(p, 255u, __uint_as_float((uint32_t)e << 23)) < hi) { e++; }
    return (uint32_t)e;
}

__global__ void k_wide_build(const rt_bvh_node* __restrict__ nodes, uint32_t n, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ wid, rt_wnode* __restrict__ out, uint32_t* __restrict__ status)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) { return; }
    uint32_t list[8];
    int cnt = 0;
    {
        const rt_bvh_node nd = nodes[i];
        list[cnt++] = nd.a;
        list[cnt++] = nd.b;
    }
    // expand inner non-wide entries (three rounds reach the next wide level)
    for (int round = 0; round < 3; round++)
    {
        uint32_t nl[8];
        int nc = 0;
        bool bad = false;
        for (int k = 0; k < cnt; k++)
        {
            const uint32_t c = list[k];
            const rt_bvh_node cn = nodes[c];
            if (cn.is_leaf || flag[c]) { if (nc < 8) { nl[nc++] = c; } else { bad = true; } }
            else
            {
                if (nc + 2 <= 8) { nl[nc++] = cn.a; nl[nc++] = cn.b; } else { bad = true; }
            }
        }
        if (bad) { atomicOr(status, ST_CAPACITY); return; }
        for (int k = 0; k < nc; k++) { list[k] = nl[k]; }
        cnt = nc;
    }
    // the quantisation frame: the union of the children's boxes
    rt_bvh_node cn[8];
    bool present[8];
    float lo3[3] = { 0.f, 0.f, 0.f }, hi3[3] = { 0.f, 0.f, 0.f };
    bool any = false;
    for (int c = 0; c < cnt; c++)
    {
        cn[c] = nodes[list[c]];
        bool empty = cn[c].is_leaf && cn[c].b == 0u;  // no triangles
        for (int a = 0; a < 3; a++) { empty |= !(cn[c].bmin[a] <= cn[c].bmax[a]); }  // empty or NaN box: never hit
        present[c] = !empty;
        if (empty) { continue; }
        for (int a = 0; a < 3; a++)
        {
            lo3[a] = any ? fminf(lo3[a], cn[c].bmin[a]) : cn[c].bmin[a];
            hi3[a] = any ? fmaxf(hi3[a], cn[c].bmax[a]) : cn[c].bmax[a];
        }
        any = true;
    }
    // slots by octant: child c goes to a slot s whose octant (bit a set: the positive side of
    // axis a) matches the offset of its box centre from the node's centre, greedily by the
    // smallest cost; a ray whose direction has the signs o (bit a set: negative) visits slot s
    // as its (s ^ o)-th, near to far along each axis
    int slot[8];
    bool used[8];
    float off[8][3];
    float ctr[3];
    for (int a = 0; a < 3; a++) { ctr[a] = __fmul_rn(__fadd_rn(lo3[a], hi3[a]), 0.5f); }
    int npres = 0;
    for (int c = 0; c < 8; c++) { slot[c] = -1; used[c] = false; }
    for (int c = 0; c < cnt; c++)
    {
        if (!present[c]) { continue; }
        npres++;
        for (int a = 0; a < 3; a++) { off[c][a] = __fsub_rn(__fmul_rn(__fadd_rn(cn[c].bmin[a], cn[c].bmax[a]), 0.5f), ctr[a]); }
    }
    for (int r = 0; r < npres; r++)
    {
        float bv = 0.f;
        int bc = -1, bs = -1;
        for (int c = 0; c < cnt; c++)
        {
            if (!present[c] || slot[c] >= 0) { continue; }
            for (int sl = 0; sl < 8; sl++)
            {
                if (used[sl]) { continue; }
                const float v = __fadd_rn(__fadd_rn((sl & 1) ? -off[c][0] : off[c][0], (sl & 2) ? -off[c][1] : off[c][1]),
                                          (sl & 4) ? -off[c][2] : off[c][2]);
                if (bc < 0 || v < bv) { bv = v; bc = c; bs = sl; }
            }
        }
        slot[bc] = bs;
        used[bs] = true;
    }
    rt_wnode w;
    uint32_t e[3];
    for (int a = 0; a < 3; a++) { w.p[a] = lo3[a]; e[a] = wexponent(lo3[a], hi3[a]); }
    uint32_t imask = 0;
    for (int c = 0; c < 8; c++)
    {
        w.ref[c] = 0u; w.cnt[c] = 0u;
        for (int a = 0; a < 3; a++) { w.qlo[a][c] = 0u; w.qhi[a][c] = 0u; }
    }
    for (int c0 = 0; c0 < cnt; c0++)
    {
        if (!present[c0]) { continue; }
        const int c = slot[c0];  // written to its slot; cn / list stay indexed by c0
        if (cn[c0].is_leaf)
        {
            if (cn[c0].b > 0xffffu) { atomicOr(status, ST_CAPACITY); return; }
            w.ref[c] = cn[c0].a;
            w.cnt[c] = (uint16_t)cn[c0].b;
        }
        else
        {
            if (!flag[list[c0]]) { atomicOr(status, ST_CAPACITY); return; }
            w.ref[c] = wid[list[c0]];
            w.cnt[c] = 1u;
            imask |= 1u << c;
        }
        for (int a = 0; a < 3; a++)
        {
            const float s = __uint_as_float(e[a] << 23);
            const float p = lo3[a];
            const double ql = floor(((double)cn[c0].bmin[a] - (double)p) / (double)s);
            const double qh = ceil(((double)cn[c0].bmax[a] - (double)p) / (double)s);
            uint32_t lo = (uint32_t)fmin(fmax(ql, 0.0), 255.0), hi = (uint32_t)fmin(fmax(qh, 0.0), 255.0);
            while (lo > 0u && wdecode(p, lo, s) > cn[c0].bmin[a]) { lo--; }
            while (hi < 255u && wdecode(p, hi, s) < cn[c0].bmax[a]) { hi++; }
            if (wdecode(p, lo, s) > cn[c0].bmin[a] || wdecode(p, hi, s) < cn[c0].bmax[a]) { atomicOr(status, ST_CAPACITY); }
            w.qlo[a][c] = (uint8_t)lo;
            w.qhi[a][c] = (uint8_t)hi;
        }
    }
    w.meta = e[0] | (e[1] << 8) | (e[2] << 16) | (imask << 24);
    for (int k = 0; k < 4; k++) { w.pad[k] = 0u; }
    out[wid[i]] = w;
}

} // namespace

int make_wide_layout(rt_bvh* B, cudaStream_t st)
{
    const uint32_t n = B->n_nodes;
    if (n == 0) { return fail(RT_E_EMPTY, "empty BVH"); }
    if (B->wid.ensure((size_t)n * 4) || B->s.wide_flag.ensure((size_t)n * 4) || B->s.wide_par.ensure((size_t)n * 4) ||
        B->trace_status.ensure(64))
    {
        return RT_E_CUDA;
    }
    uint32_t* status = B->trace_status.as<uint32_t>() + 13;
    uint32_t* total = B->trace_status.as<uint32_t>() + 14;
    RT_CUDA(cudaMemsetAsync(status, 0, 8, st));
    const uint32_t nb = (n + 255) / 256;
    k_wide_parents<<<nb, 256, 0, st>>>(B->nodes.as<rt_bvh_node>(), n, B->s.wide_par.as<uint32_t>());
    k_wide_flags<<<nb, 256, 0, st>>>(B->nodes.as<rt_bvh_node>(), n, B->s.wide_par.as<uint32_t>(),
                                     B->s.wide_flag.as<uint32_t>());
    count_launch(2);
    if (B->n_scenes > 1)
    {
        k_wide_scene_flags<<<(B->n_scenes + 255) / 256, 256, 0, st>>>(B->scene_info.as<uint32_t>(), B->n_scenes,
                                                                      B->nodes.as<rt_bvh_node>(), n,
                                                                      B->s.wide_flag.as<uint32_t>());
        count_launch();
    }
    if (int e = exclusive_scan_u32(B->s.wide_flag.as<uint32_t>(), B->wid.as<uint32_t>(), n, total, B->s.scan, st)) { return e; }
    uint32_t nw = 0;
    RT_CUDA(cudaMemcpyAsync(&nw, total, 4, cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    if (B->wnodes.ensure((size_t)std::max<uint32_t>(nw, 1) * sizeof(rt_wnode))) { return RT_E_CUDA; }
    if (nw > 0)
    {
        k_wide_build<<<nb, 256, 0, st>>>(B->nodes.as<rt_bvh_node>(), n, B->s.wide_flag.as<uint32_t>(), B->wid.as<uint32_t>(),
                                         B->wnodes.as<rt_wnode>(), status);
        count_launch();
    }
    if (int e = check_launch("wide layout")) { return e; }
    uint32_t st_h = 0;
    RT_CUDA(cudaMemcpyAsync(&st_h, status, 4, cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    if (st_h) { return fail(RT_E_CAPACITY, "wide layout: a node has more than eight children or a leaf over 65,535 triangles"); }
    B->n_wide = nw;
    return RT_OK;
}

} // namespace rtb
