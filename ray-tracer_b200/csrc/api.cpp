// api.cpp -- the C ABI of librt_b200.so (include/rt_b200.h): handles, errors, device buffers,
// .bvh v1 file I/O and host-side scene ingestion. All compute goes to the CUDA kernels of
// build.cu / sah.cu / traverse.cu / render.cu; nothing here computes a BVH or a hit.
#include "rt_internal.h"
#include "host_geom.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

// ---------------------------------------------------------------------------------------
namespace rtb
{
static thread_local std::string g_err;
static std::atomic<uint64_t> g_launches{ 0 };
static std::atomic<uint64_t> g_allocs{ 0 };

void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}
static thread_local uint64_t t_launches = 0;
void count_launch(uint64_t n)
{
    g_launches.fetch_add(n, std::memory_order_relaxed);
    t_launches += n;
}
uint64_t thread_launches() { return t_launches; }
void count_alloc() { g_allocs.fetch_add(1, std::memory_order_relaxed); }
int check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { return fail(RT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e)); }
    return RT_OK;
}

int DevBuf::ensure(size_t n)
{
    if (n <= bytes && p) { return 0; }
    if (p) { cudaFree(p); p = nullptr; bytes = 0; }
    size_t want = std::max<size_t>(n, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess)
    {
        p = nullptr;
        set_error(std::string("cudaMalloc(") + std::to_string(want) + "): " + cudaGetErrorString(e));
        return RT_E_CUDA;
    }
    bytes = want;
    count_alloc();
    return 0;
}
void DevBuf::release()
{
    if (p) { cudaFree(p); }
    p = nullptr;
    bytes = 0;
}

static std::mutex g_dev_mu;
static cudaStream_t g_streams[64];
static int g_sms[64];

static int current_device()
{
    int d = 0;
    cudaGetDevice(&d);
    return d < 0 || d >= 64 ? 0 : d;
}
cudaStream_t default_stream()
{
    std::lock_guard<std::mutex> lk(g_dev_mu);
    const int d = current_device();
    if (!g_streams[d]) { cudaStreamCreateWithFlags(&g_streams[d], cudaStreamNonBlocking); }
    return g_streams[d];
}
int device_sm_count()
{
    std::lock_guard<std::mutex> lk(g_dev_mu);
    const int d = current_device();
    if (!g_sms[d])
    {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
        g_sms[d] = v > 0 ? v : 1;
    }
    return g_sms[d];
}

static int require_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
    {
        cudaGetLastError();
        return fail(RT_E_CUDA, std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "none found"));
    }
    return RT_OK;
}
} // namespace rtb

using namespace rtb;

static cudaStream_t pick(void* s) { return s ? static_cast<cudaStream_t>(s) : default_stream(); }

static void free_bvh(rt_bvh* b)
{
    if (!b) { return; }
    DevBuf* bufs[] = { &b->nodes, &b->tris, &b->verts, &b->prim, &b->gnodes, &b->tripos, &b->trace_status, &b->trace_rays,
                       &b->trace_hits, &b->s.tri_lo, &b->s.tri_hi, &b->s.tri_cz, &b->s.keys, &b->s.vals, &b->s.hist,
                       &b->s.scene, &b->s.status, &b->s.sort.keys_alt, &b->s.sort.vals_alt, &b->s.sort.lookback,
                       &b->s.sort.tile_counters, &b->s.scan.partials, &b->s.knode, &b->s.parent, &b->s.kbox, &b->s.lvbox, &b->s.kflag, &b->s.ktab, &b->s.tpin,
                       &b->s.rank, &b->s.bnd, &b->s.wnode, &b->s.wtri, &b->s.snode, &b->s.stri, &b->s.counters,
                       &b->s.sah_roots, &b->s.sah_refs_a, &b->s.sah_refs_b, &b->s.sah_tmp, &b->s.sah_pos,
                       &b->s.sah_lvl_a, &b->s.sah_lvl_b, &b->s.sah_dec, &b->s.sah_out, &b->s.sah_leaf_refs,
                       &b->s.sah_scan_in, &b->s.sah_scan_out, &b->s.sah_node_ids, &b->s.sah_roots_lvl, &b->s.sah_root_ord, &b->s.root_sort.keys_alt,
                       &b->s.root_sort.vals_alt, &b->s.root_sort.lookback, &b->s.root_sort.tile_counters,
                       &b->s.in_verts, &b->s.in_tris, &b->s.gtris, &b->s.batch_off, &b->s.sah_budget, &b->s.sah_wide, &b->s.sah_tmp2, &b->s.sah_pos2, &b->s.wide_flag, &b->s.wide_par, &b->wnodes, &b->wid, &b->scene_info, &b->scene_roots,
                       &b->wf_cams };
    for (DevBuf* x : bufs) { x->release(); }
    b->rootbuf.release();
    for (int k = 0; k < 2; k++) { b->wf_rays[k].release(); b->wf_state[k].release(); b->wf_scene[k].release(); }
    b->wf_hits.release(); b->wf_acc.release(); b->wf_ctr.release();
    if (b->wf_exec) { cudaGraphExecDestroy(b->wf_exec); b->wf_exec = nullptr; }
    for (cudaEvent_t& e : b->wf_ev)
    {
        if (e) { cudaEventDestroy(e); e = nullptr; }
    }
    if (b->wf_stream) { cudaStreamDestroy(b->wf_stream); b->wf_stream = nullptr; }
    if (b->bake_exec) { cudaGraphExecDestroy(b->bake_exec); b->bake_exec = nullptr; }
    for (cudaEvent_t& e : b->bake_ev)
    {
        if (e) { cudaEventDestroy(e); e = nullptr; }
    }
    if (b->bake_stream) { cudaStreamDestroy(b->bake_stream); b->bake_stream = nullptr; }
    for (cudaEvent_t& e : b->ev)
    {
        if (e) { cudaEventDestroy(e); e = nullptr; }
    }
    delete b;
}

static int check_render_args(const rt_bvh* b, const rt_render_cfg* cfg, const rt_shading* sh, rt_shading* out)
{
    if (!b) { return fail(RT_E_NOT_LOADED, "BVH not loaded"); }
    if (!cfg) { return fail(RT_E_INVALID, "null argument"); }
    if (cfg->width == 0 || cfg->height == 0 || cfg->spp == 0) { return fail(RT_E_INVALID, "empty image or spp = 0"); }
    *out = sh ? *sh : rt_shading{ nullptr, nullptr, nullptr, nullptr, 0u, 0u, 0u, 0u };
    if ((out->mats != nullptr) != (out->n_mats > 0)) { return fail(RT_E_INVALID, "mats and n_mats > 0 go together"); }
    if (out->mat_of_tri && !out->mats) { return fail(RT_E_INVALID, "mat_of_tri without materials"); }
    if (cfg->env_kind > 2) { return fail(RT_E_INVALID, "env_kind must be 0, 1 or 2"); }
    if (cfg->env_kind == 2 && (!out->env_map || out->env_w == 0 || out->env_h == 0))
    {
        return fail(RT_E_INVALID, "env_kind 2 needs the shading's env_map with its size");
    }
    return RT_OK;
}

extern "C" {

void rt_build_cfg_default(rt_build_cfg* c)
{
    if (!c) { return; }
    c->lbvh_threshold = 64;
    c->max_leaf = 16;
    c->morton_bits = 21;
    c->bins_min = 8;
    c->bins_max = 32;
    c->c_trav = 1.0f;
    c->c_isect = 1.2f;
    c->centroid_eps = 1e-6f;
    c->spatial_eps = 1e-6f;
    c->spatial_mult = 1.5f;
}

const char* rt_last_error(void) { return g_err.c_str(); }
const char* rt_version(void) { return "rt_b200 1.0 (sm_100a)"; }
uint64_t rt_kernel_launches(void) { return g_launches.load(); }
uint64_t rt_device_allocations(void) { return g_allocs.load(); }

int rt_device_sync(void* stream)
{
    if (int e = require_device()) { return e; }
    RT_CUDA(cudaStreamSynchronize(pick(stream)));
    return RT_OK;
}

int rt_rebuild(rt_bvh* b, const void* verts, uint32_t n_verts, const void* tris, uint32_t n_tris, int where,
               const rt_build_cfg* cfg, void* stream)
{
    if (!b) { return fail(RT_E_INVALID, "null handle"); }
    if (n_verts == 0 || n_tris == 0) { return fail(RT_E_EMPTY, "no vertices or no triangles (initGeos)"); }
    if (!verts || !tris) { return fail(RT_E_INVALID, "null geometry pointer"); }
    if (int e = require_device()) { return e; }
    rt_build_cfg c;
    if (cfg) { c = *cfg; } else { rt_build_cfg_default(&c); }
    cudaStream_t st = pick(stream);
    const rt_vertex* dv = static_cast<const rt_vertex*>(verts);
    const rt_triangle* dt = static_cast<const rt_triangle*>(tris);
    if (where == RT_HOST)
    {
        if (b->s.in_verts.ensure((size_t)n_verts * sizeof(rt_vertex)) || b->s.in_tris.ensure((size_t)n_tris * sizeof(rt_triangle)))
        {
            return RT_E_CUDA;
        }
        RT_CUDA(cudaMemcpyAsync(b->s.in_verts.p, verts, (size_t)n_verts * sizeof(rt_vertex), cudaMemcpyHostToDevice, st));
        RT_CUDA(cudaMemcpyAsync(b->s.in_tris.p, tris, (size_t)n_tris * sizeof(rt_triangle), cudaMemcpyHostToDevice, st));
        dv = b->s.in_verts.as<rt_vertex>();
        dt = b->s.in_tris.as<rt_triangle>();
    }
    else if (where != RT_DEVICE) { return fail(RT_E_INVALID, "where must be RT_HOST or RT_DEVICE"); }
    b->depth = 0;
    if (int e = build_bvh(b, dv, n_verts, dt, n_tris, c, st)) { return e; }
    return b->trace_wide ? make_wide_layout(b, st) : RT_OK;  // the wide layout follows the tree
}

int rt_rebuild_batch(rt_bvh* b, const void* verts, const uint32_t* vert_offsets, const void* tris, const uint32_t* tri_offsets,
                     uint32_t n_scenes, int where, const rt_build_cfg* cfg, void* stream)
{
    if (!b) { return fail(RT_E_INVALID, "null handle"); }
    if (!verts || !tris || !vert_offsets || !tri_offsets) { return fail(RT_E_INVALID, "null pointer"); }
    if (n_scenes == 0) { return fail(RT_E_EMPTY, "no scenes"); }
    if (vert_offsets[0] != 0 || tri_offsets[0] != 0) { return fail(RT_E_INVALID, "offsets must start at 0"); }
    for (uint32_t s = 0; s < n_scenes; s++)
    {
        if (tri_offsets[s + 1] <= tri_offsets[s]) { return fail(RT_E_EMPTY, "scene " + std::to_string(s) + " has no triangles"); }
        if (vert_offsets[s + 1] <= vert_offsets[s]) { return fail(RT_E_EMPTY, "scene " + std::to_string(s) + " has no vertices"); }
    }
    const uint32_t V = vert_offsets[n_scenes], N = tri_offsets[n_scenes];
    if (int e = require_device()) { return e; }
    rt_build_cfg c;
    if (cfg) { c = *cfg; } else { rt_build_cfg_default(&c); }
    cudaStream_t st = pick(stream);
    auto bail = [&](int e) { return e; };
    b->depth = 0;
    const rt_vertex* dv = static_cast<const rt_vertex*>(verts);
    const rt_triangle* dt = static_cast<const rt_triangle*>(tris);
    if (b->s.batch_off.ensure((size_t)2 * (n_scenes + 1) * 4)) { return bail(RT_E_CUDA); }
    uint32_t* d_toff = b->s.batch_off.as<uint32_t>();
    uint32_t* d_voff = d_toff + (n_scenes + 1);
    if (cudaMemcpyAsync(d_toff, tri_offsets, (size_t)(n_scenes + 1) * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_voff, vert_offsets, (size_t)(n_scenes + 1) * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
    {
        return bail(fail(RT_E_CUDA, "offset upload"));
    }
    if (where == RT_HOST)
    {
        if (b->s.in_verts.ensure((size_t)V * sizeof(rt_vertex)) || b->s.in_tris.ensure((size_t)N * sizeof(rt_triangle)))
        {
            return bail(RT_E_CUDA);
        }
        if (cudaMemcpyAsync(b->s.in_verts.p, verts, (size_t)V * sizeof(rt_vertex), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(b->s.in_tris.p, tris, (size_t)N * sizeof(rt_triangle), cudaMemcpyHostToDevice, st) != cudaSuccess)
        {
            return bail(fail(RT_E_CUDA, "geometry upload"));
        }
        dv = b->s.in_verts.as<rt_vertex>();
        dt = b->s.in_tris.as<rt_triangle>();
    }
    else if (where != RT_DEVICE) { return bail(fail(RT_E_INVALID, "where must be RT_HOST or RT_DEVICE")); }
    if (int e = build_bvh_batch(b, dv, V, dt, N, c, st, n_scenes, d_toff, d_voff, tri_offsets)) { return e; }
    return b->trace_wide ? make_wide_layout(b, st) : RT_OK;
}

int rt_build_batch(const void* verts, const uint32_t* vert_offsets, const void* tris, const uint32_t* tri_offsets,
                   uint32_t n_scenes, int where, const rt_build_cfg* cfg, void* stream, rt_bvh** out)
{
    if (!out) { return fail(RT_E_INVALID, "null output handle"); }
    *out = nullptr;
    rt_bvh* b = new rt_bvh();
    cudaGetDevice(&b->device);
    const int e = rt_rebuild_batch(b, verts, vert_offsets, tris, tri_offsets, n_scenes, where, cfg, stream);
    if (e) { free_bvh(b); return e; }
    *out = b;
    return RT_OK;
}

int rt_bvh_scenes(const rt_bvh* b, uint32_t* n_scenes, uint32_t* info4)
{
    if (!b) { return fail(RT_E_NOT_LOADED, "BVH not loaded"); }
    if (n_scenes) { *n_scenes = b->n_scenes; }
    if (info4 && b->n_scenes) { std::memcpy(info4, b->scene_info_host.data(), (size_t)b->n_scenes * 16); }
    return RT_OK;
}

int rt_bvh_depth(rt_bvh* b, uint32_t* depth)
{
    if (!b) { return fail(RT_E_NOT_LOADED, "BVH not loaded"); }
    if (!depth) { return fail(RT_E_INVALID, "null argument"); }
    return tree_depth(b, default_stream(), depth);
}

int rt_render_batch(rt_bvh* b, const rt_render_cfg* cfgs, uint32_t n_scenes, const rt_shading* shading,
                    const rt_wavefront_params* params, float* rgb, float* rgb2, void* stream)
{
    rt_shading sh;
    if (int e = check_render_args(b, cfgs, shading, &sh)) { return e; }
    if (!rgb) { return fail(RT_E_INVALID, "null argument"); }
    if (n_scenes != std::max<uint32_t>(b->n_scenes, 1u)) { return fail(RT_E_INVALID, "n_scenes differs from the handle's scenes"); }
    return rtb::render_batch(b, cfgs, n_scenes, sh, params, rgb, rgb2, pick(stream));
}

int rt_autotune_wavefront(rt_bvh* b, const rt_render_cfg* cfgs, uint32_t n_scenes, const rt_shading* shading,
                          rt_wavefront_params* best, void* stream)
{
    rt_shading sh;
    if (int e = check_render_args(b, cfgs, shading, &sh)) { return e; }
    if (n_scenes != std::max<uint32_t>(b->n_scenes, 1u)) { return fail(RT_E_INVALID, "n_scenes differs from the handle's scenes"); }
    DevBuf scratch;
    if (scratch.ensure((size_t)n_scenes * cfgs[0].width * cfgs[0].height * 12)) { return RT_E_CUDA; }
    const int e = rtb::autotune_wavefront(b, cfgs, n_scenes, sh, best, scratch.as<float>(), pick(stream));
    cudaStreamSynchronize(pick(stream));
    scratch.release();
    return e;
}

int rt_build(const void* verts, uint32_t n_verts, const void* tris, uint32_t n_tris, int where, const rt_build_cfg* cfg,
             void* stream, rt_bvh** out)
{
    if (!out) { return fail(RT_E_INVALID, "null output handle"); }
    *out = nullptr;
    rt_bvh* b = new rt_bvh();
    cudaGetDevice(&b->device);
    int e = rt_rebuild(b, verts, n_verts, tris, n_tris, where, cfg, stream);
    if (e) { free_bvh(b); return e; }
    *out = b;
    return RT_OK;
}

int rt_bvh_from_arrays(const rt_bvh_node* nodes, uint32_t n_nodes, const rt_triangle* tris, uint32_t n_tris,
                       const rt_vertex* verts, uint32_t n_verts, rt_bvh** out)
{
    if (!out) { return fail(RT_E_INVALID, "null output handle"); }
    *out = nullptr;
    if (n_nodes == 0) { return fail(RT_E_FORMAT, "BVH without nodes"); }
    if (int e = require_device()) { return e; }
    // structural checks before any device pointer chasing: child and triangle indices
    uint64_t n_leaves = 0, leaf_tris = 0;
    for (uint32_t i = 0; i < n_nodes; i++)
    {
        const rt_bvh_node& nd = nodes[i];
        if (nd.is_leaf)
        {
            if ((uint64_t)nd.a + nd.b > n_tris) { return fail(RT_E_FORMAT, "leaf triangle range outside the triangle array"); }
            n_leaves++;
            leaf_tris += nd.b;
        }
        else if (nd.a >= n_nodes || nd.b >= n_nodes || nd.a <= i || nd.b <= i)
        {
            return fail(RT_E_FORMAT, "inner node child index out of range (the .bvh layout is DFS pre-order)");
        }
    }
    for (uint64_t i = 0; i < (uint64_t)n_tris; i++)
    {
        for (int k = 0; k < 3; k++)
        {
            if (tris[i].v[k] >= n_verts) { return fail(RT_E_FORMAT, "triangle vertex index out of range"); }
        }
    }
    rt_bvh* b = new rt_bvh();
    cudaGetDevice(&b->device);
    cudaStream_t st = default_stream();
    auto bail = [&](int e) { free_bvh(b); return e; };
    if (b->nodes.ensure((size_t)n_nodes * sizeof(rt_bvh_node)) || b->tris.ensure((size_t)std::max<uint32_t>(n_tris, 1) * 12) ||
        b->verts.ensure((size_t)std::max<uint32_t>(n_verts, 1) * 24))
    {
        return bail(RT_E_CUDA);
    }
    if (cudaMemcpyAsync(b->nodes.p, nodes, (size_t)n_nodes * sizeof(rt_bvh_node), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (n_tris && cudaMemcpyAsync(b->tris.p, tris, (size_t)n_tris * 12, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
        (n_verts && cudaMemcpyAsync(b->verts.p, verts, (size_t)n_verts * 24, cudaMemcpyHostToDevice, st) != cudaSuccess))
    {
        return bail(fail(RT_E_CUDA, "upload failed"));
    }
    b->n_nodes = n_nodes;
    b->n_tris = n_tris;
    b->n_verts = n_verts;
    b->has_prim = false;
    b->trace_ww = prefer_while_while(leaf_tris, n_leaves);
    if (int e = make_traversal_layout(b, st)) { return bail(e); }
    *out = b;
    return RT_OK;
}

int rt_load_bvh(const char* path, rt_bvh** out)
{
    if (!out || !path) { return fail(RT_E_INVALID, "null argument"); }
    *out = nullptr;
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open())
    {
        std::fprintf(stderr, "Error : failed to open %s on loadBVH()\n", path);
        return fail(RT_E_IO, std::string("failed to open ") + path);
    }
    uint32_t hdr[4] = { 0, 0, 0, 0 };
    in.read(reinterpret_cast<char*>(hdr), 16);
    if (!in.good())
    {
        std::fprintf(stderr, "Error : failed to read header from %s on loadBVH()\n", path);
        return fail(RT_E_FORMAT, std::string("failed to read header from ") + path);
    }
    if (hdr[0] != 1u)
    {
        std::fprintf(stderr, "Error : version mismatch in %s (got %u, expected %u) on loadBVH()\n", path, hdr[0], 1u);
        return fail(RT_E_FORMAT, "version mismatch");
    }
    std::vector<rt_bvh_node> nodes(hdr[1]);
    std::vector<rt_triangle> tris(hdr[2]);
    std::vector<rt_vertex> verts(hdr[3]);
    in.read(reinterpret_cast<char*>(nodes.data()), (std::streamsize)nodes.size() * 48);
    in.read(reinterpret_cast<char*>(tris.data()), (std::streamsize)tris.size() * 12);
    in.read(reinterpret_cast<char*>(verts.data()), (std::streamsize)verts.size() * 24);
    if (!in.good())
    {
        std::fprintf(stderr, "Error : failed to read payload from %s on loadBVH()\n", path);
        return fail(RT_E_FORMAT, std::string("failed to read payload from ") + path);
    }
    int e = rt_bvh_from_arrays(nodes.data(), hdr[1], tris.data(), hdr[2], verts.data(), hdr[3], out);
    if (e) { return e; }
    std::fprintf(stdout, "BVH loaded: %s  (%u nodes, %u tris, %u verts)\n", path, hdr[1], hdr[2], hdr[3]);
    return RT_OK;
}

int rt_bvh_trace_loop(rt_bvh* b, int form)
{
    if (!b) { return fail(RT_E_NOT_LOADED, "BVH not loaded"); }
    if (form < -1 || form > 2) { return fail(RT_E_INVALID, "form must be -1, 0, 1 or 2"); }
    if (form == 2)
    {
        if (int e = require_device()) { return e; }
        if (int e = make_wide_layout(b, default_stream())) { return e; }
        b->trace_wide = true;
        return RT_OK;
    }
    b->trace_wide = false;
    if (form == -1)
    {
        uint32_t leaves = b->stats[4];
        if (leaves == 0)  // a loaded tree: count its leaves
        {
            std::vector<rt_bvh_node> nodes(b->n_nodes);
            RT_CUDA(cudaMemcpy(nodes.data(), b->nodes.p, nodes.size() * sizeof(rt_bvh_node), cudaMemcpyDeviceToHost));
            for (const rt_bvh_node& nd : nodes) { leaves += nd.is_leaf ? 1u : 0u; }
        }
        b->trace_ww = prefer_while_while(b->n_tris, leaves);
    }
    else { b->trace_ww = form == 1; }
    return RT_OK;
}

int rt_bvh_counts(const rt_bvh* b, uint32_t* c3)
{
    if (!b || !c3) { return fail(RT_E_INVALID, "null argument"); }
    c3[0] = b->n_nodes; c3[1] = b->n_tris; c3[2] = b->n_verts;
    return RT_OK;
}

int rt_bvh_download(const rt_bvh* b, rt_bvh_node* nodes, rt_triangle* tris, rt_vertex* verts)
{
    if (!b) { return fail(RT_E_INVALID, "null handle"); }
    cudaStream_t st = default_stream();
    if (nodes) { RT_CUDA(cudaMemcpyAsync(nodes, b->nodes.p, (size_t)b->n_nodes * 48, cudaMemcpyDeviceToHost, st)); }
    if (tris && b->n_tris) { RT_CUDA(cudaMemcpyAsync(tris, b->tris.p, (size_t)b->n_tris * 12, cudaMemcpyDeviceToHost, st)); }
    if (verts && b->n_verts) { RT_CUDA(cudaMemcpyAsync(verts, b->verts.p, (size_t)b->n_verts * 24, cudaMemcpyDeviceToHost, st)); }
    RT_CUDA(cudaStreamSynchronize(st));
    return RT_OK;
}

int rt_bvh_wide_download(const rt_bvh* b, void* out, uint32_t* n_wide)
{
    if (!b || !n_wide) { return fail(RT_E_INVALID, "null argument"); }
    if (!b->trace_wide) { return fail(RT_E_INVALID, "the handle has no wide layout (rt_bvh_trace_loop form 2)"); }
    *n_wide = b->n_wide;
    if (out && b->n_wide) { RT_CUDA(cudaMemcpy(out, b->wnodes.p, (size_t)b->n_wide * sizeof(rt_wnode), cudaMemcpyDeviceToHost)); }
    return RT_OK;
}

int rt_bvh_download_async(const rt_bvh* b, rt_bvh_node* nodes, rt_triangle* tris, rt_vertex* verts, void* stream)
{
    if (!b) { return fail(RT_E_INVALID, "null handle"); }
    cudaStream_t st = pick(stream);
    if (nodes) { RT_CUDA(cudaMemcpyAsync(nodes, b->nodes.p, (size_t)b->n_nodes * 48, cudaMemcpyDeviceToHost, st)); }
    if (tris && b->n_tris) { RT_CUDA(cudaMemcpyAsync(tris, b->tris.p, (size_t)b->n_tris * 12, cudaMemcpyDeviceToHost, st)); }
    if (verts && b->n_verts) { RT_CUDA(cudaMemcpyAsync(verts, b->verts.p, (size_t)b->n_verts * 24, cudaMemcpyDeviceToHost, st)); }
    return RT_OK;
}

int rt_bvh_prim_ids(const rt_bvh* b, uint32_t* out, int where)
{
    if (!b || !out) { return fail(RT_E_INVALID, "null argument"); }
    if (!b->has_prim) { return fail(RT_E_INVALID, "this BVH was loaded from .bvh data; original triangle ids are unknown"); }
    cudaStream_t st = default_stream();
    RT_CUDA(cudaMemcpyAsync(out, b->prim.p, (size_t)b->n_tris * 4,
                            where == RT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    return RT_OK;
}

int rt_bvh_stats(const rt_bvh* b, uint32_t* s8)
{
    if (!b || !s8) { return fail(RT_E_INVALID, "null argument"); }
    std::memcpy(s8, b->stats, sizeof(b->stats));
    return RT_OK;
}

void rt_bvh_free(rt_bvh* b) { free_bvh(b); }

int rt_bvh_profile(rt_bvh* b, int enable)
{
    if (!b) { return fail(RT_E_INVALID, "null handle"); }
    if (enable)
    {
        for (cudaEvent_t& e : b->ev)
        {
            if (!e) { RT_CUDA(cudaEventCreate(&e)); }
        }
    }
    b->prof = enable != 0;
    return RT_OK;
}

int rt_bvh_stage_ms(const rt_bvh* b, float* ms8)
{
    if (!b || !ms8) { return fail(RT_E_INVALID, "null argument"); }
    std::memcpy(ms8, b->stage_ms, sizeof(b->stage_ms));
    return RT_OK;
}

int rt_write_bvh(const rt_bvh* b, const char* path)
{
    if (!b || !path) { return fail(RT_E_INVALID, "null argument"); }
    std::vector<rt_bvh_node> nodes(b->n_nodes);
    std::vector<rt_triangle> tris(b->n_tris);
    std::vector<rt_vertex> verts(b->n_verts);
    if (int e = rt_bvh_download(b, nodes.data(), tris.data(), verts.data())) { return e; }
    std::ofstream out(path, std::ios::binary);
    if (!out.is_open())
    {
        std::fprintf(stderr, "Error : failed to open output file %s on writeBakedData()\n", path);
        return fail(RT_E_IO, std::string("failed to open ") + path);
    }
    const uint32_t hdr[4] = { 1u, b->n_nodes, b->n_tris, b->n_verts };
    out.write(reinterpret_cast<const char*>(hdr), 16);
    out.write(reinterpret_cast<const char*>(nodes.data()), (std::streamsize)nodes.size() * 48);
    out.write(reinterpret_cast<const char*>(tris.data()), (std::streamsize)tris.size() * 12);
    out.write(reinterpret_cast<const char*>(verts.data()), (std::streamsize)verts.size() * 24);
    if (!out.good())
    {
        std::fprintf(stderr, "Error : write error for %s on writeBakedData()\n", path);
        return fail(RT_E_IO, std::string("write error for ") + path);
    }
    std::fprintf(stdout, "BVH baked: %s  (%u nodes, %u tris, %u verts)\n", path, b->n_nodes, b->n_tris, b->n_verts);
    return RT_OK;
}

int rt_trace(const rt_bvh* b, const rt_ray* rays, rt_hit* hits, uint64_t n, uint32_t flags, void* stream)
{
    if (!b) { return fail(RT_E_NOT_LOADED, "BVH not loaded on trace()"); }
    if (n && (!rays || !hits)) { return fail(RT_E_INVALID, "null rays/hits"); }
    rt_bvh* bm = const_cast<rt_bvh*>(b);
    if (bm->s.status.ensure(64)) { return RT_E_CUDA; }
    cudaStream_t st = pick(stream);
    uint32_t* status = bm->s.status.as<uint32_t>() + 8;
    RT_CUDA(cudaMemsetAsync(status, 0, 4, st));
    if (int e = rtb::trace(b, rays, hits, n, flags, st, status)) { return e; }
    uint32_t hs = 0;
    RT_CUDA(cudaMemcpyAsync(&hs, status, 4, cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    if (hs & ST_STACK) { return fail(RT_E_STACK, "a ray overflowed the 64-entry traversal stack"); }
    return RT_OK;
}

int rt_trace_host(const rt_bvh* b, const rt_ray* rays, rt_hit* hits, uint64_t n, uint32_t flags)
{
    if (!b) { return fail(RT_E_NOT_LOADED, "BVH not loaded on trace()"); }
    if (n == 0) { return RT_OK; }
    rt_bvh* bm = const_cast<rt_bvh*>(b);
    if (bm->trace_rays.ensure((size_t)n * 32) || bm->trace_hits.ensure((size_t)n * 32)) { return RT_E_CUDA; }
    cudaStream_t st = default_stream();
    RT_CUDA(cudaMemcpyAsync(bm->trace_rays.p, rays, (size_t)n * 32, cudaMemcpyHostToDevice, st));
    int e = rt_trace(b, bm->trace_rays.as<rt_ray>(), bm->trace_hits.as<rt_hit>(), n, flags, st);
    RT_CUDA(cudaMemcpyAsync(hits, bm->trace_hits.p, (size_t)n * 32, cudaMemcpyDeviceToHost, st));
    RT_CUDA(cudaStreamSynchronize(st));
    return e;
}

int rt_render(const rt_bvh* b, const rt_render_cfg* cfg, const rt_material* mats, uint32_t n_mats,
              const uint32_t* mat_of_tri, int mode, float* rgb, float* rgb2, void* stream)
{
    if (!b) { return fail(RT_E_NOT_LOADED, "BVH not loaded"); }
    if (!cfg || !rgb) { return fail(RT_E_INVALID, "null argument"); }
    if (cfg->width == 0 || cfg->height == 0 || cfg->spp == 0) { return fail(RT_E_INVALID, "empty image or spp = 0"); }
    if ((mats == nullptr) != (mat_of_tri == nullptr) || (mats && n_mats == 0))
    {
        return fail(RT_E_INVALID, "mats (n_mats > 0) and mat_of_tri go together");
    }
    const rt_shading sh{ mats, mat_of_tri, nullptr, nullptr, n_mats, 0u, 0u, 0u };
    return rtb::render(b, *cfg, sh, mode, rgb, rgb2, pick(stream));
}


int rt_render_ex(const rt_bvh* b, const rt_render_cfg* cfg, const rt_shading* shading, int mode, float* rgb, float* rgb2,
                 void* stream)
{
    rt_shading sh;
    if (int e = check_render_args(b, cfg, shading, &sh)) { return e; }
    if (!rgb) { return fail(RT_E_INVALID, "null argument"); }
    return rtb::render(b, *cfg, sh, mode, rgb, rgb2, pick(stream));
}

int rt_adjoint(const rt_bvh* b, const rt_render_cfg* cfg, const rt_shading* shading, const float* d_rgb, float* grad_albedo,
               float* grad_emission, void* stream)
{
    rt_shading sh;
    if (int e = check_render_args(b, cfg, shading, &sh)) { return e; }
    if (!d_rgb) { return fail(RT_E_INVALID, "null argument"); }
    if (!grad_albedo && !grad_emission) { return RT_OK; }
    return rtb::adjoint(b, *cfg, sh, d_rgb, grad_albedo, grad_emission, pick(stream));
}

int rt_render_host(const rt_bvh* b, const rt_render_cfg* cfg, const rt_shading* shading, int mode, float* rgb_host)
{
    rt_shading sh;
    if (int e = check_render_args(b, cfg, shading, &sh)) { return e; }
    if (!rgb_host) { return fail(RT_E_INVALID, "null argument"); }
    const size_t bytes = (size_t)cfg->width * cfg->height * 12;
    DevBuf out;
    if (out.ensure(bytes)) { return RT_E_CUDA; }
    cudaStream_t st = default_stream();
    int e = rtb::render(b, *cfg, sh, mode, out.as<float>(), nullptr, st);
    if (!e && (cudaMemcpyAsync(rgb_host, out.p, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
               cudaStreamSynchronize(st) != cudaSuccess))
    {
        e = fail(RT_E_CUDA, "render readback");
    }
    out.release();
    return e;
}

int rt_write_hdr(const char* path, const float* rgb, uint32_t w, uint32_t h, int flip_y)
{
    if (!path || !rgb || w == 0 || h == 0) { return fail(RT_E_INVALID, "bad argument"); }
    std::string err;
    int e;
    if (flip_y)
    {
        std::vector<float> fl((size_t)w * h * 3);
        for (uint32_t y = 0; y < h; y++)
        {
            std::memcpy(&fl[(size_t)(h - 1 - y) * w * 3], rgb + (size_t)y * w * 3, (size_t)w * 12);
        }
        e = hg::write_hdr(path, fl.data(), w, h, err);
    }
    else { e = hg::write_hdr(path, rgb, w, h, err); }
    return e ? fail(e, err) : RT_OK;
}

int rt_read_hdr(const char* path, float* rgb, uint32_t* w, uint32_t* h)
{
    if (!path || !w || !h) { return fail(RT_E_INVALID, "bad argument"); }
    std::vector<float> img;
    std::string err;
    uint32_t ww = 0, hh = 0;
    if (int e = hg::read_hdr(path, img, ww, hh, err)) { return fail(e, err); }
    *w = ww; *h = hh;
    if (rgb) { std::memcpy(rgb, img.data(), img.size() * 4); }
    return RT_OK;
}

int rt_scene_config(const char* scn_path, rt_render_cfg* cfg, char* ibl_path, uint32_t ibl_cap)
{
    if (!scn_path || !cfg) { return fail(RT_E_INVALID, "bad argument"); }
    const hg::SceneConfig sc = hg::parse_scene_config(scn_path);
    if (sc.width <= 0 || sc.height <= 0) { return fail(RT_E_FORMAT, "screen size must be positive"); }
    cfg->width = (uint32_t)sc.width;
    cfg->height = (uint32_t)sc.height;
    hg::store_camera(sc.camera, cfg);
    if (ibl_path && ibl_cap)
    {
        const size_t n = std::min<size_t>(sc.ibl_path.size(), ibl_cap - 1);
        std::memcpy(ibl_path, sc.ibl_path.data(), n);
        ibl_path[n] = 0;
    }
    return RT_OK;
}

// ---- cameras (src/main.cpp:43-66) ----
void rt_camera_lookat(const float pos[3], const float target[3], float fov_deg, rt_render_cfg* cfg)
{
    hg::Camera c = hg::camera_lookat(hg::V3(pos[0], pos[1], pos[2]), hg::V3(target[0], target[1], target[2]), fov_deg);
    hg::store_camera(c, cfg);
}

void rt_camera_quat(const float pos[3], const float q_wxyz[4], float focal, rt_render_cfg* cfg)
{
    hg::Camera c = hg::camera_quat(hg::V3(pos[0], pos[1], pos[2]),
                                   hg::quat_normalize(hg::Q(q_wxyz[1], q_wxyz[2], q_wxyz[3], q_wxyz[0])), focal);
    hg::store_camera(c, cfg);
}

// ---- host meshes and .scn ingestion ----
struct rt_mesh
{
    std::vector<rt_vertex> v;
    std::vector<rt_triangle> t;
};

rt_mesh* rt_mesh_create(void) { return new rt_mesh(); }
void rt_mesh_free(rt_mesh* m) { delete m; }

int rt_mesh_add_sphere(rt_mesh* m, float cx, float cy, float cz, float radius, int rings, int sectors)
{
    if (!m) { return fail(RT_E_INVALID, "null mesh"); }
    if (rings < 2 || sectors < 3) { return fail(RT_E_INVALID, "rings must be >= 2 and sectors >= 3"); }
    hg::add_sphere(m->v, m->t, hg::V3(cx, cy, cz), radius, rings, sectors);
    return RT_OK;
}

int rt_mesh_add_box(rt_mesh* m, float cx, float cy, float cz, float hx, float hy, float hz, float qx, float qy, float qz,
                    float qw)
{
    if (!m) { return fail(RT_E_INVALID, "null mesh"); }
    hg::add_box(m->v, m->t, hg::V3(cx, cy, cz), hg::V3(hx, hy, hz), hg::Q(qx, qy, qz, qw));
    return RT_OK;
}

int rt_mesh_read_scene(rt_mesh* m, const char* path)
{
    if (!m || !path) { return fail(RT_E_INVALID, "null argument"); }
    std::string err;
    const int e = hg::read_scene(path, m->v, m->t, err);
    if (e) { return fail(e, err); }
    return RT_OK;
}

int rt_mesh_counts(const rt_mesh* m, uint32_t* c2)
{
    if (!m || !c2) { return fail(RT_E_INVALID, "null argument"); }
    c2[0] = (uint32_t)m->v.size();
    c2[1] = (uint32_t)m->t.size();
    return RT_OK;
}
const rt_vertex* rt_mesh_vertices(const rt_mesh* m) { return m && !m->v.empty() ? m->v.data() : nullptr; }
const rt_triangle* rt_mesh_triangles(const rt_mesh* m) { return m && !m->t.empty() ? m->t.data() : nullptr; }

int rt_bake_scene(const char* scn_path, const char* out_bvh, const rt_build_cfg* cfg)
{
    if (!scn_path || !*scn_path)
    {
        std::fprintf(stderr, "Error : empty scene path on readScene()\n");
        return fail(RT_E_INVALID, "empty scene path");
    }
    rt_mesh m;
    if (int e = rt_mesh_read_scene(&m, scn_path)) { return e; }
    if (m.v.empty())
    {
        std::fprintf(stderr, "Error : no vertices loaded on initGeos()\n");
        return fail(RT_E_EMPTY, "no vertices loaded");
    }
    if (m.t.empty())
    {
        std::fprintf(stderr, "Error : no triangles loaded on initGeos()\n");
        return fail(RT_E_EMPTY, "no triangles loaded");
    }
    rt_bvh* b = nullptr;
    int e = rt_build(m.v.data(), (uint32_t)m.v.size(), m.t.data(), (uint32_t)m.t.size(), RT_HOST, cfg, nullptr, &b);
    if (e) { return e; }
    std::string out = out_bvh ? std::string(out_bvh) : hg::replace_extension(scn_path, ".bvh");
    e = rt_write_bvh(b, out.c_str());
    rt_bvh_free(b);
    return e;
}

} // extern "C"
