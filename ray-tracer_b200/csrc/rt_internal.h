// rt_internal.h -- internal declarations shared by the librt_b200 translation units.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rt_b200.h"

namespace rtb
{

// ---- errors ---------------------------------------------------------------------------
void set_error(const std::string& msg);
int  fail(int code, const std::string& msg);
// Wraps a CUDA call: on failure records the error text and returns RT_E_CUDA from the caller.
#define RT_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
        {                                                                                    \
            return ::rtb::fail(RT_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
        }                                                                                    \
    } while (0)

// A setting made once per device. Function attributes (the dynamic shared-memory limit of a
// kernel above 48 KB, for one) belong to the context of the device that was current when they
// were set, so a process driving several GPUs sets them on each. once(f) runs f the first time
// it is reached with a given current device (devices 64 and up: every time) and records the
// device when f returns RT_OK; two host threads may both run f for the same device, which is
// harmless for idempotent settings.
class PerDeviceOnce
{
    std::atomic<uint64_t> done_{ 0 };

public:
    template <typename F> int once(F&& f)
    {
        int dev = 0;
        RT_CUDA(cudaGetDevice(&dev));
        const bool tracked = dev >= 0 && dev < 64;
        if (tracked && ((done_.load(std::memory_order_acquire) >> dev) & 1ull)) { return RT_OK; }
        if (int e = f()) { return e; }
        if (tracked) { done_.fetch_or(1ull << dev, std::memory_order_acq_rel); }
        return RT_OK;
    }
};

// Counts this library's kernel launches (rt_kernel_launches()).
void count_launch(uint64_t n = 1);
// Counts this library's device allocations (rt_device_allocations()).
void count_alloc();
uint64_t thread_launches();  // launches counted by the calling host thread
// Checks the last launch; returns RT_OK or RT_E_CUDA.
int  check_launch(const char* what);

// Device status word bits, written by kernels instead of trapping.
enum : uint32_t
{
    ST_INDEX    = 1u << 0,  // triangle vertex index out of range
    ST_TIMEOUT  = 1u << 1,  // a bounded spin-wait gave up
    ST_CAPACITY = 1u << 2,  // an internal capacity was exceeded
    ST_STACK    = 1u << 3,  // traversal stack overflow
};

// ---- device memory ---------------------------------------------------------------------
// Grows on demand and is reused between builds (cudaMalloc only when a larger size is needed).
struct DevBuf
{
    void*  p     = nullptr;
    size_t bytes = 0;
    int    ensure(size_t n);
    void   release();
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Per-device default stream and the current device's properties.
cudaStream_t default_stream();
int          device_sm_count();

// ---- radix sort (radix_sort.cu) ---------------------------------------------------------
// Stable sort of `n` keys with uint32 values by their low `key_bits` bits: onesweep LSD
// passes, or up to 2^21 keys an MSD pass on the top digit and a per-bucket sort in shared
// memory (radix_sort_pairs). Histograms of all digit passes must already be in `hist` (256
// counters per pass, built by the producer of the keys). keys/vals are ping-ponged: the
// sorted result ends in the buffer returned through *keys_out / *vals_out.
struct SortScratch
{
    DevBuf keys_alt, vals_alt, lookback, tile_counters;
};
// hist: the counts of every LSD digit (256 per pass); msd_hist (optional): the counts of the
// key's top digit, bits key_bits-8 .. key_bits-1, which enables the MSD + per-bucket path.
template <typename K>
int radix_sort_pairs(K* keys, uint32_t* vals, bool vals_identity, uint32_t n, int key_bits,
                     const uint32_t* hist, const uint32_t* msd_hist, SortScratch& s, uint32_t* status,
                     cudaStream_t st, K** keys_out, uint32_t** vals_out, bool scratch_zeroed = false,
                     uint32_t* msd_only_flag = nullptr, uint32_t* msd_table = nullptr,
                     const uint32_t** table_flag = nullptr);
// (scratch_zeroed: the caller zeroed s.lookback's first sort_lookback_words(n, passes) words
// and s.tile_counters' first 64 words, so the sort skips its memsets. msd_only_flag: when the
// MSD path applies, launch no LSD fallback and write its flag there instead -- nonzero means a
// bucket overflowed and the keys are NOT sorted: the caller must sort again without it.
// msd_table: where the MSD path writes the bucket table of the sorted keys' top 16 bits
// (2^16 + 1 words: tab[v] = the first index whose top 16 bits are >= v) when its sub-buckets
// are exactly those values (more than 16 key bits); *table_flag then points at the device word
// that is nonzero when that path did not finish (a bucket overflowed: no table), and is
// nullptr when no table is written.)
// The same sort on caller-provided scratch; allocates nothing.
template <typename K>
int radix_sort_pairs_raw(K* keys, uint32_t* vals, uint32_t n, int key_bits, const uint32_t* hist, K* keys_alt,
                         uint32_t* vals_alt, uint32_t* lookback, uint32_t* tile_counters, uint32_t* status,
                         cudaStream_t st, K** keys_out, uint32_t** vals_out);
// Number of 8-bit digit passes for a key width.
inline int sort_passes(int key_bits) { return (key_bits + 7) / 8; }
// Look-back words (passes x tiles x 256) a sort of n keys uses.
size_t sort_lookback_words(uint32_t n, int passes);
// Keys per tile of the onesweep passes up to RS_SMALL_MAX_KEYS keys (256 threads x 16 keys),
// the shape radix_sort_pairs_raw always uses; above that size the tile is half as large.
constexpr uint32_t RS_SMALL_TILE_KEYS = 4096;
constexpr uint32_t RS_SMALL_MAX_KEYS = 1u << 21;
// Look-back words of a radix_sort_pairs_raw sort of n keys (n <= RS_SMALL_MAX_KEYS).
constexpr size_t sort_raw_lookback_words(uint32_t n, int passes)
{
    return (size_t)passes * ((n + RS_SMALL_TILE_KEYS - 1) / RS_SMALL_TILE_KEYS) * 256;
}

// Device-wide exclusive scan of uint32 (scan.cu is in build.cu); returns total through *d_total.
struct ScanScratch { DevBuf partials; };
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* d_total, ScanScratch& s,
                       cudaStream_t st);

} // namespace rtb

// ---- the BVH handle ----------------------------------------------------------------------

// Traversal node (64 bytes): the boxes of both children next to their references, so one
// node fetch (four 128-bit loads) tests both children. cnt = 0x80000000 | triangle count for a
// leaf child (ref = first triangle), 0 for an inner child (ref = node index).
struct rt_gnode
{
    float4 a;  // l.min.x l.min.y l.min.z l.max.x
    float4 b;  // l.max.y l.max.z r.min.x r.min.y
    float4 c;  // r.min.z r.max.x r.max.y r.max.z
    uint4  d;  // l.ref   r.ref   l.cnt   r.cnt
};

// 128-byte node of the 8-wide traversal layout (wide.cu): child c's box is
// [p + qlo * 2^e, p + qhi * 2^e] per axis, conservative.
struct rt_wnode
{
    float    p[3];       // quantisation origin
    uint32_t meta;       // bits 0-7 / 8-15 / 16-23: biased exponents of the x / y / z scales; 24-31: inner-child mask
    uint32_t ref[8];     // inner child: wide node index; leaf child: first triangle
    uint16_t cnt[8];     // leaf child: triangle count; inner child: 1; 0: an empty slot
    uint8_t  qlo[3][8];  // lower planes, per axis and child
    uint8_t  qhi[3][8];  // upper planes
    uint32_t pad[4];
};
static_assert(sizeof(rt_wnode) == 128, "rt_wnode is one 128-byte line");

struct BuildScratch
{
    rtb::DevBuf tri_lo, tri_hi, tri_cz, keys, vals, hist, scene, status;
    rtb::SortScratch sort;
    rtb::ScanScratch scan;
    rtb::DevBuf knode;         // Karras inner nodes
    rtb::DevBuf parent;        // parent of every Karras node (2N-1)
    rtb::DevBuf kbox;          // boxes of kept Karras nodes (2N-1) x 6 floats
    rtb::DevBuf lvbox;         // box hierarchy over the sorted keys (blocks of 16^k keys)
    rtb::DevBuf kflag, ktab;   // per Karras node kept / Morton-split flags; bucket table of the sorted keys
    rtb::DevBuf tpin;          // per input triangle: positions and vertex indices (48-byte records)
    rtb::DevBuf rank;          // left-chain rank of kept Karras nodes
    rtb::DevBuf bnd;           // boundary node id per start key (or ~0)
    rtb::DevBuf wnode, wtri;   // per start key weights (nodes, triangles)
    rtb::DevBuf snode, stri;   // their exclusive scans
    rtb::DevBuf counters;      // small device counters
    rtb::DevBuf sah_roots;     // SAH subtree roots
    // SAH builder state
    rtb::DevBuf sah_refs_a, sah_refs_b, sah_tmp, sah_pos, sah_lvl_a, sah_lvl_b, sah_dec, sah_out, sah_leaf_refs,
        sah_scan_in, sah_scan_out, sah_node_ids, sah_roots_lvl;
    rtb::DevBuf sah_root_ord;       // the roots' sort keys, order, counts and their scan, per-depth runs
    rtb::SortScratch root_sort;     // (their sort's own scratch: the bake's sorted keys stay live)
    rtb::DevBuf in_verts, in_tris;  // staging for host geometry
    rtb::DevBuf gtris;              // batched build: triangles with concatenated-array vertex indices
    rtb::DevBuf batch_off;          // batched build: triangle and vertex offsets per scene
    rtb::DevBuf sah_budget;         // spatial-split budget per scene: used, cap
    rtb::DevBuf sah_wide;           // SAH nodes evaluated by many blocks: bins, list, block offsets
    rtb::DevBuf sah_tmp2, sah_pos2; // their partitions' second buffer and satisfying-right positions
    rtb::DevBuf wide_flag, wide_par;  // wide layout: which binary nodes are wide nodes; parents
};

struct rt_bvh
{
    int          device = 0;
    rtb::DevBuf  nodes, tris, verts, prim, gnodes, tripos;
    uint32_t     n_nodes = 0, n_tris = 0, n_verts = 0;
    bool         has_prim = false;
    rtb::DevBuf  rootbuf;                   // traversal entry record (box and reference of node 0)
    // batched builds: per scene {root node, node count, first triangle, triangle count} and the
    // traversal entry record of each scene's root
    uint32_t     n_scenes = 0;
    rtb::DevBuf  scene_info, scene_roots;
    std::vector<uint32_t> scene_info_host;
    uint32_t     depth = 0;                 // tree depth (computed on demand; 0 = unknown)
    bool         trace_ww = true;           // traversal loop form: while-while for large leaves
    bool         trace_wide = false;        // traverse the 8-wide layout (rebuilt after every rebuild)
    rtb::DevBuf  wnodes, wid;               // wide layout and the wide index of each binary node
    uint32_t     n_wide = 0;
    uint32_t     stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    BuildScratch s;
    rtb::DevBuf  trace_status, trace_rays, trace_hits;
    rtb::DevBuf  wf_rays[2], wf_state[2], wf_hits, wf_acc, wf_ctr;  // wavefront path tracer
    rtb::DevBuf  wf_scene[2], wf_cams;      // scene of each queued ray; per-scene cameras
    cudaStream_t wf_stream = nullptr;       // the graph replays here, fenced by wf_ev
    cudaEvent_t  wf_ev[2] = { nullptr, nullptr };
    // an LBVH bake's launch sequence, captured on the second call with the same key (sizes,
    // settings, inputs, buffer addresses) and replayed on bake_stream (fenced with the caller's
    // stream by bake_ev); its key, and the key the last plain bake left
    cudaGraphExec_t bake_exec = nullptr;
    std::vector<unsigned char> bake_key, bake_seen;
    uint64_t     bake_kernels = 0;
    void*        bake_skeys = nullptr;      // where the captured sort left keys and permutation
    uint32_t*    bake_perm = nullptr;
    cudaStream_t bake_stream = nullptr;
    cudaEvent_t  bake_ev[2] = { nullptr, nullptr };
    cudaGraphExec_t wf_exec = nullptr;      // the captured launch sequence and its key
    std::vector<unsigned char> wf_key;
    uint32_t     wf_kernels = 0;
    rt_wavefront_params wf_tuned = { 0, 0, 0, 0 };
    bool         wf_tuned_valid = false;
    // stage timing (rt_bvh_profile): events at the stage boundaries of a build
    bool         prof = false;
    cudaEvent_t  ev[8] = { nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr };
    float        stage_ms[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
};

namespace rtb
{
// The traversal loop form for a tree with n_tris triangles in n_leaves leaves: the
// while-while loop pays off when leaves hold 6 or more triangles on average.
inline bool prefer_while_while(uint64_t n_tris, uint64_t n_leaves) { return n_tris >= 6 * n_leaves; }

// Records the boundary event of stage `i` (0 = build start) when profiling is on.
inline void prof_mark(rt_bvh* b, int i, cudaStream_t st)
{
    if (b->prof) { cudaEventRecord(b->ev[i], st); }
}
} // namespace rtb

namespace rtb
{
// build.cu
int build_bvh(rt_bvh* b, const rt_vertex* d_verts, uint32_t n_verts, const rt_triangle* d_tris, uint32_t n_tris,
              const rt_build_cfg& cfg, cudaStream_t st);
// n_scenes scenes in one build; d_toff / d_voff: n_scenes + 1 triangle / vertex offsets on the
// device, triangle vertex indices local to their scene.
int build_bvh_batch(rt_bvh* b, const rt_vertex* d_verts, uint32_t n_verts, const rt_triangle* d_tris, uint32_t n_tris,
                    const rt_build_cfg& cfg, cudaStream_t st, uint32_t n_scenes, const uint32_t* d_toff,
                    const uint32_t* d_voff, const uint32_t* h_toff);
// traverse.cu: the traversal entry record of every scene root of a batched build
int launch_scene_roots(rt_bvh* b, uint32_t n_scenes, const uint32_t* d_counts, uint32_t* status, cudaStream_t st);
// wide.cu: the 8-wide traversal layout of the handle's tree (synchronises the stream)
int make_wide_layout(rt_bvh* b, cudaStream_t st);
// traverse.cu: depth of the tree (levels of inner nodes above the deepest leaf), cached in b->depth
int tree_depth(rt_bvh* b, cudaStream_t st, uint32_t* depth);
// traverse.cu: (re)creates the traversal layout from the .bvh-layout arrays on the device
int make_traversal_layout(rt_bvh* b, cudaStream_t st);
// The same kernels without a host synchronisation: grids sized for max_nodes / max_tris,
// d_counts (optional) = {nodes, triangles} on the device; structure violations set *vstatus;
// tripos_ready / gnodes_ready: the triangle position records / the traversal nodes and the
// entry record were written by the build already.
int launch_traversal_layout(rt_bvh* b, cudaStream_t st, uint32_t max_nodes, uint32_t max_tris, const uint32_t* d_counts,
                            uint32_t* vstatus, bool tripos_ready = false, bool gnodes_ready = false);
int trace(const rt_bvh* b, const rt_ray* d_rays, rt_hit* d_hits, uint64_t n, uint32_t flags, cudaStream_t st,
          uint32_t* d_status);
// Launch options of the persistent trace kernel: block size (0: default), stack entries
// (32 or 64; 32 only for closest hits), and per-ray subtree roots (roots[rscene[i]], device).
struct TraceRoot;
struct TraceLaunch
{
    int              block = 0;
    int              stack = 64;
    const TraceRoot* roots = nullptr;
    const uint32_t*  rscene = nullptr;
};
// Launches the persistent trace kernel; n_dev (optional) holds the ray count on the device.
// d_counter must be zero on entry.
int trace_launch(const rt_bvh* b, const void* d_rays, void* d_hits, uint64_t n, const uint32_t* n_dev, uint32_t flags,
                 cudaStream_t st, uint32_t* d_status, unsigned long long* d_counter, const TraceLaunch& opt);
// render.cu
int render(const rt_bvh* b, const rt_render_cfg& cfg, const rt_shading& sh, int mode, float* rgb, float* rgb2,
           cudaStream_t st);
int adjoint(const rt_bvh* b, const rt_render_cfg& cfg, const rt_shading& sh, const float* d_rgb, float* g_alb, float* g_em,
            cudaStream_t st);
int render_batch(rt_bvh* b, const rt_render_cfg* cfgs, uint32_t n_scenes, const rt_shading& sh,
                 const rt_wavefront_params* params, float* rgb, float* rgb2, cudaStream_t st);
int autotune_wavefront(rt_bvh* b, const rt_render_cfg* cfgs, uint32_t n_scenes, const rt_shading& sh,
                       rt_wavefront_params* best, float* scratch_rgb, cudaStream_t st);
} // namespace rtb
