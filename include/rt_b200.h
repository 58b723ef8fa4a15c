/* rt_b200.h -- C ABI of librt_b200.so: BVH bake, load, trace and the path loop of the
 * minsuk0519/ray-tracer hot path, computed by hand-written CUDA kernels on one B200.
 *
 * Each entry point names the reference interface it replaces (path:line in the
 * reference project). Plain pointers and sizes only; no C++ or torch types. Every call
 * runs on the GPU; there is no CPU fallback: without a usable CUDA device the calls
 * return RT_E_CUDA.
 *
 * Memory: functions taking `const void* ..., int where` accept host (RT_HOST) or device
 * (RT_DEVICE) pointers. The library owns the buffers behind an rt_bvh handle; caller
 * pointers are borrowed for the duration of the call. A NULL stream means the library's
 * own stream for the current device. Calls on one rt_bvh handle are not thread-safe for
 * build/free; concurrent traces on a built handle are safe.
 */
#ifndef RT_B200_H
#define RT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference returns bool and prints "Error : ..." lines) ---- */
enum rt_status
{
    RT_OK          = 0,
    RT_E_INVALID   = 1,  /* bad argument */
    RT_E_IO        = 2,  /* file open/read/write failed (bvh_IO.cpp:247-250, bvh_traverse.cpp:185-189) */
    RT_E_FORMAT    = 3,  /* malformed .bvh / .scn content (bvh_traverse.cpp:199-210) */
    RT_E_CAPACITY  = 4,  /* a size limit of this library was exceeded */
    RT_E_STACK     = 5,  /* a traversal stack would have overflowed (the reference has no check) */
    RT_E_CUDA      = 6,  /* CUDA error, or no CUDA device */
    RT_E_TIMEOUT   = 7,  /* a bounded device-side wait gave up */
    RT_E_EMPTY     = 8,  /* no vertices / triangles (bvh_IO.cpp:74-83) */
    RT_E_INDEX     = 9,  /* triangle vertex index out of range (bvh_IO.cpp:88-99) */
    RT_E_NOT_LOADED= 10  /* trace before load (bvh_traverse.cpp:239-243) */
};

enum rt_mem { RT_HOST = 0, RT_DEVICE = 1 };

/* ---- data layouts shared with the .bvh v1 file (src/bvh/bvh.hpp:10-41) ---- */
typedef struct rt_vertex { float x, y, z, nx, ny, nz; } rt_vertex;           /* 24 bytes */
typedef struct rt_triangle { uint32_t v[3]; } rt_triangle;                  /* 12 bytes */
typedef struct rt_bvh_node                                                   /* 48 bytes */
{
    float    bmin[4];   /* AABB min; lane 3 is the reference's padding lane */
    float    bmax[4];
    uint8_t  is_leaf;
    uint8_t  pad0[3];
    uint32_t a;         /* inner: left child;  leaf: first triangle (beginTriIndex) */
    uint32_t b;         /* inner: right child; leaf: triangle count (triSize) */
    uint32_t pad1;
} rt_bvh_node;

/* bvh::Ray (src/bvh/bvh_traverse.hpp:10-16) as a 32-byte record */
typedef struct rt_ray { float o[3]; float tmin; float d[3]; float tmax; } rt_ray;
/* bvh::Hit (src/bvh/bvh_traverse.hpp:18-26) as a 32-byte record; flags bit 0 = hit */
typedef struct rt_hit { float t, u, v; uint32_t tri; float n[3]; uint32_t flags; } rt_hit;

#define RT_HIT_FLAG_HIT      1u
#define RT_HIT_FLAG_OVERFLOW 2u   /* traversal stack overflow: this ray's result is incomplete */

/* ---- build configuration: the reference's constexpr constants (src/bvh/bvh_defines.hpp:7-21)
 * as runtime values; rt_build_cfg_default() gives the reference's values. ---- */
typedef struct rt_build_cfg
{
    uint32_t lbvh_threshold; /* BVH_LBVH_THRESHOLD (64): nodes <= this many tris use binned SAH.
                                0 = pure Morton split ("LBVH"); 0xFFFFFFFF = SAH from the root */
    uint32_t max_leaf;       /* BVH_MAX_LEAF_SIZE (16) */
    uint32_t morton_bits;    /* MORTON_UNIT_BIT_SIZE: 21 (63-bit codes) or 10 (30-bit codes) */
    uint32_t bins_min;       /* BVH_SAH_BINS_MIN (8) */
    uint32_t bins_max;       /* BVH_SAH_BINS_MAX (32), at most 32 */
    float    c_trav;         /* BVH_C_TRAV (1.0) */
    float    c_isect;        /* BVH_C_ISECT (1.2) */
    float    centroid_eps;   /* BVH_CENTROID_EPS (1e-6) */
    float    spatial_eps;    /* BVH_SPATIAL_EPS (1e-6); a value above every node extent disables spatial splits */
    float    spatial_mult;   /* SPATIAL_TRICOUNT_MULTIPLIER (1.5) */
} rt_build_cfg;

void rt_build_cfg_default(rt_build_cfg* cfg);

typedef struct rt_bvh rt_bvh;

/* Builds a BVH from vertices and triangles, with the semantics of bvh::bakeBVH
 * (src/bvh/bvh_bake.cpp:180-194; the reference reads them from a .scn first):
 * normal renormalisation (bvh_IO.cpp:102-118), Morton codes and radix sort
 * (bvh_morton.cpp:40-159), the Morton-split / binned-SAH top-down build with spatial splits
 * (bvh_bfs.cpp:72-134, bvh_sah.cpp:24-460) and the DFS re-layout (bvh_bake.cpp:75-149).
 * The result lives on the device; `where` says where verts/tris point. */
int rt_build(const void* verts, uint32_t n_verts, const void* tris, uint32_t n_tris, int where,
             const rt_build_cfg* cfg, void* stream, rt_bvh** out);

/* Re-builds into an existing handle, reusing its device buffers when they are large
 * enough (no allocation in the steady state). */
int rt_rebuild(rt_bvh* bvh, const void* verts, uint32_t n_verts, const void* tris, uint32_t n_tris,
               int where, const rt_build_cfg* cfg, void* stream);

/* Loads a .bvh v1 file onto the device (bvh::loadBVH, src/bvh/bvh_traverse.cpp:182-235). */
int rt_load_bvh(const char* path, rt_bvh** out);
/* Writes the baked data as a .bvh v1 file (bvh::writeBakedData, src/bvh/bvh_IO.cpp:236-275). */
int rt_write_bvh(const rt_bvh* bvh, const char* path);
/* Builds from host arrays already in the .bvh layout (what loadBVH reads). */
int rt_bvh_from_arrays(const rt_bvh_node* nodes, uint32_t n_nodes, const rt_triangle* tris, uint32_t n_tris,
                       const rt_vertex* verts, uint32_t n_verts, rt_bvh** out);

/* counts3 = nodes, triangles, vertices (the .bvh header counts) */
int rt_bvh_counts(const rt_bvh* bvh, uint32_t* counts3);
/* Copies the baked arrays to host memory in the .bvh layout; any pointer may be NULL. */
int rt_bvh_download(const rt_bvh* bvh, rt_bvh_node* nodes, rt_triangle* tris, rt_vertex* verts);
/* The same copies queued on `stream` without waiting (no counterpart in the reference): a
 * caller baking a sequence of meshes downloads one bake while the next one uploads and builds
 * on another stream (PCIe moves both directions at once). Host buffers should be pinned; they
 * are written when the stream reaches the copies, so synchronise the stream before reading
 * them, and order any rebuild of the handle after the copies (same stream, or a sync). */
int rt_bvh_download_async(const rt_bvh* bvh, rt_bvh_node* nodes, rt_triangle* tris, rt_vertex* verts, void* stream);
/* Original triangle index of each baked triangle (n = triangle count); host or device out. */
int rt_bvh_prim_ids(const rt_bvh* bvh, uint32_t* out, int where);
/* stats8: spatial splits taken, spatial splits refused for capacity, SAH roots,
 * inner nodes, leaves, tree depth, build kernels launched, reserved */
int rt_bvh_stats(const rt_bvh* bvh, uint32_t* stats8);
/* Stage timing of later (re)builds on this handle: CUDA events recorded on the build's
 * stream between stages. ms8 = prep (normals, triangle boxes, Morton codes), radix sort,
 * topology (Karras tree, boundary, refit), binned SAH, emit (pre-order layout), traversal
 * layout, total, reserved. No counterpart in the reference (it has no instrumentation). */
int rt_bvh_profile(rt_bvh* bvh, int enable);
int rt_bvh_stage_ms(const rt_bvh* bvh, float* ms8);
void rt_bvh_free(rt_bvh* bvh);

/* ---- tracing: bvh::trace (src/bvh/bvh_traverse.cpp:237-246), batched ---- */
#define RT_TRACE_CLOSEST     0u  /* closest hit, reference-exact (Moller-Trumbore, back faces culled) */
#define RT_TRACE_ANY_HIT     1u  /* stop at the first accepted triangle */
#define RT_TRACE_WATERTIGHT  2u  /* watertight test (Woop, Benthin, Wald 2013), no culling */

/* Traversal loop form of a handle (no counterpart in the reference): 0 the one-loop form of
 * traverse() (bvh_traverse.cpp:91-178), 1 the while-while form (lanes of a warp walk inner
 * nodes, then test leaves, together), -1 the default: while-while when leaves hold 6 or more
 * triangles on average. Both visit the same nodes in the same order and give identical hits;
 * only their speed differs. 2: the 8-wide layout (128-byte nodes of up to eight children with
 * 8-bit quantised, conservative child boxes), built now and again after every rebuild of the
 * handle; rt_trace and the wavefront path tracer's trace stage use it (the plain per-pixel
 * renderer keeps the binary loop). It is not the reference's visiting
 * order: the closest hit's distance is the same, but on an exact tie in distance the reported
 * triangle may differ, and a triangle that the binary boxes cull -- one an exact box test
 * loses by rounding at a face, or, in trees with spatial splits, one outside a collapsed
 * intermediate node's box -- may be found. */
int rt_bvh_trace_loop(rt_bvh* bvh, int form);
/* The wide layout of a handle in form 2 (no counterpart in the reference): *n_wide nodes of
 * 128 bytes each -- {float p[3]; uint32 meta (x / y / z scale exponents in bits 0-23, inner-
 * child mask in 24-31); uint32 ref[8]; uint16 cnt[8]; uint8 qlo[3][8], qhi[3][8]; 16 bytes
 * zero} -- into out (host memory; out = NULL only reports the count). */
int rt_bvh_wide_download(const rt_bvh* bvh, void* out, uint32_t* n_wide);

/* Traces n rays; rays and hits are device pointers. Returns RT_E_STACK if any ray
 * overflowed its 64-entry stack (those hits carry RT_HIT_FLAG_OVERFLOW). */
int rt_trace(const rt_bvh* bvh, const rt_ray* rays, rt_hit* hits, uint64_t n, uint32_t flags, void* stream);
/* Same with host buffers: copies in, traces, copies out (what bvh::trace callers use). */
int rt_trace_host(const rt_bvh* bvh, const rt_ray* rays, rt_hit* hits, uint64_t n, uint32_t flags);

/* ---- the path loop: pathTrace + the pixel loop (src/main.cpp:145-204, 323-365) ---- */
typedef struct rt_material
{
    float    albedo[3];
    float    emission[3]; /* extension: area lights (the reference has none) */
    uint32_t kind;        /* 0 Lambertian (the reference's only material), 1 mirror (extension) */
    uint32_t pad;
} rt_material;

typedef struct rt_render_cfg
{
    uint32_t width, height, spp;
    uint32_t max_bounce;    /* bounce = 0..max_bounce inclusive (main.cpp:155; reference 8) */
    int32_t  rr_after;      /* Russian roulette when bounce > rr_after (reference 2); < 0 disables */
    uint32_t env_kind;      /* 0 sky gradient (main.cpp:167-173), 1 constant env_color,
                               2 the shading's equirectangular map (IBL::sample, main.cpp:107-117) */
    float    env_color[3];
    float    cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];
    float    tan_half_fov_y;
    uint32_t seed;          /* per-pixel counter RNG key */
    uint32_t sample_offset; /* first sample index (progressive accumulation) */
} rt_render_cfg;

/* Camera bases of the reference (src/main.cpp:43-66). */
void rt_camera_lookat(const float pos[3], const float target[3], float fov_deg, rt_render_cfg* cfg);
void rt_camera_quat(const float pos[3], const float q_wxyz[4], float focal, rt_render_cfg* cfg);

enum rt_render_mode { RT_RENDER_PLAIN = 0, RT_RENDER_WAVEFRONT = 1 };

/* Renders the image (rgb: W*H*3 float, row y = 0 at the bottom as in the reference's buffer
 * before its flip) as the mean over spp samples; rgb2 (optional) receives the mean of
 * squares for standard-error tests. mats/mat_of_tri (device pointers, optional): n_mats
 * materials and the material index per baked triangle (indices >= n_mats use the last
 * material); NULL gives the reference's albedo 0.8. rgb/rgb2 are device pointers. */
int rt_render(const rt_bvh* bvh, const rt_render_cfg* cfg, const rt_material* mats, uint32_t n_mats,
              const uint32_t* mat_of_tri, int mode, float* rgb, float* rgb2, void* stream);

/* Shading inputs of the path loop, all device pointers and all optional (extension: the
 * reference shades every surface with albedo 0.8 and has no emitters). */
typedef struct rt_shading
{
    const rt_material* mats;       /* n_mats materials */
    const uint32_t*    mat_of_tri; /* material per baked triangle (NULL: material 0; >= n_mats: the last) */
    const float*       tri_albedo; /* RGB albedo per baked triangle (n_tris*3), replacing the material's */
    const float*       env_map;    /* RGB equirectangular environment, env_h rows of env_w (env_kind 2) */
    uint32_t           n_mats;
    uint32_t           env_w, env_h;
    uint32_t           pad;
} rt_shading;

/* rt_render with the shading record (a NULL shading is the reference's albedo 0.8). */
int rt_render_ex(const rt_bvh* bvh, const rt_render_cfg* cfg, const rt_shading* shading, int mode, float* rgb,
                 float* rgb2, void* stream);

/* Adjoint of rt_render (no counterpart in the reference): with d_rgb = dLoss/d(rgb) (W*H*3,
 * device), accumulates (+=) dLoss/d(albedo used at each baked triangle) into grad_albedo
 * (n_tris*3) and dLoss/d(material emission) into grad_emission (n_mats*3); either may be
 * NULL. Path-replay backpropagation: each sample's path is traced once for its radiance and
 * once more, from the same counter-based random numbers, to distribute it; nothing per
 * sample is stored. Russian-roulette probabilities are treated as constants. Geometry is
 * held fixed. Pixels with d_rgb = 0 cost nothing. Gradient adds are FP32 atomics combined
 * per warp first, so the low bits of the sums vary from run to run. */
int rt_adjoint(const rt_bvh* bvh, const rt_render_cfg* cfg, const rt_shading* shading, const float* d_rgb,
               float* grad_albedo, float* grad_emission, void* stream);

/* ---- batched scenes (no counterpart in the reference: it bakes one scene per process) ----
 * Many independent scenes in one handle: one build (the launches of one rt_build over all
 * triangles, with the scene id above the Morton code bits of the sort key, so the radix tree
 * first separates the scenes) and one wavefront render over all their pixels. Each scene's
 * subtree, triangles and vertices are those rt_build gives for that scene alone, renumbered:
 * node indices + the scene's root node, triangle indices + its first triangle, vertex indices
 * + its vertex offset (rt_bvh_scenes). Spatial splits share one budget over the batch, so this
 * identity needs that budget not to bind (always so for the LBVH presets, where the binned SAH
 * only runs on ranges of identical Morton codes).
 *   verts: all scenes' vertices concatenated; tris: all scenes' triangles concatenated with
 *   vertex indices LOCAL to their scene; vert_offsets / tri_offsets: host arrays of
 *   n_scenes + 1 ascending offsets starting at 0 (every scene needs a triangle). Key bits
 *   3 * morton_bits + ceil(log2(n_scenes)) must not exceed 64: 30-bit codes (morton_bits 10)
 *   take up to 1024 scenes. */
int rt_build_batch(const void* verts, const uint32_t* vert_offsets, const void* tris, const uint32_t* tri_offsets,
                   uint32_t n_scenes, int where, const rt_build_cfg* cfg, void* stream, rt_bvh** out);
/* Re-builds a batch into an existing handle, reusing its device buffers. */
int rt_rebuild_batch(rt_bvh* bvh, const void* verts, const uint32_t* vert_offsets, const void* tris,
                     const uint32_t* tri_offsets, uint32_t n_scenes, int where, const rt_build_cfg* cfg, void* stream);
/* n_scenes (0 for a handle from rt_build) and, if info4 is given, 4 values per scene: root
 * node, node count of its subtree (contiguous from the root), first triangle, triangle count. */
int rt_bvh_scenes(const rt_bvh* bvh, uint32_t* n_scenes, uint32_t* info4);
/* Depth of the tree: inner nodes above the deepest leaf (a traversal stack of depth + 1
 * entries never overflows). */
int rt_bvh_depth(rt_bvh* bvh, uint32_t* depth);

/* Launch parameters of the wavefront path tracer. */
typedef struct rt_wavefront_params
{
    uint32_t trace_block;  /* threads per block of the persistent trace kernel (32..256) */
    uint32_t chunk_paths;  /* paths in flight per generate/extend/shade round */
    uint32_t stack_depth;  /* traversal stack entries: 64, or 32 when the tree is at most 31 deep */
    uint32_t shade_block;  /* threads per block of the shade kernel */
} rt_wavefront_params;

/* Renders every scene of a batched handle in one wavefront kernel set, replayed from a CUDA
 * graph captured on first use of a configuration. cfgs[s]: camera and seed of scene s;
 * size, spp, bounces, roulette, background and sample offset come from cfgs[0]. shading:
 * materials over all scenes, mat_of_tri / tri_albedo per baked triangle of the handle.
 * rgb (rgb2 optional): n_scenes * H * W * 3 floats, scene-major (device). Scene s gets the
 * samples that rt_render_ex of scene s alone with cfgs[s] takes (same random numbers).
 * params NULL: the handle's tuned parameters (rt_autotune_wavefront), else defaults. A
 * handle from rt_build renders as one scene. */
int rt_render_batch(rt_bvh* bvh, const rt_render_cfg* cfgs, uint32_t n_scenes, const rt_shading* shading,
                    const rt_wavefront_params* params, float* rgb, float* rgb2, void* stream);
/* Times each candidate parameter set (trace block 64/128/256, chunk 1-8 Mi paths, stack
 * 32/64 where the tree allows) on a short render of the batch -- enough samples per pixel for
 * 8 Mi paths, at most the configuration's own -- and keeps the fastest in the handle (and in
 * *best). */
int rt_autotune_wavefront(rt_bvh* bvh, const rt_render_cfg* cfgs, uint32_t n_scenes, const rt_shading* shading,
                          rt_wavefront_params* best, void* stream);

/* ---- allocation-free Morton order ----
 * No counterpart in the reference. For callers that may not allocate device memory while
 * they run: a renderer re-baking deforming geometry inside its frame loop, where a cudaMalloc
 * would synchronise the device and stall the frame, or a host application that owns a fixed
 * device-memory budget and forbids plugins from growing it. It computes the triangle order
 * the reference's sortTrisByMorton produces (src/bvh/bvh_morton.cpp:109-159; equal to the
 * baked triangle order of the LBVH presets on meshes without runs of identical codes) and
 * calls no cudaMalloc / cudaFree or allocating library routine: its scratch is a fixed
 * device array of about 3.8 MB inside this library, which every GPU that loads the library
 * holds until the process exits.
 *   verts, tris, perm_out: device pointers; perm_out receives n_tris original triangle
 *   indices in Morton order. At most RT_NOALLOC_MAX_TRIS triangles (larger meshes get
 *   RT_E_CAPACITY; use rt_build). The first call on a device looks up the scratch array's
 *   device address (cudaGetSymbolAddress); make that first call before any stream capture.
 *   Every call shares the one scratch array, so calls whose work overlaps on the GPU
 *   (different streams or threads at once) race and must be serialised by the caller. Each
 *   call reads the kernels' status word back and synchronises `stream` before returning, so
 *   perm_out is complete when it returns RT_OK. */
#define RT_NOALLOC_MAX_TRIS 65536u
int rt_morton_order_noalloc(const rt_vertex* verts, uint32_t n_verts, const rt_triangle* tris, uint32_t n_tris,
                            uint32_t morton_bits, uint32_t* perm_out, void* stream);

/* ---- scene ingestion (src/bvh/bvh_IO.cpp:125-234, src/bvh/bvh_geo.cpp) on the host ---- */
typedef struct rt_mesh rt_mesh;
rt_mesh* rt_mesh_create(void);
void     rt_mesh_free(rt_mesh* m);
/* addSphere (bvh_geo.cpp:22-112) / addBox (bvh_geo.cpp:114-192), appended */
int      rt_mesh_add_sphere(rt_mesh* m, float cx, float cy, float cz, float radius, int rings, int sectors);
int      rt_mesh_add_box(rt_mesh* m, float cx, float cy, float cz, float hx, float hy, float hz,
                         float qx, float qy, float qz, float qw);
/* The geometry lines of a .scn file (sphere / box / mesh), appended (readScene). */
int      rt_mesh_read_scene(rt_mesh* m, const char* scn_path);
int      rt_mesh_counts(const rt_mesh* m, uint32_t* counts2);
const rt_vertex*   rt_mesh_vertices(const rt_mesh* m);
const rt_triangle* rt_mesh_triangles(const rt_mesh* m);

/* bvh::bakeBVH: reads the .scn, builds on the GPU, writes the .bvh (the reference writes
 * "<scene without extension>.bvh"; out_bvh NULL keeps that rule). */
int rt_bake_scene(const char* scn_path, const char* out_bvh, const rt_build_cfg* cfg);

/* ---- images and scene settings (the reference's main, src/main.cpp:87-118, 207-386) ---- */
/* Writes rgb (w*h*3 floats, host) as a Radiance RGBE .hdr file (what stbi_write_hdr writes
 * for the reference); flip_y != 0 writes row h-1 first (the reference's image has y = 0 at the
 * bottom and flips before writing, main.cpp:368-376). */
int rt_write_hdr(const char* path, const float* rgb, uint32_t w, uint32_t h, int flip_y);
/* Reads a Radiance RGBE .hdr file (stbi_loadf for the IBL map, main.cpp:96-104): with rgb
 * NULL only *w and *h are set; otherwise rgb receives w*h*3 floats (file row order). */
int rt_read_hdr(const char* path, float* rgb, uint32_t* w, uint32_t* h);
/* The settings lines of a .scn file (parseSceneConfig, main.cpp:207-285): sets cfg->width,
 * height and the camera; copies the ibl path (empty if none) into ibl_path (ibl_cap bytes). */
int rt_scene_config(const char* scn_path, rt_render_cfg* cfg, char* ibl_path, uint32_t ibl_cap);
/* rt_render_ex into host memory (rgb_host: W*H*3 floats), for callers without device buffers. */
int rt_render_host(const rt_bvh* bvh, const rt_render_cfg* cfg, const rt_shading* shading, int mode, float* rgb_host);

/* ---- diagnostics ---- */
const char* rt_last_error(void);     /* thread-local text of the last failure */
const char* rt_version(void);
/* Number of this library's kernels launched so far in this process (all devices). */
uint64_t    rt_kernel_launches(void);
/* Number of device allocations (cudaMalloc) this library has made so far in this process (all
 * devices): handles grow their buffers on demand, so a steady-state rebuild adds none. */
uint64_t    rt_device_allocations(void);
int         rt_device_sync(void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_H */
