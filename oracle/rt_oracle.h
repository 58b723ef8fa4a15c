/* rt_oracle.h -- CPU restatement of the reference path tracer's hot path (TEST ORACLE).
 *
 * This is test infrastructure, not product code. Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may load liboracle.so, and only as the checker. The
 * product library (librt_b200.so) never links or calls it.
 *
 * Each function restates the reference algorithm with the same float operation order
 * (x86-64 SSE, no FMA contraction), citing the reference file:line it follows.
 * Parity is pinned against the reference itself (oracle/_ref, built from its sources)
 * and against the known answers of its tests/test_traverse.cpp and tests/test_aabb.cpp.
 */
#ifndef RT_ORACLE_H
#define RT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Build parameters: the reference's compile-time constants (src/bvh/bvh_defines.hpp:7-21)
 * as runtime values. */
typedef struct orc_cfg
{
    uint32_t lbvh_threshold; /* BVH_LBVH_THRESHOLD: nodes with <= this many tris use SAH */
    uint32_t max_leaf;       /* BVH_MAX_LEAF_SIZE */
    uint32_t morton_bits;    /* MORTON_UNIT_BIT_SIZE: 21 (63-bit codes) or 10 (30-bit) */
    uint32_t bins_min;       /* BVH_SAH_BINS_MIN */
    uint32_t bins_max;       /* BVH_SAH_BINS_MAX (<= 64) */
    float    c_trav;         /* BVH_C_TRAV */
    float    c_isect;        /* BVH_C_ISECT */
    float    centroid_eps;   /* BVH_CENTROID_EPS */
    float    spatial_eps;    /* BVH_SPATIAL_EPS (a huge value turns spatial splits off) */
    float    spatial_mult;   /* SPATIAL_TRICOUNT_MULTIPLIER */
} orc_cfg;

/* .bvh v1 node record, 48 bytes (src/bvh/bvh.hpp:16-30 with AABB of two 16-byte lanes). */
typedef struct orc_node
{
    float    bmin[4];
    float    bmax[4];
    uint8_t  is_leaf;
    uint8_t  pad0[3];
    uint32_t a; /* left child, or first triangle of a leaf */
    uint32_t b; /* right child, or triangle count of a leaf */
    uint32_t pad1;
} orc_node;

typedef struct orc_bvh orc_bvh;

void orc_cfg_default(orc_cfg* cfg);

/* Morton codes in input order, the stable radix-sorted permutation and the scene box
 * (src/bvh/bvh_morton.cpp:40-159). */
int orc_morton(const float* verts6, uint32_t V, const uint32_t* tris3, uint32_t N,
               const orc_cfg* cfg, uint64_t* codes, uint32_t* sorted, float* scene6);

/* Full bake (src/bvh/bvh_bake.cpp:180-194) of injected geometry. Returns NULL on the
 * reference's error paths (empty geometry, out-of-range vertex index). */
orc_bvh* orc_build(const float* verts6, uint32_t V, const uint32_t* tris3, uint32_t N,
                   const orc_cfg* cfg);
/* counts3 = nodes, triangles, vertices of the baked result */
void orc_counts(const orc_bvh* b, uint32_t* counts3);
/* stats4 = spatial splits taken, spatial splits refused for capacity, SAH leaves, Morton splits */
void orc_stats(const orc_bvh* b, uint32_t* stats4);
void orc_get(const orc_bvh* b, orc_node* nodes, uint32_t* tris3, float* verts6);
/* Wrap caller arrays (e.g. a .bvh file read by the test) as a BVH for tracing. Copies. */
orc_bvh* orc_from_arrays(const orc_node* nodes, uint32_t n_nodes, const uint32_t* tris3,
                         uint32_t n_tris, const float* verts6, uint32_t n_verts);
void orc_free(orc_bvh* b);

/* initGeos normal renormalisation (src/bvh/bvh_IO.cpp:102-118), in place. */
void orc_normalize_normals(float* verts6, uint32_t V);

/* clipTriangleToAABB (src/bvh/AABB.cpp:86-171). */
void orc_clip_triangle(const float* v9, const float* box6, float* out6);

/* Trace flags */
#define ORC_TRACE_ANY_HIT 1u /* stop at the first accepted triangle */
#define ORC_TRACE_WATERTIGHT 2u /* watertight triangle test (Woop, Benthin, Wald 2013), both faces */

/* Closest-hit trace of n rays (o.xyz, tmin, d.xyz, tmax) through a BVH
 * (src/bvh/bvh_traverse.cpp:22-178). out6 = t,u,v,n.xyz; counters (optional, 3 per
 * ray) = nodes popped, triangles tested, max stack depth. Returns the number of rays
 * whose 64-entry stack would have overflowed (those rays are cut short). */
uint64_t orc_trace(const orc_bvh* b, const float* rays8, uint64_t n, uint32_t flags,
                   float* out6, uint32_t* tri, uint8_t* hit, uint32_t* counters, int nthreads);

/* ---- path loop (src/main.cpp:69-204) with the scene extensions the benchmark configs need ---- */

typedef struct orc_material
{
    float    albedo[3];
    float    emission[3];
    uint32_t kind; /* 0 Lambertian, 1 mirror */
    uint32_t pad;
} orc_material;

typedef struct orc_render_cfg
{
    uint32_t width, height, spp;
    uint32_t max_bounce;   /* loop runs bounce = 0..max_bounce (src/main.cpp:155) */
    int32_t  rr_after;     /* Russian roulette when bounce > rr_after; < 0 disables */
    uint32_t env_kind;     /* 0 sky gradient (src/main.cpp:167-173), 1 constant env_color, 2 map (main.cpp:107-117) */
    float    env_color[3];
    float    cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];
    float    tan_half_fov_y;
    uint32_t seed;
    uint32_t sample_offset; /* first sample index (for progressive accumulation) */
} orc_render_cfg;

/* Render rows [row0, row1) into rgb (W*H*3, mean over spp) and optionally rgb2 (mean of
 * squares). mat_of_tri maps the BVH's triangle order to a material index (NULL: albedo
 * 0.8 everywhere, the reference material). */
void orc_render(const orc_bvh* b, const orc_render_cfg* cfg, const orc_material* mats,
                const uint32_t* mat_of_tri, uint32_t row0, uint32_t row1, float* rgb,
                float* rgb2, int nthreads);

/* orc_render with a material count (indices >= n_mats use the last material), an optional
 * RGB albedo per baked triangle (tri_albedo, n_tris*3) replacing the material's, and the
 * equirectangular environment map of env_kind 2 (env_h rows of env_w RGB texels). */
void orc_render_ex(const orc_bvh* b, const orc_render_cfg* cfg, const orc_material* mats, uint32_t n_mats,
                   const uint32_t* mat_of_tri, const float* tri_albedo, const float* env_map, uint32_t env_w,
                   uint32_t env_h, uint32_t row0, uint32_t row1, float* rgb, float* rgb2, int nthreads);

/* orc_render_ex (without rgb2) that also counts, over every sample of rows [row0, row1), the
 * segments traced (trace calls of pathTrace), the BVH nodes popped and the triangles tested:
 * counts3 = those three totals, for the path loop's algorithmic traversal work. */
void orc_render_stats(const orc_bvh* b, const orc_render_cfg* cfg, const orc_material* mats, uint32_t n_mats,
                      const uint32_t* mat_of_tri, const float* tri_albedo, const float* env_map, uint32_t env_w,
                      uint32_t env_h, uint32_t row0, uint32_t row1, float* rgb, uint64_t* counts3, int nthreads);

/* Gradients of sum(d_rgb * image) with respect to the per-triangle albedo (grad_albedo,
 * n_tris*3, used when tri_albedo is given or materials supply the albedo) and the material
 * emission (grad_emission, n_mats*3), accumulated in double precision into the arrays.
 * Each sample's path is traced once with the same arithmetic as orc_render_ex, stored
 * (at most 64 vertices), and differentiated by explicit products over its vertices. */
void orc_adjoint(const orc_bvh* b, const orc_render_cfg* cfg, const orc_material* mats, uint32_t n_mats,
                 const uint32_t* mat_of_tri, const float* tri_albedo, const float* d_rgb, double* grad_albedo,
                 double* grad_emission, int nthreads);

/* The pieces of the path loop, for bit-level checks against the reference's own functions:
 * primaryRay (src/main.cpp:69-83) for n (pixel, jitter) pairs with cfg's camera and size
 * (rays8 = origin, tmin, dir, tmax); toWorld(sampleCosineHemisphere(u1, u2), n)
 * (main.cpp:123-141); IBL::sample (main.cpp:107-117) of an h x w RGB map. */
void orc_primary_rays(const orc_render_cfg* cfg, uint64_t n, const int32_t* px, const int32_t* py, const float* jx,
                      const float* jy, float* rays8);
void orc_cosine_dirs(uint64_t n, const float* u1, const float* u2, const float* nrm3, float* out3);
void orc_ibl_lookup(const float* map, uint32_t w, uint32_t h, uint64_t n, const float* dirs3, float* out3);

/* Every ray against every triangle, no BVH (the triangle tests alone): nearest accepted hit,
 * out3 = t, u, v; flags as orc_trace. */
void orc_trace_brute(const float* verts6, const uint32_t* tris3, uint32_t n_tris, const float* rays8, uint64_t n,
                     uint32_t flags, float* out3, uint32_t* tri, uint8_t* hit);

/* Counter-based RNG shared with the device code: Philox4x32-10 (Salmon et al., SC'11). */
void orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                uint32_t* out4);

#ifdef __cplusplus
}
#endif
#endif
