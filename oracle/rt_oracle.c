/* rt_oracle.c -- CPU restatement of the reference path tracer's hot path (TEST ORACLE).
 *
 * Test infrastructure only: tests/, the smoke check and bench.py's CPU-baseline leg load
 * liboracle.so as the checker; the product library never does. Every function restates
 * the reference algorithm in plain C with the reference's float operation order, so that
 * on x86-64 (SSE scalar, no FMA contraction: built with -ffp-contract=off) it reproduces
 * the reference bit for bit. Parity of this restatement is pinned by tests against the
 * reference itself (oracle/_ref, compiled from the reference's own sources) and against
 * the known answers in the reference's tests/test_traverse.cpp and tests/test_aabb.cpp.
 *
 * Reference citations are path:line inside the reference project.
 */
#include "rt_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------ */
/* scalar helpers with the reference's exact semantics                                   */
/* ------------------------------------------------------------------------------------ */

/* SSE minps/maxps (math::min / math::max, src/math/vec3.hpp:72-73): the second operand
 * is returned unless the first compares strictly smaller / larger. */
static inline float sse_min(float a, float b) { return a < b ? a : b; }
static inline float sse_max(float a, float b) { return a > b ? a : b; }
/* std::min / std::max as used in src/bvh/bvh_traverse.cpp:36-37 and bvh_sah.cpp. */
static inline float std_min(float a, float b) { return (b < a) ? b : a; }
static inline float std_max(float a, float b) { return (a < b) ? b : a; }
static inline int   std_mini(int a, int b) { return (b < a) ? b : a; }
static inline int   std_clampi(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }

/* float -> int32 as x86-64 cvttss2si does it: truncation, and INT32_MIN for NaN or
 * out-of-range values (the reference's (int) casts in src/bvh/bvh_sah.cpp:85,179-180). */
static inline int x86_f2i(float f)
{
    if (!(f > -2147483904.0f && f < 2147483648.0f)) { return (int)0x80000000u; }
    return (int)f;
}
/* float -> uint32 as g++ emits it on x86-64: 64-bit cvttss2si, low 32 bits kept
 * (the (uint) cast of src/bvh/bvh_morton.cpp:78). */
static inline uint32_t x86_f2u(float f)
{
    int64_t v;
    if (!(f > -9223373136366403584.0f && f < 9223372036854775808.0f)) { v = INT64_MIN; }
    else { v = (int64_t)f; }
    return (uint32_t)(uint64_t)v;
}

typedef struct { float x, y, z; } v3;

static inline v3 mk3(float x, float y, float z) { v3 r = { x, y, z }; return r; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul3(v3 a, v3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 muls(v3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
static inline v3 divs(v3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
/* dot of src/math/vec3.hpp:42-50: (x*x' + y*y') + (z*z' + w*w'), the padded w lane 0. */
static inline float dot3(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + (a.z * b.z + 0.0f); }
/* cross of src/math/vec3.hpp:52-59 */
static inline v3 cross3(v3 a, v3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* normalize of src/math/vec3.hpp:66-70 */
static inline v3 norm3(v3 v)
{
    float inv = 1.0f / sqrtf(dot3(v, v));
    return muls(v, inv);
}

/* AABB (src/bvh/AABB.cpp:4-60); the empty box is +inf / -inf. */
typedef struct { float mn[3], mx[3]; } box3;

static inline box3 box_empty(void)
{
    box3 b;
    for (int k = 0; k < 3; k++) { b.mn[k] = INFINITY; b.mx[k] = -INFINITY; }
    return b;
}
static inline void box_pt(box3* b, v3 p)
{
    b->mn[0] = sse_min(b->mn[0], p.x); b->mn[1] = sse_min(b->mn[1], p.y); b->mn[2] = sse_min(b->mn[2], p.z);
    b->mx[0] = sse_max(b->mx[0], p.x); b->mx[1] = sse_max(b->mx[1], p.y); b->mx[2] = sse_max(b->mx[2], p.z);
}
static inline void box_box(box3* b, const box3* o)
{
    for (int k = 0; k < 3; k++) { b->mn[k] = sse_min(b->mn[k], o->mn[k]); b->mx[k] = sse_max(b->mx[k], o->mx[k]); }
}
/* half_area, src/bvh/AABB.cpp:29-33 */
static inline float box_half_area(const box3* b)
{
    float dx = b->mx[0] - b->mn[0], dy = b->mx[1] - b->mn[1], dz = b->mx[2] - b->mn[2];
    return dx * dy + dy * dz + dz * dx;
}
static inline int box_valid(const box3* b)
{
    return b->mn[0] <= b->mx[0] && b->mn[1] <= b->mx[1] && b->mn[2] <= b->mx[2];
}
static inline float v3_get(v3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

/* clipTriangleToAABB, src/bvh/AABB.cpp:86-171: Sutherland-Hodgman against the min then
 * the max plane of x, y, z; returns the box of the clipped polygon or the empty box. */
static box3 clip_triangle(v3 v0, v3 v1, v3 v2, const box3* region)
{
    v3 poly[12], tmp[12];
    int n = 3;
    poly[0] = v0; poly[1] = v1; poly[2] = v2;
    for (int axis = 0; axis < 3; axis++)
    {
        for (int side = 0; side < 2; side++)
        {
            float plane = side == 0 ? region->mn[axis] : region->mx[axis];
            int m = 0;
            for (int i = 0; i < n; i++)
            {
                int nx = (i + 1) % n;
                float pi = v3_get(poly[i], axis), pn = v3_get(poly[nx], axis);
                int cin = side == 0 ? (pi >= plane) : (pi <= plane);
                int nin = side == 0 ? (pn >= plane) : (pn <= plane);
                if (cin) { tmp[m++] = poly[i]; }
                if (cin != nin)
                {
                    float t = (plane - pi) / (pn - pi);
                    tmp[m++] = add3(poly[i], muls(sub3(poly[nx], poly[i]), t));
                }
            }
            for (int i = 0; i < m; i++) { poly[i] = tmp[i]; }
            n = m;
            if (n == 0) { return box_empty(); }
        }
    }
    box3 r = box_empty();
    for (int i = 0; i < n; i++) { box_pt(&r, poly[i]); }
    return r;
}

void orc_clip_triangle(const float* v9, const float* box6, float* out6)
{
    box3 b;
    for (int k = 0; k < 3; k++) { b.mn[k] = box6[k]; b.mx[k] = box6[3 + k]; }
    box3 r = clip_triangle(mk3(v9[0], v9[1], v9[2]), mk3(v9[3], v9[4], v9[5]), mk3(v9[6], v9[7], v9[8]), &b);
    for (int k = 0; k < 3; k++) { out6[k] = r.mn[k]; out6[3 + k] = r.mx[k]; }
}

void orc_cfg_default(orc_cfg* c)
{
    c->lbvh_threshold = 64;
    c->max_leaf       = 16;
    c->morton_bits    = 21;
    c->bins_min       = 8;
    c->bins_max       = 32;
    c->c_trav         = 1.0f;
    c->c_isect        = 1.2f;
    c->centroid_eps   = 1e-6f;
    c->spatial_eps    = 1e-6f;
    c->spatial_mult   = 1.5f;
}

/* ------------------------------------------------------------------------------------ */
/* vertex normals (initGeos, src/bvh/bvh_IO.cpp:102-118)                                 */
/* ------------------------------------------------------------------------------------ */

/* Three-argument hypot by scaling with the largest magnitude (the overflow-safe textbook
 * form), which is what std::hypot(float, float, float) evaluates in the reference's C++
 * library; pinned bit for bit against the reference by the oracle tests. */
static float hypot3f(float x, float y, float z)
{
    x = fabsf(x); y = fabsf(y); z = fabsf(z);
    float a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a == 0.0f) { return 0.0f; }
    float xa = x / a, ya = y / a, za = z / a;
    return a * sqrtf(xa * xa + ya * ya + za * za);
}

void orc_normalize_normals(float* v6, uint32_t V)
{
    for (uint32_t i = 0; i < V; i++)
    {
        float* n = v6 + 6 * (size_t)i + 3;
        float len = hypot3f(n[0], n[1], n[2]);
        if (len > 1e-6f) { n[0] /= len; n[1] /= len; n[2] /= len; }
        else { n[0] = 0.f; n[1] = 1.f; n[2] = 0.f; }
    }
}

/* ------------------------------------------------------------------------------------ */
/* Morton codes + radix sort (src/bvh/bvh_morton.cpp:19-159)                             */
/* ------------------------------------------------------------------------------------ */

/* Spread bit i of v to bit 3i (the interleave of expandBits, bvh_morton.cpp:19-28). */
static uint64_t spread3(uint32_t v)
{
    uint64_t r = 0;
    for (int i = 0; i < 21; i++) { r |= (uint64_t)((v >> i) & 1u) << (3 * i); }
    return r;
}

static inline v3 vpos(const float* v6, uint32_t i) { const float* p = v6 + 6 * (size_t)i; return mk3(p[0], p[1], p[2]); }

/* centroid as in bvh_morton.cpp:88-90 and bvh_bake.cpp:50-54: ((a + b) + c) / 3 */
static inline v3 tri_centroid(const float* v6, const uint32_t* t)
{
    v3 a = vpos(v6, t[0]), b = vpos(v6, t[1]), c = vpos(v6, t[2]);
    return mk3((a.x + b.x + c.x) / 3.0f, (a.y + b.y + c.y) / 3.0f, (a.z + b.z + c.z) / 3.0f);
}

static box3 scene_box(const float* v6, const uint32_t* t3, uint32_t N)
{
    box3 b = box_empty();
    for (uint32_t i = 0; i < N; i++)
    {
        for (int j = 0; j < 3; j++) { box_pt(&b, vpos(v6, t3[3 * (size_t)i + j])); }
    }
    return b;
}

static void morton_codes(const float* v6, const uint32_t* t3, uint32_t N, uint32_t bits,
                         uint64_t* codes, box3* sb)
{
    *sb = scene_box(v6, t3, N);
    float mn[3], size[3];
    for (int k = 0; k < 3; k++)
    {
        mn[k] = sb->mn[k];
        size[k] = sb->mx[k] - sb->mn[k];
        if (size[k] == 0.f) { size[k] = 1.f; }
    }
    const uint32_t qmax = (1u << bits) - 1u;
    const float    fmax = (float)qmax;
    for (uint32_t i = 0; i < N; i++)
    {
        v3 c = tri_centroid(v6, t3 + 3 * (size_t)i);
        float cc[3] = { c.x, c.y, c.z };
        uint32_t q[3];
        for (int k = 0; k < 3; k++)
        {
            uint32_t v = x86_f2u((cc[k] - mn[k]) * fmax / size[k]);
            q[k] = v > qmax ? qmax : v;
        }
        codes[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    }
}

/* Stable LSD radix sort of the identity permutation by code, 8 passes of 8 bits
 * (bvh_morton.cpp:121-156). */
static void radix_sort_perm(const uint64_t* codes, uint32_t N, uint32_t* perm)
{
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (N ? N : 1));
    for (uint32_t i = 0; i < N; i++) { perm[i] = i; }
    for (int pass = 0; pass < 8; pass++)
    {
        int shift = pass * 8;
        uint32_t count[256];
        memset(count, 0, sizeof(count));
        for (uint32_t i = 0; i < N; i++) { count[(codes[perm[i]] >> shift) & 255u]++; }
        uint32_t total = 0;
        for (int b = 0; b < 256; b++) { uint32_t c = count[b]; count[b] = total; total += c; }
        for (uint32_t i = 0; i < N; i++) { tmp[count[(codes[perm[i]] >> shift) & 255u]++] = perm[i]; }
        memcpy(perm, tmp, sizeof(uint32_t) * N);
    }
    free(tmp);
}

int orc_morton(const float* v6, uint32_t V, const uint32_t* t3, uint32_t N, const orc_cfg* cfg,
               uint64_t* codes, uint32_t* sorted, float* scene6)
{
    (void)V;
    if (N == 0) { return 0; }
    box3 sb;
    morton_codes(v6, t3, N, cfg->morton_bits, codes, &sb);
    radix_sort_perm(codes, N, sorted);
    for (int k = 0; k < 3; k++) { scene6[k] = sb.mn[k]; scene6[3 + k] = sb.mx[k]; }
    return 1;
}

/* ------------------------------------------------------------------------------------ */
/* the bake (src/bvh/bvh_bake.cpp, bvh_bfs.cpp, bvh_sah.cpp)                            */
/* ------------------------------------------------------------------------------------ */

typedef struct bnode { box3 box; uint8_t leaf; uint32_t a, b; } bnode;

struct orc_bvh
{
    /* baked result */
    orc_node* nodes; uint32_t n_nodes;
    uint32_t* tris;  uint32_t n_tris;
    float*    verts; uint32_t n_verts;
    uint32_t  stats[4];
};

typedef struct bstate
{
    orc_cfg         cfg;
    const float*    v6;
    const uint32_t* t3;
    uint32_t        N;
    uint64_t*       codes;
    uint32_t*       sorted;     /* s_sortedTris */
    uint32_t*       tidx;       /* s_triIndex */
    uint32_t        cap, tidx_size, sorted_size;
    float*          cent;       /* s_centroids, 3 per triangle */
    bnode*          nodes;
    uint32_t        node_cap, node_count;
    uint32_t*       q_node;
    uint8_t*        q_sah;
    uint32_t        q_head, q_tail;
    uint32_t        stats[4];
} bstate;

static inline void tri_verts(const bstate* S, uint32_t ti, v3* a, v3* b, v3* c)
{
    const uint32_t* t = S->t3 + 3 * (size_t)ti;
    *a = vpos(S->v6, t[0]); *b = vpos(S->v6, t[1]); *c = vpos(S->v6, t[2]);
}

static inline void q_push(bstate* S, uint32_t node, int sah)
{
    S->q_node[S->q_tail] = node;
    S->q_sah[S->q_tail]  = (uint8_t)sah;
    S->q_tail++;
}

/* computeRangeAABB, src/bvh/bvh_bfs.cpp:14-28 */
static box3 range_box(const bstate* S, uint32_t begin, uint32_t end)
{
    box3 b = box_empty();
    for (uint32_t i = begin; i < end; i++)
    {
        v3 a, bb, c;
        tri_verts(S, S->sorted[S->tidx[i]], &a, &bb, &c);
        box_pt(&b, a); box_pt(&b, bb); box_pt(&b, c);
    }
    return b;
}

/* std::partition as the reference's C++ library performs it for bidirectional
 * iterators (src/bvh/bvh_sah.cpp:257,304,318,348): Hoare's scheme -- advance from the
 * left past elements that satisfy the predicate, retreat from the right past elements
 * that do not, swap the pair, repeat until the cursors meet. flag[] holds the
 * predicate value of each element and moves with it. Returns the split position. */
static uint32_t hoare_partition(uint32_t* a, uint8_t* flag, uint32_t first, uint32_t last)
{
    for (;;)
    {
        for (;;)
        {
            if (first == last) { return first; }
            if (flag[first]) { ++first; } else { break; }
        }
        --last;
        for (;;)
        {
            if (first == last) { return first; }
            if (!flag[last]) { --last; } else { break; }
        }
        uint32_t t = a[first]; a[first] = a[last]; a[last] = t;
        uint8_t  f = flag[first]; flag[first] = flag[last]; flag[last] = f;
        ++first;
    }
}

static void make_children(bstate* S, uint32_t ni, uint32_t lb, uint32_t ln, box3 lbox,
                          uint32_t rb, uint32_t rn, box3 rbox)
{
    uint32_t l = S->node_count++, r = S->node_count++;
    S->nodes[ni].leaf = 0; S->nodes[ni].a = l; S->nodes[ni].b = r;
    S->nodes[l].box = lbox; S->nodes[l].leaf = 1; S->nodes[l].a = lb; S->nodes[l].b = ln;
    S->nodes[r].box = rbox; S->nodes[r].leaf = 1; S->nodes[r].a = rb; S->nodes[r].b = rn;
}

/* Object split of bvh_sah.cpp:254-293 (and its fallback copy, :335-388). */
static int apply_object_split(bstate* S, uint32_t ni, uint32_t begin, uint32_t end, int axis,
                              int bin, float cmin, float scale, int nb, uint8_t* flag)
{
    if (axis == -1) { S->nodes[ni].leaf = 1; S->stats[2]++; return 0; }
    for (uint32_t i = begin; i < end; i++)
    {
        float c = S->cent[3 * (size_t)S->sorted[S->tidx[i]] + axis];
        flag[i] = std_mini(x86_f2i((c - cmin) * scale), nb - 1) < bin;
    }
    uint32_t mid = hoare_partition(S->tidx, flag, begin, end);
    if (mid == begin || mid == end) { S->nodes[ni].leaf = 1; S->stats[2]++; return 0; }
    make_children(S, ni, begin, mid - begin, range_box(S, begin, mid), mid, end - mid, range_box(S, mid, end));
    q_push(S, S->nodes[ni].a, 1);
    q_push(S, S->nodes[ni].b, 1);
    return 1;
}

typedef struct { box3 box; uint32_t count; } obin;
typedef struct { box3 box; uint32_t cin, cout; } sbin;

/* trySAHSplit, src/bvh/bvh_sah.cpp:24-460 */
static int sah_split(bstate* S, uint32_t ni, uint8_t* flag)
{
    const orc_cfg* C = &S->cfg;
    uint32_t begin = S->nodes[ni].a, n = S->nodes[ni].b, end = begin + n;
    int nb = std_clampi((int)n / 4, (int)C->bins_min, (int)C->bins_max);

    float best_cost = C->c_isect * (float)n; /* leaf cost, :32 */
    int   best_axis = -1, best_bin = -1;
    float best_cmin = 0.f, best_scale = 0.f;
    float parent_inv_area = 1.0f / box_half_area(&S->nodes[ni].box);

    obin  bins[64];
    box3  l_box[64];
    uint32_t l_cnt[64];

    /* phase 1: centroid-binned object split, :52-126 */
    for (int axis = 0; axis < 3; axis++)
    {
        float cmin = FLT_MAX, cmax = -FLT_MAX;
        for (uint32_t i = begin; i < end; i++)
        {
            float c = S->cent[3 * (size_t)S->sorted[S->tidx[i]] + axis];
            cmin = std_min(cmin, c);
            cmax = std_max(cmax, c);
        }
        if (cmax - cmin < C->centroid_eps) { continue; }
        float scale = (float)nb / (cmax - cmin);
        for (int b = 0; b < nb; b++) { bins[b].box = box_empty(); bins[b].count = 0; }
        for (uint32_t i = begin; i < end; i++)
        {
            uint32_t ti = S->sorted[S->tidx[i]];
            float c = S->cent[3 * (size_t)ti + axis];
            int b = std_mini(x86_f2i((c - cmin) * scale), nb - 1);
            bins[b].count++;
            v3 a, bb, cc;
            tri_verts(S, ti, &a, &bb, &cc);
            box_pt(&bins[b].box, a); box_pt(&bins[b].box, bb); box_pt(&bins[b].box, cc);
        }
        box3 la = box_empty(); uint32_t lc = 0;
        for (int b = 0; b < nb - 1; b++)
        {
            box_box(&la, &bins[b].box);
            lc += bins[b].count;
            l_box[b] = la; l_cnt[b] = lc;
        }
        box3 ra = box_empty(); uint32_t rc = 0;
        for (int b = nb - 1; b >= 1; b--)
        {
            box_box(&ra, &bins[b].box);
            rc += bins[b].count;
            uint32_t lc2 = l_cnt[b - 1];
            if (lc2 == 0 || rc == 0) { continue; }
            float cost = C->c_trav + C->c_isect *
                (box_half_area(&l_box[b - 1]) * (float)lc2 + box_half_area(&ra) * (float)rc) * parent_inv_area;
            if (cost < best_cost)
            {
                best_cost = cost; best_axis = axis; best_bin = b; best_cmin = cmin; best_scale = scale;
            }
        }
    }
    const int   obj_axis = best_axis, obj_bin = best_bin;
    const float obj_cmin = best_cmin, obj_scale = best_scale;

    /* phase 2: spatial bins over the node box with per-bin clipping, :135-243 */
    sbin sb[64];
    box3 sl_box[64];
    uint32_t sl_cnt[64];
    int   is_spatial = 0;
    float best_node_min = 0.f, best_sscale = 0.f;
    const box3 nbox = S->nodes[ni].box;
    for (int axis = 0; axis < 3; axis++)
    {
        float node_min = nbox.mn[axis], node_max = nbox.mx[axis];
        if (node_max - node_min < C->spatial_eps) { continue; }
        float sscale = (float)nb / (node_max - node_min);
        for (int b = 0; b < nb; b++) { sb[b].box = box_empty(); sb[b].cin = 0; sb[b].cout = 0; }
        for (uint32_t i = begin; i < end; i++)
        {
            uint32_t ti = S->sorted[S->tidx[i]];
            v3 a, bb, cc;
            tri_verts(S, ti, &a, &bb, &cc);
            box3 tb = box_empty();
            box_pt(&tb, a); box_pt(&tb, bb); box_pt(&tb, cc);
            int bmin = std_clampi(x86_f2i((tb.mn[axis] - node_min) * sscale), 0, nb - 1);
            int bmax = std_clampi(x86_f2i((tb.mx[axis] - node_min) * sscale), 0, nb - 1);
            sb[bmin].cin++;
            sb[bmax].cout++;
            box3 region = nbox;
            for (int b = bmin; b <= bmax; b++)
            {
                region.mn[axis] = node_min + (float)b / sscale;
                region.mx[axis] = node_min + (float)(b + 1) / sscale;
                box3 cl = clip_triangle(a, bb, cc, &region);
                if (box_valid(&cl)) { box_box(&sb[b].box, &cl); }
            }
        }
        box3 spa = box_empty(); uint32_t splc = 0;
        for (int b = 0; b < nb - 1; b++)
        {
            box_box(&spa, &sb[b].box);
            splc += sb[b].cin;
            sl_box[b] = spa; sl_cnt[b] = splc;
        }
        box3 spra = box_empty(); uint32_t sprc = 0;
        for (int b = nb - 1; b >= 1; b--)
        {
            box_box(&spra, &sb[b].box);
            sprc += sb[b].cout;
            uint32_t lc2 = sl_cnt[b - 1];
            if (lc2 == 0 || sprc == 0) { continue; }
            float cost = C->c_trav + C->c_isect *
                (box_half_area(&sl_box[b - 1]) * (float)lc2 + box_half_area(&spra) * (float)sprc) * parent_inv_area;
            if (cost < best_cost)
            {
                best_cost = cost; best_axis = axis; best_bin = b; is_spatial = 1;
                best_node_min = node_min; best_sscale = sscale;
            }
        }
    }

    /* phase 3, :249-459 */
    if (best_axis == -1) { S->nodes[ni].leaf = 1; S->stats[2]++; return 0; }
    if (!is_spatial)
    {
        return apply_object_split(S, ni, begin, end, best_axis, best_bin, best_cmin, best_scale, nb, flag);
    }

    const int axis = best_axis;
    float plane = best_node_min + (float)best_bin / best_sscale;
    for (uint32_t i = begin; i < end; i++)
    {
        v3 a, bb, cc;
        tri_verts(S, S->sorted[S->tidx[i]], &a, &bb, &cc);
        box3 tb = box_empty();
        box_pt(&tb, a); box_pt(&tb, bb); box_pt(&tb, cc);
        flag[i] = tb.mx[axis] <= plane;
    }
    uint32_t left_end = hoare_partition(S->tidx, flag, begin, end);
    for (uint32_t i = left_end; i < end; i++)
    {
        v3 a, bb, cc;
        tri_verts(S, S->sorted[S->tidx[i]], &a, &bb, &cc);
        box3 tb = box_empty();
        box_pt(&tb, a); box_pt(&tb, bb); box_pt(&tb, cc);
        flag[i] = tb.mn[axis] < plane;
    }
    uint32_t straddle_end = hoare_partition(S->tidx, flag, left_end, end);
    uint32_t left_cnt = left_end - begin, straddle_cnt = straddle_end - left_end, right_cnt = end - straddle_end;

    if ((left_cnt + straddle_cnt == 0) || (straddle_cnt + right_cnt == 0))
    {
        return apply_object_split(S, ni, begin, end, obj_axis, obj_bin, obj_cmin, obj_scale, nb, flag);
    }
    if (S->tidx_size + right_cnt + straddle_cnt > S->cap || S->sorted_size + straddle_cnt > S->cap)
    {
        S->stats[1]++;
        return apply_object_split(S, ni, begin, end, obj_axis, obj_bin, obj_cmin, obj_scale, nb, flag);
    }
    S->stats[0]++;

    uint32_t right_begin = S->tidx_size;
    for (uint32_t k = 0; k < right_cnt; k++) { S->tidx[S->tidx_size++] = S->tidx[straddle_end + k]; }
    for (uint32_t k = 0; k < straddle_cnt; k++)
    {
        uint32_t old = S->tidx[left_end + k];
        S->sorted[S->sorted_size] = S->sorted[old];
        S->tidx[S->tidx_size] = S->sorted_size;
        S->sorted_size++;
        S->tidx_size++;
    }
    uint32_t right_size = right_cnt + straddle_cnt;
    uint32_t left_size  = left_cnt + straddle_cnt;

    box3 lclip = nbox, rclip = nbox;
    lclip.mx[axis] = plane;
    rclip.mn[axis] = plane;
    box3 lbox = box_empty(), rbox = box_empty();
    for (uint32_t k = begin; k < begin + left_size; k++)
    {
        v3 a, bb, cc;
        tri_verts(S, S->sorted[S->tidx[k]], &a, &bb, &cc);
        box3 cl = clip_triangle(a, bb, cc, &lclip);
        if (box_valid(&cl)) { box_box(&lbox, &cl); }
    }
    for (uint32_t k = right_begin; k < right_begin + right_size; k++)
    {
        v3 a, bb, cc;
        tri_verts(S, S->sorted[S->tidx[k]], &a, &bb, &cc);
        box3 cl = clip_triangle(a, bb, cc, &rclip);
        if (box_valid(&cl)) { box_box(&rbox, &cl); }
    }
    make_children(S, ni, begin, left_size, lbox, right_begin, right_size, rbox);
    q_push(S, S->nodes[ni].a, 1);
    q_push(S, S->nodes[ni].b, 1);
    return 1;
}

static inline uint64_t bit_floor64(uint64_t x)
{
    if (x == 0) { return 0; }
    return (uint64_t)1 << (63 - __builtin_clzll(x));
}

/* bfsLoop, src/bvh/bvh_bfs.cpp:72-134 */
static void bfs_loop(bstate* S, uint8_t* flag)
{
    const orc_cfg* C = &S->cfg;
    while (S->q_head < S->q_tail)
    {
        uint32_t ni  = S->q_node[S->q_head];
        int      sah = S->q_sah[S->q_head];
        S->q_head++;
        if (S->nodes[ni].b <= C->max_leaf) { S->nodes[ni].leaf = 1; continue; }
        if (sah) { sah_split(S, ni, flag); continue; }

        uint32_t begin = S->nodes[ni].a, n = S->nodes[ni].b, end = begin + n;
        uint64_t x = S->codes[S->sorted[begin]] ^ S->codes[S->sorted[end - 1]];
        if (x == 0) { sah_split(S, ni, flag); continue; }
        uint64_t mask = bit_floor64(x);
        uint32_t split = 0xFFFFFFFFu;
        for (uint32_t i = 0; i + 1 < n; i++) /* findMortonSplitIndex, :35-48 */
        {
            if ((S->codes[S->sorted[begin + i]] & mask) != (S->codes[S->sorted[begin + i + 1]] & mask))
            {
                split = begin + i + 1;
                break;
            }
        }
        S->stats[3]++;
        make_children(S, ni, begin, split - begin, range_box(S, begin, split), split, end - split,
                      range_box(S, split, end));
        uint32_t l = S->nodes[ni].a, r = S->nodes[ni].b;
        q_push(S, l, S->nodes[l].b <= C->lbvh_threshold);
        q_push(S, r, S->nodes[r].b <= C->lbvh_threshold);
    }
}

static void write_box(orc_node* o, const box3* b)
{
    int empty = !(b->mn[0] <= b->mx[0]) && b->mn[0] == INFINITY;
    for (int k = 0; k < 3; k++) { o->bmin[k] = b->mn[k]; o->bmax[k] = b->mx[k]; }
    /* padded lane: 0 once a point was added, else the +inf / -inf of the empty box */
    o->bmin[3] = empty ? INFINITY : 0.f;
    o->bmax[3] = empty ? -INFINITY : 0.f;
}

orc_bvh* orc_build(const float* verts6, uint32_t V, const uint32_t* tris3, uint32_t N, const orc_cfg* cfg)
{
    /* initGeos checks, src/bvh/bvh_IO.cpp:74-100 */
    if (V == 0 || N == 0) { return NULL; }
    for (uint64_t i = 0; i < 3ull * N; i++) { if (tris3[i] >= V) { return NULL; } }

    orc_bvh* out = (orc_bvh*)calloc(1, sizeof(orc_bvh));
    out->n_verts = V;
    out->verts = (float*)malloc(sizeof(float) * 6 * (size_t)V);
    memcpy(out->verts, verts6, sizeof(float) * 6 * (size_t)V);
    orc_normalize_normals(out->verts, V);

    bstate S;
    memset(&S, 0, sizeof(S));
    S.cfg = *cfg;
    S.v6 = out->verts; /* positions are untouched by the normalisation */
    S.t3 = tris3;
    S.N  = N;
    S.cap = (uint32_t)((float)N * cfg->spatial_mult); /* bvh_morton.cpp:46-47 */
    if (S.cap < N) { S.cap = N; }
    S.codes  = (uint64_t*)malloc(sizeof(uint64_t) * N);
    S.sorted = (uint32_t*)malloc(sizeof(uint32_t) * S.cap);
    S.tidx   = (uint32_t*)malloc(sizeof(uint32_t) * S.cap);
    S.cent   = (float*)malloc(sizeof(float) * 3 * (size_t)N);
    box3 sb;
    morton_codes(S.v6, tris3, N, cfg->morton_bits, S.codes, &sb);
    radix_sort_perm(S.codes, N, S.sorted);
    for (uint32_t i = 0; i < N; i++) { S.tidx[i] = i; }
    S.tidx_size = N; S.sorted_size = N;
    for (uint32_t i = 0; i < N; i++) /* buildCentroidCache, bvh_bake.cpp:44-58 */
    {
        v3 c = tri_centroid(S.v6, tris3 + 3 * (size_t)i);
        S.cent[3 * (size_t)i] = c.x; S.cent[3 * (size_t)i + 1] = c.y; S.cent[3 * (size_t)i + 2] = c.z;
    }
    S.node_cap = S.cap * 2 - 1; /* initRoot, bvh_bfs.cpp:58 */
    S.nodes  = (bnode*)calloc(S.node_cap, sizeof(bnode));
    S.q_node = (uint32_t*)malloc(sizeof(uint32_t) * S.node_cap);
    S.q_sah  = (uint8_t*)malloc(S.node_cap);
    uint8_t* flag = (uint8_t*)malloc(S.cap);
    S.node_count = 1;
    S.nodes[0].box = sb; S.nodes[0].leaf = 1; S.nodes[0].a = 0; S.nodes[0].b = N;
    q_push(&S, 0, N <= cfg->lbvh_threshold);
    bfs_loop(&S, flag);

    /* reorderNodes, bvh_bake.cpp:75-118: DFS pre-order, left child first */
    uint32_t* remap = (uint32_t*)malloc(sizeof(uint32_t) * S.node_count);
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * S.node_count);
    uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * (S.node_count + 1));
    uint32_t top = 0, cnt = 0;
    stack[top++] = 0;
    while (top > 0)
    {
        uint32_t o = stack[--top];
        remap[o] = cnt;
        order[cnt++] = o;
        if (!S.nodes[o].leaf) { stack[top++] = S.nodes[o].b; stack[top++] = S.nodes[o].a; }
    }
    out->n_nodes = cnt;
    out->nodes = (orc_node*)calloc(cnt, sizeof(orc_node));
    /* reorderTriangles, bvh_bake.cpp:120-149: leaves' triangles made contiguous in DFS order */
    uint32_t total = 0;
    for (uint32_t i = 0; i < cnt; i++) { if (S.nodes[order[i]].leaf) { total += S.nodes[order[i]].b; } }
    out->n_tris = total;
    out->tris = (uint32_t*)malloc(sizeof(uint32_t) * 3 * (size_t)(total ? total : 1));
    uint32_t pos = 0;
    for (uint32_t i = 0; i < cnt; i++)
    {
        const bnode* s = &S.nodes[order[i]];
        orc_node* o = &out->nodes[i];
        write_box(o, &s->box);
        o->is_leaf = s->leaf;
        if (s->leaf)
        {
            o->a = pos; o->b = s->b;
            for (uint32_t k = 0; k < s->b; k++)
            {
                uint32_t ti = S.sorted[S.tidx[s->a + k]];
                memcpy(out->tris + 3 * (size_t)pos, tris3 + 3 * (size_t)ti, 12);
                pos++;
            }
        }
        else
        {
            o->a = remap[s->a]; o->b = remap[s->b];
        }
    }
    memcpy(out->stats, S.stats, sizeof(S.stats));
    free(remap); free(order); free(stack); free(flag);
    free(S.codes); free(S.sorted); free(S.tidx); free(S.cent); free(S.nodes); free(S.q_node); free(S.q_sah);
    return out;
}

void orc_counts(const orc_bvh* b, uint32_t* c3) { c3[0] = b->n_nodes; c3[1] = b->n_tris; c3[2] = b->n_verts; }
void orc_stats(const orc_bvh* b, uint32_t* s4) { memcpy(s4, b->stats, sizeof(b->stats)); }

void orc_get(const orc_bvh* b, orc_node* nodes, uint32_t* tris3, float* verts6)
{
    if (nodes) { memcpy(nodes, b->nodes, sizeof(orc_node) * b->n_nodes); }
    if (tris3) { memcpy(tris3, b->tris, 12 * (size_t)b->n_tris); }
    if (verts6) { memcpy(verts6, b->verts, 24 * (size_t)b->n_verts); }
}

orc_bvh* orc_from_arrays(const orc_node* nodes, uint32_t n_nodes, const uint32_t* tris3, uint32_t n_tris,
                         const float* verts6, uint32_t n_verts)
{
    orc_bvh* b = (orc_bvh*)calloc(1, sizeof(orc_bvh));
    b->n_nodes = n_nodes; b->n_tris = n_tris; b->n_verts = n_verts;
    b->nodes = (orc_node*)malloc(sizeof(orc_node) * (n_nodes ? n_nodes : 1));
    b->tris  = (uint32_t*)malloc(12 * (size_t)(n_tris ? n_tris : 1));
    b->verts = (float*)malloc(24 * (size_t)(n_verts ? n_verts : 1));
    memcpy(b->nodes, nodes, sizeof(orc_node) * n_nodes);
    memcpy(b->tris, tris3, 12 * (size_t)n_tris);
    memcpy(b->verts, verts6, 24 * (size_t)n_verts);
    return b;
}

void orc_free(orc_bvh* b)
{
    if (!b) { return; }
    free(b->nodes); free(b->tris); free(b->verts); free(b);
}

/* ------------------------------------------------------------------------------------ */
/* traversal (src/bvh/bvh_traverse.cpp:22-178)                                           */
/* ------------------------------------------------------------------------------------ */

typedef struct { v3 o, d; float tmin, tmax; } oray;
typedef struct { int hit; float t, u, v; uint32_t tri; v3 n; } ohit;

/* rayAABB, bvh_traverse.cpp:22-41 */
static inline float ray_box(const oray* r, const orc_node* nd, float tmax)
{
    float ix = 1.f / r->d.x, iy = 1.f / r->d.y, iz = 1.f / r->d.z;
    float t0x = (nd->bmin[0] - r->o.x) * ix, t1x = (nd->bmax[0] - r->o.x) * ix;
    float t0y = (nd->bmin[1] - r->o.y) * iy, t1y = (nd->bmax[1] - r->o.y) * iy;
    float t0z = (nd->bmin[2] - r->o.z) * iz, t1z = (nd->bmax[2] - r->o.z) * iz;
    float tn = std_max(std_max(std_min(t0x, t1x), std_min(t0y, t1y)), std_max(std_min(t0z, t1z), r->tmin));
    float tf = std_min(std_min(std_max(t0x, t1x), std_max(t0y, t1y)), std_min(std_max(t0z, t1z), tmax));
    return (tn <= tf) ? tn : INFINITY;
}

/* rayTriangle, bvh_traverse.cpp:47-87: Moller-Trumbore, back faces (a >= 0) culled */
static inline int ray_tri(const oray* r, v3 v0, v3 v1, v3 v2, float* t, float* u, float* v)
{
    v3 e1 = sub3(v1, v0), e2 = sub3(v2, v0);
    v3 h = cross3(r->d, e2);
    float a = dot3(e1, h);
    if (a >= 0) { return 0; }
    float f = 1.f / a;
    v3 s = sub3(r->o, v0);
    float uu = f * dot3(s, h);
    if (uu < 0.f || uu > 1.f) { return 0; }
    v3 q = cross3(s, e1);
    float vv = f * dot3(r->d, q);
    if (vv < 0.f || uu + vv > 1.f) { return 0; }
    float tt = f * dot3(e2, q);
    if (tt < r->tmin || tt > r->tmax) { return 0; }
    *t = tt; *u = uu; *v = vv;
    return 1;
}

static inline float flip_sign(float x, uint32_t sign_bit)
{
    uint32_t b;
    memcpy(&b, &x, 4);
    b ^= sign_bit;
    memcpy(&x, &b, 4);
    return x;
}

/* Watertight ray/triangle intersection after Woop, Benthin and Wald, "Watertight Ray/Triangle
 * Intersection", Journal of Computer Graphics Techniques 2(1), 2013, section 3 and its
 * listing, without back-face culling. Not in the reference (its rayTriangle culls back faces
 * and is not watertight); the test of the library's RT_TRACE_WATERTIGHT mode. Steps:
 *  1. kz = the axis of the largest |dir| component, kx = kz + 1, ky = kx + 1 (mod 3), kx and
 *     ky swapped when dir[kz] < 0 so the winding is kept;
 *  2. shear constants Sx = dir[kx] / dir[kz], Sy = dir[ky] / dir[kz], Sz = 1 / dir[kz];
 *  3. vertices relative to the origin, sheared: A = v0 - org, Ax = A[kx] - Sx * A[kz], ...;
 *  4. scaled barycentrics U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax,
 *     all three recomputed in double precision when any is exactly zero (edge hits);
 *  5. miss when the signs of U, V, W differ; det = U + V + W, miss when det = 0;
 *  6. scaled distance T = U * (Sz A[kz]) + V * (Sz B[kz]) + W * (Sz C[kz]), tested against the
 *     ray's [tmin, tmax] scaled by |det| with det's sign taken off T (no division yet);
 *  7. t = T / det and the barycentrics of v1 and v2 (V / det, W / det) through one reciprocal.
 * The paper's lower distance bound of 0 is the ray's tmin here, its upper bound the ray's tmax
 * (the reference's rayTriangle tests the ray's own range; traverse keeps the nearest). */
static inline int ray_tri_watertight(const oray* r, v3 v0, v3 v1, v3 v2, float* t, float* u, float* v)
{
    const float adx = fabsf(r->d.x), ady = fabsf(r->d.y), adz = fabsf(r->d.z);
    int kz = (adx > ady) ? (adx > adz ? 0 : 2) : (ady > adz ? 1 : 2);
    int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
    const float dz = v3_get(r->d, kz);
    if (dz < 0.f) { int sw = kx; kx = ky; ky = sw; }
    const float Sx = v3_get(r->d, kx) / dz, Sy = v3_get(r->d, ky) / dz, Sz = 1.f / dz;
    const v3 A = sub3(v0, r->o), B = sub3(v1, r->o), C = sub3(v2, r->o);
    const float Ax = v3_get(A, kx) - Sx * v3_get(A, kz), Ay = v3_get(A, ky) - Sy * v3_get(A, kz);
    const float Bx = v3_get(B, kx) - Sx * v3_get(B, kz), By = v3_get(B, ky) - Sy * v3_get(B, kz);
    const float Cx = v3_get(C, kx) - Sx * v3_get(C, kz), Cy = v3_get(C, ky) - Sy * v3_get(C, kz);
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.f || V == 0.f || W == 0.f)
    {
        const double CxBy = (double)Cx * (double)By, CyBx = (double)Cy * (double)Bx;
        const double AxCy = (double)Ax * (double)Cy, AyCx = (double)Ay * (double)Cx;
        const double BxAy = (double)Bx * (double)Ay, ByAx = (double)By * (double)Ax;
        U = (float)(CxBy - CyBx);
        V = (float)(AxCy - AyCx);
        W = (float)(BxAy - ByAx);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) { return 0; }
    const float det = U + V + W;
    if (det == 0.f) { return 0; }
    const float Az = Sz * v3_get(A, kz), Bz = Sz * v3_get(B, kz), Cz = Sz * v3_get(C, kz);
    const float T = U * Az + V * Bz + W * Cz;
    uint32_t db;
    memcpy(&db, &det, 4);
    const uint32_t sign_bit = db & 0x80000000u;
    const float Ts = flip_sign(T, sign_bit), Ds = flip_sign(det, sign_bit);
    if (!(Ts >= r->tmin * Ds && Ts <= r->tmax * Ds)) { return 0; }
    const float rcp = 1.f / det;
    *t = T * rcp; *u = V * rcp; *v = W * rcp;
    return 1;
}

/* Every ray against every triangle (no BVH), nearest accepted hit: isolates the triangle
 * tests from the box tests of the traversal. out3 = t, u, v. */
void orc_trace_brute(const float* verts6, const uint32_t* tris3, uint32_t n_tris, const float* rays8, uint64_t n,
                     uint32_t flags, float* out3, uint32_t* tri, uint8_t* hit)
{
    for (uint64_t i = 0; i < n; i++)
    {
        const float* rp = rays8 + 8 * i;
        oray r;
        r.o = mk3(rp[0], rp[1], rp[2]); r.tmin = rp[3];
        r.d = mk3(rp[4], rp[5], rp[6]); r.tmax = rp[7];
        float best = r.tmax;
        hit[i] = 0; tri[i] = 0; out3[3 * i] = 0.f; out3[3 * i + 1] = 0.f; out3[3 * i + 2] = 0.f;
        for (uint32_t k = 0; k < n_tris; k++)
        {
            const uint32_t* tv = tris3 + 3 * (size_t)k;
            v3 p0 = vpos(verts6, tv[0]), p1 = vpos(verts6, tv[1]), p2 = vpos(verts6, tv[2]);
            float t = INFINITY, u = 0.f, v = 0.f;
            const int acc = (flags & ORC_TRACE_WATERTIGHT) ? ray_tri_watertight(&r, p0, p1, p2, &t, &u, &v)
                                                           : ray_tri(&r, p0, p1, p2, &t, &u, &v);
            if (acc && t < best)
            {
                best = t;
                hit[i] = 1; tri[i] = k; out3[3 * i] = t; out3[3 * i + 1] = u; out3[3 * i + 2] = v;
                if (flags & ORC_TRACE_ANY_HIT) { break; }
            }
        }
    }
}

/* traverse, bvh_traverse.cpp:91-178. Returns 1 if the 64-entry stack would overflow. */
static int traverse(const orc_bvh* B, const oray* r, uint32_t flags, ohit* best, uint32_t* ctr)
{
    best->hit = 0; best->t = 0.f; best->u = 0.f; best->v = 0.f; best->tri = 0; best->n = mk3(0, 0, 0);
    float best_t = r->tmax;
    uint32_t stack[64];
    int top = 0, overflow = 0;
    uint32_t popped = 0, tested = 0, maxdepth = 1;
    stack[top++] = 0;
    while (top > 0)
    {
        uint32_t ni = stack[--top];
        const orc_node* nd = &B->nodes[ni];
        popped++;
        float tb = ray_box(r, nd, best_t);
        if (tb >= best_t) { continue; }
        if (nd->is_leaf)
        {
            for (uint32_t k = 0; k < nd->b; k++)
            {
                uint32_t ti = nd->a + k;
                const uint32_t* tv = B->tris + 3 * (size_t)ti;
                v3 p0 = vpos(B->verts, tv[0]), p1 = vpos(B->verts, tv[1]), p2 = vpos(B->verts, tv[2]);
                float t = INFINITY, u = 0.f, v = 0.f;
                tested++;
                const int acc = (flags & ORC_TRACE_WATERTIGHT) ? ray_tri_watertight(r, p0, p1, p2, &t, &u, &v)
                                                               : ray_tri(r, p0, p1, p2, &t, &u, &v);
                if (!acc) { t = INFINITY; }
                if (t < best_t)
                {
                    best_t = t;
                    best->hit = 1; best->t = t; best->u = u; best->v = v; best->tri = ti;
                    float w = 1.f - u - v;
                    const float* n0 = B->verts + 6 * (size_t)tv[0] + 3;
                    const float* n1 = B->verts + 6 * (size_t)tv[1] + 3;
                    const float* n2 = B->verts + 6 * (size_t)tv[2] + 3;
                    v3 nn = add3(add3(muls(mk3(n0[0], n0[1], n0[2]), w), muls(mk3(n1[0], n1[1], n1[2]), u)),
                                 muls(mk3(n2[0], n2[1], n2[2]), v));
                    best->n = norm3(nn);
                    if (flags & ORC_TRACE_ANY_HIT) { top = 0; break; }
                }
            }
        }
        else
        {
            uint32_t l = nd->a, rr = nd->b;
            float tl = ray_box(r, &B->nodes[l], best_t);
            float tr = ray_box(r, &B->nodes[rr], best_t);
            uint32_t first_push, second_push;
            float tfirst, tsecond;
            if (tl <= tr) { first_push = rr; tfirst = tr; second_push = l; tsecond = tl; }
            else          { first_push = l;  tfirst = tl; second_push = rr; tsecond = tr; }
            if (tfirst < best_t)
            {
                if (top >= 64) { overflow = 1; break; }
                stack[top++] = first_push;
            }
            if (tsecond < best_t)
            {
                if (top >= 64) { overflow = 1; break; }
                stack[top++] = second_push;
            }
            if ((uint32_t)top > maxdepth) { maxdepth = (uint32_t)top; }
        }
    }
    if (ctr) { ctr[0] = popped; ctr[1] = tested; ctr[2] = maxdepth; }
    return overflow;
}

typedef struct
{
    const orc_bvh* B; const float* rays; uint64_t b, e; uint32_t flags;
    float* out6; uint32_t* tri; uint8_t* hit; uint32_t* ctr; uint64_t overflow;
} trace_job;

static void* trace_worker(void* p)
{
    trace_job* J = (trace_job*)p;
    for (uint64_t i = J->b; i < J->e; i++)
    {
        const float* rp = J->rays + 8 * i;
        oray r;
        r.o = mk3(rp[0], rp[1], rp[2]); r.tmin = rp[3];
        r.d = mk3(rp[4], rp[5], rp[6]); r.tmax = rp[7];
        ohit h;
        J->overflow += (uint64_t)traverse(J->B, &r, J->flags, &h, J->ctr ? J->ctr + 3 * i : NULL);
        J->hit[i] = (uint8_t)h.hit;
        J->tri[i] = h.tri;
        float* o = J->out6 + 6 * i;
        o[0] = h.t; o[1] = h.u; o[2] = h.v; o[3] = h.n.x; o[4] = h.n.y; o[5] = h.n.z;
    }
    return NULL;
}

uint64_t orc_trace(const orc_bvh* B, const float* rays8, uint64_t n, uint32_t flags, float* out6,
                   uint32_t* tri, uint8_t* hit, uint32_t* counters, int nthreads)
{
    if (nthreads < 1) { nthreads = 1; }
    if (nthreads > 256) { nthreads = 256; }
    trace_job jobs[256];
    pthread_t th[256];
    uint64_t chunk = (n + (uint64_t)nthreads - 1) / (uint64_t)nthreads;
    int used = 0;
    for (int t = 0; t < nthreads; t++)
    {
        uint64_t b = (uint64_t)t * chunk, e = b + chunk > n ? n : b + chunk;
        if (b >= e) { break; }
        trace_job J = { B, rays8, b, e, flags, out6, tri, hit, counters, 0 };
        jobs[used] = J;
        used++;
    }
    if (used == 1) { trace_worker(&jobs[0]); return jobs[0].overflow; }
    for (int t = 0; t < used; t++) { pthread_create(&th[t], NULL, trace_worker, &jobs[t]); }
    uint64_t of = 0;
    for (int t = 0; t < used; t++) { pthread_join(th[t], NULL); of += jobs[t].overflow; }
    return of;
}

/* ------------------------------------------------------------------------------------ */
/* path loop (src/main.cpp:69-204, 323-365) with a counter-based per-pixel RNG           */
/* ------------------------------------------------------------------------------------ */

static inline uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t* hi)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    return (uint32_t)p;
}

/* Philox4x32 with 10 rounds (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key increments
 * 0x9E3779B9 / 0xBB67AE85. */
void orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t* out)
{
    for (int r = 0; r < 10; r++)
    {
        uint32_t hi0, hi1;
        uint32_t lo0 = mulhilo32(0xD2511F53u, c0, &hi0);
        uint32_t lo1 = mulhilo32(0xCD9E8D57u, c2, &hi1);
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

#define ORC_PI 3.14159265358979323846f

typedef struct
{
    const orc_bvh* B; const orc_render_cfg* C; const orc_material* mats; const uint32_t* mot;
    const float* talb; uint32_t n_mats;
    const float* env_map; uint32_t env_w, env_h;
} render_ctx;

/* IBL::sample (src/main.cpp:107-117): nearest texel of an equirectangular map. */
static v3 ibl_sample(const render_ctx* R, v3 d)
{
    float phi = atan2f(d.z, d.x);
    float y = d.y < -1.f ? -1.f : (1.f < d.y ? 1.f : d.y);
    float theta = acosf(y);
    float u = (phi + ORC_PI) / (2.f * ORC_PI);
    float v = theta / ORC_PI;
    int px = (int)(u * (float)R->env_w), py = (int)(v * (float)R->env_h);
    if (px > (int)R->env_w - 1) { px = (int)R->env_w - 1; }
    if (py > (int)R->env_h - 1) { py = (int)R->env_h - 1; }
    const float* p = R->env_map + ((size_t)py * R->env_w + (size_t)px) * 3;
    return mk3(p[0], p[1], p[2]);
}

/* One path vertex as the adjoint needs it: the triangle, its material, the albedo and
 * emission used there and the Russian-roulette probability that divided the throughput
 * after it (1 when roulette did not run). */
typedef struct { uint32_t tri, mat; v3 albedo, emission; float p; } path_vtx;
typedef struct { uint32_t n; path_vtx v[64]; int missed; v3 env; } path_rec;

static void surface(const render_ctx* R, uint32_t tri, v3* albedo, v3* emission, uint32_t* kind, uint32_t* mat)
{
    *albedo = mk3(0.8f, 0.8f, 0.8f);
    *emission = mk3(0.f, 0.f, 0.f);
    *kind = 0; *mat = 0;
    if (R->mats)
    {
        uint32_t m = R->mot ? R->mot[tri] : 0u;
        if (m >= R->n_mats) { m = R->n_mats - 1u; }
        const orc_material* M = &R->mats[m];
        *albedo = mk3(M->albedo[0], M->albedo[1], M->albedo[2]);
        *emission = mk3(M->emission[0], M->emission[1], M->emission[2]);
        *kind = M->kind; *mat = m;
    }
    if (R->talb) { const float* a = R->talb + 3 * (size_t)tri; *albedo = mk3(a[0], a[1], a[2]); }
}

/* primaryRay (src/main.cpp:69-83): the ray through pixel (x, y) at jitter (jx, jy). */
static oray primary_ray(const orc_render_cfg* C, uint32_t x, uint32_t y, float jx, float jy)
{
    const uint32_t W = C->width, H = C->height;
    const float aspect = (float)W / (float)H;
    const v3 pos = mk3(C->cam_pos[0], C->cam_pos[1], C->cam_pos[2]);
    const v3 fwd = mk3(C->cam_fwd[0], C->cam_fwd[1], C->cam_fwd[2]);
    const v3 rgt = mk3(C->cam_right[0], C->cam_right[1], C->cam_right[2]);
    const v3 up  = mk3(C->cam_up[0], C->cam_up[1], C->cam_up[2]);
    const float th = C->tan_half_fov_y;
    float u = (((float)x + jx) / (float)W * 2.f - 1.f) * aspect;
    float v = ((float)y + jy) / (float)H * 2.f - 1.f;
    oray ray;
    ray.o = pos;
    ray.d = norm3(add3(add3(fwd, muls(rgt, u * th)), muls(up, v * th)));
    ray.tmin = 1e-3f;
    ray.tmax = INFINITY;
    return ray;
}

/* toWorld(sampleCosineHemisphere(u1, u2), n) (src/main.cpp:123-141). */
static v3 cosine_dir(float u1, float u2, v3 n)
{
    float rr = sqrtf(u1);
    float theta = 2.f * ORC_PI * u2;
    v3 ld = mk3(rr * cosf(theta), sqrtf(std_max(0.f, 1.f - u1)), rr * sinf(theta));
    v3 axis = fabsf(n.x) < 0.9f ? mk3(1.f, 0.f, 0.f) : mk3(0.f, 1.f, 0.f);
    v3 t = norm3(cross3(n, axis));
    v3 b = cross3(n, t);
    return add3(add3(muls(t, ld.x), muls(n, ld.y)), muls(b, ld.z));
}

void orc_primary_rays(const orc_render_cfg* C, uint64_t n, const int32_t* px, const int32_t* py, const float* jx,
                      const float* jy, float* rays8)
{
    for (uint64_t i = 0; i < n; i++)
    {
        oray r = primary_ray(C, (uint32_t)px[i], (uint32_t)py[i], jx[i], jy[i]);
        float* o = rays8 + 8 * i;
        o[0] = r.o.x; o[1] = r.o.y; o[2] = r.o.z; o[3] = r.tmin;
        o[4] = r.d.x; o[5] = r.d.y; o[6] = r.d.z; o[7] = r.tmax;
    }
}

void orc_cosine_dirs(uint64_t n, const float* u1, const float* u2, const float* nrm3, float* out3)
{
    for (uint64_t i = 0; i < n; i++)
    {
        v3 w = cosine_dir(u1[i], u2[i], mk3(nrm3[3 * i], nrm3[3 * i + 1], nrm3[3 * i + 2]));
        out3[3 * i] = w.x; out3[3 * i + 1] = w.y; out3[3 * i + 2] = w.z;
    }
}

void orc_ibl_lookup(const float* map, uint32_t w, uint32_t h, uint64_t n, const float* dirs3, float* out3)
{
    render_ctx R;
    memset(&R, 0, sizeof(R));
    R.env_map = map; R.env_w = w; R.env_h = h;
    for (uint64_t i = 0; i < n; i++)
    {
        v3 c = ibl_sample(&R, mk3(dirs3[3 * i], dirs3[3 * i + 1], dirs3[3 * i + 2]));
        out3[3 * i] = c.x; out3[3 * i + 1] = c.y; out3[3 * i + 2] = c.z;
    }
}

/* primaryRay + pathTrace (src/main.cpp:69-83, 145-204) for one sample of one pixel; rec
 * (optional) receives the vertices of the path. */
static v3 path_sample(const render_ctx* R, uint32_t x, uint32_t y, uint32_t sidx, path_rec* rec, uint64_t* st3)
{
    const orc_render_cfg* C = R->C;
    const uint32_t W = C->width, pix = y * W + x;
    if (rec) { rec->n = 0; rec->missed = 0; }
    uint32_t r4[4];
    orc_philox(pix, sidx, 0u, 0u, C->seed, 0x5EEDu, r4);
    oray ray = primary_ray(C, x, y, u01(r4[0]), u01(r4[1]));
    v3 tp = mk3(1.f, 1.f, 1.f), L = mk3(0.f, 0.f, 0.f);
    for (uint32_t bounce = 0; bounce <= C->max_bounce; bounce++)
    {
        ohit h;
        uint32_t ctr[3];
        traverse(R->B, &ray, 0u, &h, st3 ? ctr : NULL);
        if (st3) { st3[0] += 1u; st3[1] += ctr[0]; st3[2] += ctr[1]; }
        if (!h.hit)
        {
            v3 env;
            if (C->env_kind == 0)
            {
                float t = ray.d.y * 0.5f + 0.5f;
                env = add3(muls(mk3(1.0f, 1.0f, 1.0f), 1.f - t), muls(mk3(0.5f, 0.7f, 1.0f), t));
            }
            else if (C->env_kind == 2) { env = ibl_sample(R, ray.d); }
            else { env = mk3(C->env_color[0], C->env_color[1], C->env_color[2]); }
            L = add3(L, mul3(tp, env));
            if (rec) { rec->missed = 1; rec->env = env; }
            break;
        }
        v3 albedo, emission;
        uint32_t kind, mat;
        surface(R, h.tri, &albedo, &emission, &kind, &mat);
        L = add3(L, mul3(tp, emission));
        path_vtx* pv = NULL;
        if (rec && rec->n < 64)
        {
            pv = &rec->v[rec->n++];
            pv->tri = h.tri; pv->mat = mat; pv->albedo = albedo; pv->emission = emission; pv->p = 1.f;
        }
        orc_philox(pix, sidx, bounce + 1u, 0u, C->seed, 0x5EEDu, r4);
        v3 wdir;
        if (kind == 1)
        {
            wdir = sub3(ray.d, muls(h.n, 2.f * dot3(ray.d, h.n)));
        }
        else
        {
            wdir = cosine_dir(u01(r4[0]), u01(r4[1]), h.n);  /* sampleCosineHemisphere + toWorld */
        }
        tp = mul3(tp, albedo);
        if (C->rr_after >= 0 && (int32_t)bounce > C->rr_after)
        {
            float pr = std_max(std_max(tp.x, tp.y), tp.z);
            if (u01(r4[2]) > pr) { break; }
            tp = divs(tp, pr);
            if (pv) { pv->p = pr; }
        }
        v3 hp = add3(ray.o, muls(ray.d, h.t));
        ray.o = hp; ray.d = wdir; ray.tmin = 1e-4f; ray.tmax = INFINITY;
    }
    return L;
}

typedef struct
{
    const render_ctx* R;
    uint32_t row0, row1; float* rgb; float* rgb2;
    /* adjoint */
    const float* dimg; double* g_alb; double* g_em;
    /* traversal counts (orc_render_stats): segments traced, nodes popped, triangles tested */
    int want_stats; uint64_t stats[3];
} render_job;

static void* render_worker(void* p)
{
    render_job* J = (render_job*)p;
    const orc_render_cfg* C = J->R->C;
    const uint32_t W = C->width;
    for (uint32_t y = J->row0; y < J->row1; y++)
    {
        for (uint32_t x = 0; x < W; x++)
        {
            const uint32_t pix = y * W + x;
            v3 acc = mk3(0, 0, 0), acc2 = mk3(0, 0, 0);
            for (uint32_t s = 0; s < C->spp; s++)
            {
                const v3 L = path_sample(J->R, x, y, C->sample_offset + s, NULL, J->want_stats ? J->stats : NULL);
                acc = add3(acc, L);
                acc2 = add3(acc2, mul3(L, L));
            }
            float inv = (float)C->spp;
            float* o = J->rgb + 3 * (size_t)pix;
            o[0] = acc.x / inv; o[1] = acc.y / inv; o[2] = acc.z / inv;
            if (J->rgb2)
            {
                float* o2 = J->rgb2 + 3 * (size_t)pix;
                o2[0] = acc2.x / inv; o2[1] = acc2.y / inv; o2[2] = acc2.z / inv;
            }
        }
    }
    return NULL;
}

/* The adjoint from a stored path, in double precision. With w_j = albedo_j / p_j the
 * sample's radiance is sum_i T_i E_i (+ T_n env on a miss), T_i = prod_{j<i} w_j, and the
 * roulette probabilities p_j are held constant (they select the path, as in the forward
 * estimator). So dL/dE(mat of vertex i) += T_i and dL/dalbedo_k += sum_{i>k} E_i prod_{j<i, j!=k} w_j
 * / p_k: explicit products over the stored path, no replay and no division by the albedo. */
static void* adjoint_worker(void* p)
{
    render_job* J = (render_job*)p;
    const orc_render_cfg* C = J->R->C;
    const uint32_t W = C->width;
    path_rec rec;
    double T[65][3];
    for (uint32_t y = J->row0; y < J->row1; y++)
    {
        for (uint32_t x = 0; x < W; x++)
        {
            const uint32_t pix = y * W + x;
            const float* dp = J->dimg + 3 * (size_t)pix;
            const double dl[3] = { (double)dp[0] / C->spp, (double)dp[1] / C->spp, (double)dp[2] / C->spp };
            if (dl[0] == 0.0 && dl[1] == 0.0 && dl[2] == 0.0) { continue; }
            for (uint32_t s = 0; s < C->spp; s++)
            {
                (void)path_sample(J->R, x, y, C->sample_offset + s, &rec, NULL);
                const uint32_t n = rec.n;
                /* T[i] = prod_{j<i} w_j */
                for (int c = 0; c < 3; c++) { T[0][c] = 1.0; }
                for (uint32_t i = 0; i < n; i++)
                {
                    const double a[3] = { rec.v[i].albedo.x, rec.v[i].albedo.y, rec.v[i].albedo.z };
                    for (int c = 0; c < 3; c++) { T[i + 1][c] = T[i][c] * a[c] / (double)rec.v[i].p; }
                }
                if (J->g_em)
                {
                    for (uint32_t i = 0; i < n; i++)
                    {
                        double* g = J->g_em + 3 * (size_t)rec.v[i].mat;
                        for (int c = 0; c < 3; c++) { g[c] += dl[c] * T[i][c]; }
                    }
                }
                if (J->g_alb)
                {
                    for (uint32_t k = 0; k < n; k++)
                    {
                        double sum[3] = { 0.0, 0.0, 0.0 };
                        /* contributions of vertices i > k and of the environment after the last one */
                        for (uint32_t i = k + 1; i <= n; i++)
                        {
                            double e[3];
                            if (i < n) { e[0] = rec.v[i].emission.x; e[1] = rec.v[i].emission.y; e[2] = rec.v[i].emission.z; }
                            else if (rec.missed) { e[0] = rec.env.x; e[1] = rec.env.y; e[2] = rec.env.z; }
                            else { break; }
                            for (int c = 0; c < 3; c++)
                            {
                                double w = 1.0 / (double)rec.v[k].p;
                                for (uint32_t j = 0; j < i; j++)
                                {
                                    if (j == k) { continue; }
                                    const double aj = c == 0 ? rec.v[j].albedo.x : c == 1 ? rec.v[j].albedo.y : rec.v[j].albedo.z;
                                    w *= aj / (double)rec.v[j].p;
                                }
                                sum[c] += w * e[c];
                            }
                        }
                        double* g = J->g_alb + 3 * (size_t)rec.v[k].tri;
                        for (int c = 0; c < 3; c++) { g[c] += dl[c] * sum[c]; }
                    }
                }
            }
        }
    }
    return NULL;
}

static void run_rows(render_job* proto, uint32_t row0, uint32_t row1, int nthreads, void* (*fn)(void*),
                     size_t n_alb, size_t n_em)
{
    if (nthreads < 1) { nthreads = 1; }
    if (nthreads > 256) { nthreads = 256; }
    if (row0 >= row1) { return; }
    uint32_t rows = row1 - row0;
    if ((uint32_t)nthreads > rows) { nthreads = (int)rows; }
    render_job jobs[256];
    pthread_t th[256];
    uint32_t per = (rows + (uint32_t)nthreads - 1) / (uint32_t)nthreads;
    int used = 0;
    for (int t = 0; t < nthreads; t++)
    {
        uint32_t b = row0 + (uint32_t)t * per, e = b + per > row1 ? row1 : b + per;
        if (b >= e) { break; }
        render_job J = *proto;
        J.row0 = b; J.row1 = e;
        /* gradient threads accumulate privately, summed in thread order below */
        if (fn == adjoint_worker && used > 0)
        {
            J.g_alb = proto->g_alb ? (double*)calloc(n_alb, sizeof(double)) : NULL;
            J.g_em = proto->g_em ? (double*)calloc(n_em, sizeof(double)) : NULL;
        }
        jobs[used++] = J;
    }
    if (used == 1) { fn(&jobs[0]); }
    else
    {
        for (int t = 0; t < used; t++) { pthread_create(&th[t], NULL, fn, &jobs[t]); }
        for (int t = 0; t < used; t++) { pthread_join(th[t], NULL); }
    }
    if (fn == render_worker && proto->want_stats)
    {
        for (int t = 0; t < used; t++) { for (int k = 0; k < 3; k++) { proto->stats[k] += jobs[t].stats[k]; } }
    }
    if (used == 1) { return; }
    if (fn == adjoint_worker)
    {
        for (int t = 1; t < used; t++)
        {
            if (jobs[t].g_alb) { for (size_t i = 0; i < n_alb; i++) { proto->g_alb[i] += jobs[t].g_alb[i]; } free(jobs[t].g_alb); }
            if (jobs[t].g_em) { for (size_t i = 0; i < n_em; i++) { proto->g_em[i] += jobs[t].g_em[i]; } free(jobs[t].g_em); }
        }
    }
}

void orc_render_ex(const orc_bvh* B, const orc_render_cfg* C, const orc_material* mats, uint32_t n_mats,
                   const uint32_t* mot, const float* tri_albedo, const float* env_map, uint32_t env_w, uint32_t env_h,
                   uint32_t row0, uint32_t row1, float* rgb, float* rgb2, int nthreads)
{
    if (row1 > C->height) { row1 = C->height; }
    render_ctx R = { B, C, mats, mot, tri_albedo, n_mats, env_map, env_w, env_h };
    render_job P = { &R, 0, 0, rgb, rgb2, NULL, NULL, NULL, 0, { 0, 0, 0 } };
    run_rows(&P, row0, row1, nthreads, render_worker, 0, 0);
}

void orc_render_stats(const orc_bvh* B, const orc_render_cfg* C, const orc_material* mats, uint32_t n_mats,
                      const uint32_t* mot, const float* tri_albedo, const float* env_map, uint32_t env_w,
                      uint32_t env_h, uint32_t row0, uint32_t row1, float* rgb, uint64_t* counts3, int nthreads)
{
    if (row1 > C->height) { row1 = C->height; }
    render_ctx R = { B, C, mats, mot, tri_albedo, n_mats, env_map, env_w, env_h };
    render_job P = { &R, 0, 0, rgb, NULL, NULL, NULL, NULL, 1, { 0, 0, 0 } };
    run_rows(&P, row0, row1, nthreads, render_worker, 0, 0);
    for (int k = 0; k < 3; k++) { counts3[k] = P.stats[k]; }
}

void orc_render(const orc_bvh* B, const orc_render_cfg* C, const orc_material* mats, const uint32_t* mot,
                uint32_t row0, uint32_t row1, float* rgb, float* rgb2, int nthreads)
{
    orc_render_ex(B, C, mats, mats ? 0xFFFFFFFFu : 0u, mot, NULL, NULL, 0, 0, row0, row1, rgb, rgb2, nthreads);
}

void orc_adjoint(const orc_bvh* B, const orc_render_cfg* C, const orc_material* mats, uint32_t n_mats,
                 const uint32_t* mot, const float* tri_albedo, const float* d_rgb, double* grad_albedo,
                 double* grad_emission, int nthreads)
{
    render_ctx R = { B, C, mats, mot, tri_albedo, n_mats, NULL, 0, 0 };
    render_job P = { &R, 0, 0, NULL, NULL, d_rgb, grad_albedo, mats ? grad_emission : NULL, 0, { 0, 0, 0 } };
    run_rows(&P, 0, C->height, nthreads, adjoint_worker, (size_t)B->n_tris * 3, (size_t)n_mats * 3);
}
