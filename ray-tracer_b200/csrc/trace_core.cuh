// trace_core.cuh -- the traversal loop shared by the trace kernels and the path tracers:
// bvh::trace (src/bvh/bvh_traverse.cpp:91-178) over the 64-byte two-child node layout.
#pragma once

#include "device_math.cuh"
#include "rt_internal.h"

namespace rtb
{
using namespace rtd;

constexpr int STACK = 64;  // the reference's fixed stack (bvh_traverse.cpp:98)
constexpr uint32_t LEAF_BIT = 0x80000000u;
constexpr uint32_t MAX_POPS = 1u << 24;  // per ray

// rayAABB, bvh_traverse.cpp:22-41, with 1/dir precomputed (the same IEEE quotient).
__device__ __forceinline__ float ray_box(f3 o, f3 inv, float tmin, float tmax, float mnx, float mny, float mnz,
                                         float mxx, float mxy, float mxz)
{
    const float t0x = (mnx - o.x) * inv.x, t1x = (mxx - o.x) * inv.x;
    const float t0y = (mny - o.y) * inv.y, t1y = (mxy - o.y) * inv.y;
    const float t0z = (mnz - o.z) * inv.z, t1z = (mxz - o.z) * inv.z;
    const float tn = std_max(std_max(std_min(t0x, t1x), std_min(t0y, t1y)), std_max(std_min(t0z, t1z), tmin));
    const float tf = std_min(std_min(std_max(t0x, t1x), std_max(t0y, t1y)), std_min(std_max(t0z, t1z), tmax));
    return (tn <= tf) ? tn : bits2f(0x7f800000u);
}

// rayTriangle, bvh_traverse.cpp:47-87: Moller-Trumbore with back faces (a >= 0) culled.
__device__ __forceinline__ bool ray_tri(f3 o, f3 d, float tmin, float tmax, f3 v0, f3 v1, f3 v2, float& t, float& u,
                                        float& v)
{
    const f3 e1 = sub3(v1, v0), e2 = sub3(v2, v0);
    const f3 h = cross3(d, e2);
    const float a = dot3(e1, h);
    if (a >= 0) { return false; }
    const float f = 1.f / a;
    const f3 s = sub3(o, v0);
    const float uu = f * dot3(s, h);
    if (uu < 0.f || uu > 1.f) { return false; }
    const f3 q = cross3(s, e1);
    const float vv = f * dot3(d, q);
    if (vv < 0.f || uu + vv > 1.f) { return false; }
    const float tt = f * dot3(e2, q);
    if (tt < tmin || tt > tmax) { return false; }
    t = tt; u = uu; v = vv;
    return true;
}

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013), both faces, as an option:
// shear and scale into the ray's frame, edge functions U / V / W (again in double precision
// when one is exactly zero), the distance range tested on T against [tmin, tmax] * |det| with
// det's sign taken off T, and the division by det only for an accepted hit. u, v are the
// weights of v1 and v2, as in the reference's rayTriangle.
__device__ __forceinline__ bool ray_tri_watertight(f3 o, f3 d, float tmin, float tmax, f3 v0, f3 v1, f3 v2, float& t,
                                                   float& u, float& v)
{
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    if (get3(d, kz) < 0.f) { const int tmp = kx; kx = ky; ky = tmp; }
    const float dz = get3(d, kz);
    const float Sx = get3(d, kx) / dz, Sy = get3(d, ky) / dz, Sz = 1.f / dz;
    const f3 A = sub3(v0, o), Bv = sub3(v1, o), Cv = sub3(v2, o);
    const float Ax = get3(A, kx) - Sx * get3(A, kz), Ay = get3(A, ky) - Sy * get3(A, kz);
    const float Bx = get3(Bv, kx) - Sx * get3(Bv, kz), By = get3(Bv, ky) - Sy * get3(Bv, kz);
    const float Cx = get3(Cv, kx) - Sx * get3(Cv, kz), Cy = get3(Cv, ky) - Sy * get3(Cv, kz);
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.f || V == 0.f || W == 0.f)
    {
        U = (float)((double)Cx * By - (double)Cy * Bx);
        V = (float)((double)Ax * Cy - (double)Ay * Cx);
        W = (float)((double)Bx * Ay - (double)By * Ax);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) { return false; }
    const float det = U + V + W;
    if (det == 0.f) { return false; }
    const float Az = Sz * get3(A, kz), Bz = Sz * get3(Bv, kz), Cz = Sz * get3(Cv, kz);
    const float T = U * Az + V * Bz + W * Cz;
    const uint32_t sign_bit = __float_as_uint(det) & 0x80000000u;
    const float Ts = __uint_as_float(__float_as_uint(T) ^ sign_bit);
    const float Ds = __uint_as_float(__float_as_uint(det) ^ sign_bit);
    if (!(Ts >= tmin * Ds && Ts <= tmax * Ds)) { return false; }
    const float rd = 1.f / det;
    t = T * rd; u = V * rd; v = W * rd;
    return true;
}

struct TraceRoot
{
    float    box[6];
    uint32_t ref, cnt;
};

struct TraceCtx
{
    const rt_gnode*    gn;
    const float4*      tp;
    const rt_triangle* tris;
    const rt_vertex*   verts;
    const TraceRoot*   root;  // device record written by the layout kernel
    uint32_t           ww;    // 1: while-while loop (leaves of 6 or more triangles on average)
    const rt_wnode*    wn;    // the 8-wide layout (trace_ray_wide; built on request)
    const uint32_t*    wid;   // wide node index of each binary node that is a wide node
};

struct THit
{
    float    t, u, v;
    uint32_t tri;
    bool     hit, overflow;
};

// The one-loop form of the reference's traverse() (bvh_traverse.cpp:91-178): pop a node,
// re-test its entry distance against the best t, then test a leaf's triangles or push both
// children, farther first. Used for trees with small leaves, where the while-while form's
// meeting points cost more than they save.
template <int MODE, int STK>
__device__ __forceinline__ THit trace_ray_oneloop(const TraceCtx& T, const TraceRoot& R, rtd::f3 o, rtd::f3 d, float tmin,
                                                  float tmax)
{
    using namespace rtd;
    uint32_t sref[STK], scnt[STK];
    float stn[STK];
    const f3 inv = mk3(1.f / d.x, 1.f / d.y, 1.f / d.z);
    THit H;
    H.t = tmax; H.u = 0.f; H.v = 0.f; H.tri = 0; H.hit = false; H.overflow = false;
    float best = tmax;
    int top = 0;
    const float troot = ray_box(o, inv, tmin, best, R.box[0], R.box[1], R.box[2], R.box[3], R.box[4], R.box[5]);
    if (troot < best) { sref[0] = R.ref; scnt[0] = R.cnt; stn[0] = troot; top = 1; }
    uint32_t pops = 0;
    while (top > 0)
    {
        // A validated BVH is a DAG with children after parents; the cap only bounds the work
        // a malformed one could cause.
        if (++pops > MAX_POPS) { H.overflow = true; break; }
        --top;
        if (stn[top] >= best) { continue; }
        const uint32_t ref = sref[top], cnt = scnt[top];
        if (cnt & LEAF_BIT)
        {
            const uint32_t c = cnt & ~LEAF_BIT;
            bool done = false;
            for (uint32_t k = 0; k < c; k++)
            {
                const uint32_t ti = ref + k;
                const float4 p0 = __ldg(&T.tp[3 * ti]), p1 = __ldg(&T.tp[3 * ti + 1]), p2 = __ldg(&T.tp[3 * ti + 2]);
                const f3 v0 = mk3(p0.x, p0.y, p0.z), v1 = mk3(p0.w, p1.x, p1.y), v2 = mk3(p1.z, p1.w, p2.x);
                float t, u, v;
                const bool acc = (MODE & 2) ? ray_tri_watertight(o, d, tmin, tmax, v0, v1, v2, t, u, v)
                                            : ray_tri(o, d, tmin, tmax, v0, v1, v2, t, u, v);
                if (acc && t < best)
                {
                    best = t; H.u = u; H.v = v; H.tri = ti; H.hit = true;
                    if (MODE & 1) { done = true; break; }
                }
            }
            if (done) { break; }
        }
        else
        {
            const rt_gnode* g = T.gn + ref;
            const float4 a = __ldg(&g->a), b = __ldg(&g->b), c = __ldg(&g->c);
            const uint4 dd = __ldg(&g->d);
            const float tl = ray_box(o, inv, tmin, best, a.x, a.y, a.z, a.w, b.x, b.y);
            const float tr = ray_box(o, inv, tmin, best, b.z, b.w, c.x, c.y, c.z, c.w);
            // push the farther child first so the nearer one pops first; left first on ties
            uint32_t fr, fc, nr, nc;
            float ft, nt;
            if (tl <= tr) { fr = dd.y; fc = dd.w; ft = tr; nr = dd.x; nc = dd.z; nt = tl; }
            else { fr = dd.x; fc = dd.z; ft = tl; nr = dd.y; nc = dd.w; nt = tr; }
            if (ft < best)
            {
                if (top >= STK) { H.overflow = true; break; }
                sref[top] = fr; scnt[top] = fc; stn[top] = ft; top++;
            }
            if (nt < best)
            {
                if (top >= STK) { H.overflow = true; break; }
                sref[top] = nr; scnt[top] = nc; stn[top] = nt; top++;
            }
        }
    }
    H.t = best;
    return H;
}

// The while-while form (Aila & Laine, HPG 2009): an inner loop walks inner nodes
// until the current node is a leaf, then the leaf's triangles are tested; lanes of a warp meet
// after each phase, so they test leaves together instead of interleaving leaf and inner-node
// steps. The node the reference would pop next after pushing both children -- the nearer one --
// is kept in registers instead of being pushed and popped; a stack entry is one 16-byte record
// {reference, count, entry distance}. The visiting order, the pop-time test "entry distance >=
// best t" and the points where a 64-entry stack would overflow (the held node counts as its
// stack entry) are those of the one-loop form of the reference's traverse().
template <int MODE, int STK>
__device__ __forceinline__ THit trace_ray_ww(const TraceCtx& T, const TraceRoot& R, rtd::f3 o, rtd::f3 d, float tmin,
                                             float tmax)
{
    using namespace rtd;
    uint4 stk[STK];
    const f3 inv = mk3(1.f / d.x, 1.f / d.y, 1.f / d.z);
    THit H;
    H.t = tmax; H.u = 0.f; H.v = 0.f; H.tri = 0; H.hit = false; H.overflow = false;
    float best = tmax;
    int top = 0;
    uint32_t cref = R.ref, ccnt = R.cnt;
    const float troot = ray_box(o, inv, tmin, best, R.box[0], R.box[1], R.box[2], R.box[3], R.box[4], R.box[5]);
    bool have = troot < best;
    uint32_t pops = 0;
    // the next stack entry whose entry distance is below best, or none
    auto pop = [&]() {
        have = false;
        while (top > 0)
        {
            // A validated BVH is a DAG with children after parents; the cap only bounds the work
            // a malformed one could cause.
            if (++pops > MAX_POPS) { H.overflow = true; top = 0; break; }
            const uint4 e = stk[--top];
            if (__uint_as_float(e.z) < best) { cref = e.x; ccnt = e.y; have = true; break; }
        }
    };
    while (have)
    {
        // inner nodes
        while (have && !(ccnt & LEAF_BIT))
        {
            if (++pops > MAX_POPS) { H.overflow = true; have = false; break; }
            const rt_gnode* g = T.gn + cref;
            const float4 a = __ldg(&g->a), b = __ldg(&g->b), c = __ldg(&g->c);
            const uint4 dd = __ldg(&g->d);
            const float tl = ray_box(o, inv, tmin, best, a.x, a.y, a.z, a.w, b.x, b.y);
            const float tr = ray_box(o, inv, tmin, best, b.z, b.w, c.x, c.y, c.z, c.w);
            // the farther child waits on the stack, the nearer one is next; left first on ties
            uint32_t fr, fc, nr, nc;
            float ft, nt;
            if (tl <= tr) { fr = dd.y; fc = dd.w; ft = tr; nr = dd.x; nc = dd.z; nt = tl; }
            else { fr = dd.x; fc = dd.z; ft = tl; nr = dd.y; nc = dd.w; nt = tr; }
            if (nt < best)  // (the farther child is hit only if the nearer one is)
            {
                if (ft < best)
                {
                    if (top >= STK) { H.overflow = true; have = false; break; }
                    stk[top++] = make_uint4(fr, fc, __float_as_uint(ft), 0u);
                }
                if (top >= STK) { H.overflow = true; have = false; break; }
                cref = nr; ccnt = nc;
            }
            else { pop(); }
        }
        if (!have) { break; }
        // a leaf: its triangles in order, strict "t < best" (bvh_traverse.cpp:112-142)
        const uint32_t cnt = ccnt & ~LEAF_BIT;
        bool done = false;
        for (uint32_t k = 0; k < cnt; k++)
        {
            const uint32_t ti = cref + k;
            const float4 p0 = __ldg(&T.tp[3 * ti]), p1 = __ldg(&T.tp[3 * ti + 1]), p2 = __ldg(&T.tp[3 * ti + 2]);
            const f3 v0 = mk3(p0.x, p0.y, p0.z), v1 = mk3(p0.w, p1.x, p1.y), v2 = mk3(p1.z, p1.w, p2.x);
            float t, u, v;
            const bool acc = (MODE & 2) ? ray_tri_watertight(o, d, tmin, tmax, v0, v1, v2, t, u, v)
                                        : ray_tri(o, d, tmin, tmax, v0, v1, v2, t, u, v);
            if (acc && t < best)
            {
                best = t; H.u = u; H.v = v; H.tri = ti; H.hit = true;
                if (MODE & 1) { done = true; break; }
            }
        }
        if (done) { break; }
        pop();
    }
    H.t = best;
    return H;
}

// Traversal of the 8-wide layout (wide.cu). A visited wide node's eight child boxes are decoded
// and tested at once; the node goes on the stack as one entry {node, mask of the children hit}
// with the mask in the ray's visiting order -- the builder puts children in octant slots, and a
// ray whose direction has the signs o visits slot s as its (s ^ o)-th, near to far along each
// axis -- and each step takes the next child from the top entry: a leaf's triangles are tested
// in order, an inner child is visited. The closest hit's distance is that of the binary
// traversal; on an exact tie in distance the triangle found first may differ, since the
// visiting order differs, and a triangle the binary boxes cull may be found: the conservative
// child boxes admit one an exact box test rejects by rounding at a face, and the boxes of the
// collapsed binary levels are not tested (with spatial splits they need not contain their
// children's). Not the reference's order: an opt-in form.
template <int MODE, int STK>
__device__ __forceinline__ THit trace_ray_wide(const TraceCtx& T, const TraceRoot& R, rtd::f3 o, rtd::f3 d, float tmin,
                                               float tmax)
{
    using namespace rtd;
    uint2 stk[STK];  // {wide node, remaining children hit, in visiting order}
    const f3 inv = mk3(1.f / d.x, 1.f / d.y, 1.f / d.z);
    const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    THit H;
    H.t = tmax; H.u = 0.f; H.v = 0.f; H.tri = 0; H.hit = false; H.overflow = false;
    float best = tmax;
    int top = 0;
    const float troot = ray_box(o, inv, tmin, best, R.box[0], R.box[1], R.box[2], R.box[3], R.box[4], R.box[5]);
    if (!(troot < best)) { return H; }
    // the entry to visit: a wide node (cnt 0) or a leaf's triangle range
    uint32_t cref = (R.cnt & LEAF_BIT) ? R.ref : __ldg(&T.wid[R.ref]);
    uint32_t ccnt = R.cnt;
    bool have = true;
    uint32_t pops = 0;
    for (;;)
    {
        if (++pops > MAX_POPS) { H.overflow = true; break; }
        if (have)
        {
            have = false;
            if (ccnt & LEAF_BIT)
            {
                const uint32_t c = ccnt & ~LEAF_BIT;
                bool done = false;
                for (uint32_t k = 0; k < c; k++)
                {
                    const uint32_t ti = cref + k;
                    const float4 p0 = __ldg(&T.tp[3 * ti]), p1 = __ldg(&T.tp[3 * ti + 1]), p2 = __ldg(&T.tp[3 * ti + 2]);
                    const f3 v0 = mk3(p0.x, p0.y, p0.z), v1 = mk3(p0.w, p1.x, p1.y), v2 = mk3(p1.z, p1.w, p2.x);
                    float t, u, v;
                    const bool acc = (MODE & 2) ? ray_tri_watertight(o, d, tmin, tmax, v0, v1, v2, t, u, v)
                                                : ray_tri(o, d, tmin, tmax, v0, v1, v2, t, u, v);
                    if (acc && t < best)
                    {
                        best = t; H.u = u; H.v = v; H.tri = ti; H.hit = true;
                        if (MODE & 1) { done = true; break; }
                    }
                }
                if (done) { break; }
            }
            else
            {
                const uint4* g = reinterpret_cast<const uint4*>(T.wn + cref);
                const uint4 w0 = __ldg(g), w3 = __ldg(g + 3), w4 = __ldg(g + 4), w5 = __ldg(g + 5), w6 = __ldg(g + 6);
                const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
                const float sx = __uint_as_float((w0.w & 0xffu) << 23), sy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23),
                            sz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23);
                const uint32_t cn[4] = { w3.x, w3.y, w3.z, w3.w };  // two 16-bit counts per word
                uint32_t mask = 0;
#pragma unroll
                for (int c = 0; c < 8; c++)
                {
                    const uint32_t cc = (cn[c >> 1] >> (16 * (c & 1))) & 0xffffu;
                    const int sb = 8 * (c & 3);
                    const uint32_t lx = ((c < 4 ? w4.x : w4.y) >> sb) & 0xffu, ly = ((c < 4 ? w4.z : w4.w) >> sb) & 0xffu;
                    const uint32_t lz = ((c < 4 ? w5.x : w5.y) >> sb) & 0xffu, hx = ((c < 4 ? w5.z : w5.w) >> sb) & 0xffu;
                    const uint32_t hy = ((c < 4 ? w6.x : w6.y) >> sb) & 0xffu, hz = ((c < 4 ? w6.z : w6.w) >> sb) & 0xffu;
                    // the decoded planes (the layout builder checks these very operations are conservative)
                    const float bx0 = __fadd_rn(px, __fmul_rn((float)lx, sx)), bx1 = __fadd_rn(px, __fmul_rn((float)hx, sx));
                    const float by0 = __fadd_rn(py, __fmul_rn((float)ly, sy)), by1 = __fadd_rn(py, __fmul_rn((float)hy, sy));
                    const float bz0 = __fadd_rn(pz, __fmul_rn((float)lz, sz)), bz1 = __fadd_rn(pz, __fmul_rn((float)hz, sz));
                    const float t = ray_box(o, inv, tmin, best, bx0, by0, bz0, bx1, by1, bz1);
                    if (cc != 0u && t < best) { mask |= 1u << ((uint32_t)c ^ oct); }
                }
                if (mask)
                {
                    if (top >= STK) { H.overflow = true; break; }
                    stk[top++] = make_uint2(cref, mask);
                }
            }
        }
        if (top == 0) { break; }
        // the next child of the top entry
        uint2& e = stk[top - 1];
        const uint32_t k = (uint32_t)__ffs((int)e.y) - 1u;
        const uint32_t node = e.x;
        e.y &= e.y - 1u;
        if (e.y == 0u) { --top; }
        const uint32_t c = k ^ oct;
        const rt_wnode* wn = T.wn + node;
        cref = __ldg(&wn->ref[c]);
        ccnt = ((__ldg(&wn->meta) >> (24 + c)) & 1u) ? 0u : (LEAF_BIT | (uint32_t)__ldg(&wn->cnt[c]));
        have = true;
    }
    H.t = best;
    return H;
}

// Closest hit (MODE bit 0 clear) or first accepted hit (bit 0 set); bit 1 selects the
// watertight triangle test. Reproduces the reference's visiting order exactly, in either loop
// form (T.ww picks one per tree; both visit the same nodes in the same order). STK entries of
// stack: the loop holds at most one entry per level of the tree plus one, so a stack deeper
// than the tree never overflows (overflow is reported, never silent). R: the subtree to trace.
template <int MODE, int STK = STACK>
__device__ __forceinline__ THit trace_ray(const TraceCtx& T, const TraceRoot& R, rtd::f3 o, rtd::f3 d, float tmin,
                                          float tmax)
{
    return T.ww ? trace_ray_ww<MODE, STK>(T, R, o, d, tmin, tmax) : trace_ray_oneloop<MODE, STK>(T, R, o, d, tmin, tmax);
}

// The whole tree (the handle's root record).
template <int MODE, int STK = STACK>
__device__ __forceinline__ THit trace_ray(const TraceCtx& T, rtd::f3 o, rtd::f3 d, float tmin, float tmax)
{
    const TraceRoot R = *T.root;
    return trace_ray<MODE, STK>(T, R, o, d, tmin, tmax);
}

// Interpolated shading normal of a hit: normalize(w n0 + u n1 + v n2), bvh_traverse.cpp:135-139.
__device__ __forceinline__ rtd::f3 hit_normal(const TraceCtx& T, uint32_t tri, float u, float v)
{
    using namespace rtd;
    const rt_triangle tr = T.tris[tri];
    const rt_vertex& a = T.verts[tr.v[0]];
    const rt_vertex& b = T.verts[tr.v[1]];
    const rt_vertex& c = T.verts[tr.v[2]];
    const float w = 1.f - u - v;
    const f3 nn = add3(add3(muls(mk3(a.nx, a.ny, a.nz), w), muls(mk3(b.nx, b.ny, b.nz), u)), muls(mk3(c.nx, c.ny, c.nz), v));
    return norm3(nn);
}

TraceCtx make_trace_ctx(const rt_bvh* B);

} // namespace rtb
