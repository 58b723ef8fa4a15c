// device_math.cuh -- float helpers with the exact semantics of the reference's x86-64 build.
//
// The reference evaluates every float expression in SSE single precision with no FMA
// contraction; this library is compiled with -fmad=false and IEEE division / square root,
// and the helpers below keep the reference's operand order, so device results are bit
// identical to the reference's. The min/max helpers reproduce the exact NaN and signed-zero
// behaviour of the two flavours the reference mixes:
//   sse_min/sse_max  -- SSE minps/maxps (math::min / math::max, src/math/vec3.hpp:72-73):
//                       the second operand unless the first is strictly smaller / larger;
//   std_min/std_max  -- std::min / std::max (src/bvh/bvh_traverse.cpp:36-37, bvh_sah.cpp).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define RT_HD __host__ __device__ __forceinline__

namespace rtd
{

RT_HD float bits2f(uint32_t u)
{
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f; __builtin_memcpy(&f, &u, 4); return f;
#endif
}
RT_HD uint32_t f2bits(float f)
{
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u; __builtin_memcpy(&u, &f, 4); return u;
#endif
}

RT_HD float sse_min(float a, float b) { return a < b ? a : b; }
RT_HD float sse_max(float a, float b) { return a > b ? a : b; }
RT_HD float std_min(float a, float b) { return (b < a) ? b : a; }
RT_HD float std_max(float a, float b) { return (a < b) ? b : a; }
RT_HD int   std_mini(int a, int b) { return (b < a) ? b : a; }
RT_HD int   std_clampi(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }

// float -> int32 as x86-64 cvttss2si: truncation; INT32_MIN for NaN and out-of-range
// values (the (int) casts of src/bvh/bvh_sah.cpp:85,179-180).
RT_HD int x86_f2i(float f)
{
    if (!(f > -2147483904.0f && f < 2147483648.0f)) { return (int)0x80000000u; }
    return (int)f;
}
// float -> uint32 as g++ emits it on x86-64 (64-bit cvttss2si, low word kept): the (uint)
// cast of src/bvh/bvh_morton.cpp:78.
RT_HD uint32_t x86_f2u(float f)
{
    long long v;
    if (!(f > -9223373136366403584.0f && f < 9223372036854775808.0f)) { v = (long long)0x8000000000000000ull; }
    else { v = (long long)f; }
    return (uint32_t)(unsigned long long)v;
}

struct f3 { float x, y, z; };

RT_HD f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
RT_HD f3 add3(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
RT_HD f3 sub3(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
RT_HD f3 mul3(f3 a, f3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
RT_HD f3 muls(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
RT_HD f3 divs(f3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
// dot of src/math/vec3.hpp:42-50: (x*x' + y*y') + (z*z' + w*w'), the padding lane w = 0.
RT_HD float dot3(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + (a.z * b.z + 0.0f); }
// cross of src/math/vec3.hpp:52-59
RT_HD f3 cross3(f3 a, f3 b) { return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
// normalize of src/math/vec3.hpp:66-70 (IEEE sqrt and division)
RT_HD f3 norm3(f3 v)
{
    float inv = 1.0f / sqrtf(dot3(v, v));
    return muls(v, inv);
}
RT_HD float get3(f3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

// AABB with the reference's empty box (+inf / -inf), src/bvh/AABB.cpp:4-60
struct box3 { float mn[3], mx[3]; };

RT_HD box3 box_empty()
{
    box3 b;
    for (int k = 0; k < 3; k++) { b.mn[k] = bits2f(0x7f800000u); b.mx[k] = bits2f(0xff800000u); }
    return b;
}
RT_HD void box_pt(box3& b, f3 p)
{
    b.mn[0] = sse_min(b.mn[0], p.x); b.mn[1] = sse_min(b.mn[1], p.y); b.mn[2] = sse_min(b.mn[2], p.z);
    b.mx[0] = sse_max(b.mx[0], p.x); b.mx[1] = sse_max(b.mx[1], p.y); b.mx[2] = sse_max(b.mx[2], p.z);
}
RT_HD void box_box(box3& b, const box3& o)
{
    for (int k = 0; k < 3; k++) { b.mn[k] = sse_min(b.mn[k], o.mn[k]); b.mx[k] = sse_max(b.mx[k], o.mx[k]); }
}
// half_area, src/bvh/AABB.cpp:29-33
RT_HD float box_half_area(const box3& b)
{
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    return dx * dy + dy * dz + dz * dx;
}
RT_HD bool box_valid(const box3& b) { return b.mn[0] <= b.mx[0] && b.mn[1] <= b.mx[1] && b.mn[2] <= b.mx[2]; }

// clipTriangleToAABB, src/bvh/AABB.cpp:86-171: Sutherland-Hodgman clip of the triangle
// against the min then the max plane of x, y and z; returns the clipped polygon's box or
// the empty box. At most 9 polygon vertices are live; 12 slots as in the reference. This is
// the general form, with the polygon in indexed arrays; clip_triangle below computes the same
// result in registers for the usual cases and falls back to it.
RT_HD box3 clip_triangle_general(f3 v0, f3 v1, f3 v2, const box3& region)
{
    // All three vertices inside the region: no plane removes or adds a vertex, so the clipped
    // polygon is the triangle and its box the vertices' box (the loop below would return the
    // same values).
    {
        bool inside = true;
        const f3 vs[3] = { v0, v1, v2 };
        for (int i = 0; i < 3; i++)
        {
            for (int axis = 0; axis < 3; axis++)
            {
                const float c = get3(vs[i], axis);
                inside = inside && (c >= region.mn[axis]) && (c <= region.mx[axis]);
            }
        }
        if (inside)
        {
            box3 r = box_empty();
            box_pt(r, v0); box_pt(r, v1); box_pt(r, v2);
            return r;
        }
    }
    f3 poly[12], tmp[12];
    int n = 3;
    poly[0] = v0; poly[1] = v1; poly[2] = v2;
    for (int axis = 0; axis < 3; axis++)
    {
        for (int side = 0; side < 2; side++)
        {
            const float plane = side == 0 ? region.mn[axis] : region.mx[axis];
            int m = 0;
            for (int i = 0; i < n; i++)
            {
                const int nx = (i + 1 == n) ? 0 : i + 1;
                const float pi = get3(poly[i], axis), pn = get3(poly[nx], axis);
                const bool cin = side == 0 ? (pi >= plane) : (pi <= plane);
                const bool nin = side == 0 ? (pn >= plane) : (pn <= plane);
                if (cin) { tmp[m++] = poly[i]; }
                if (cin != nin)
                {
                    const float t = (plane - pi) / (pn - pi);
                    tmp[m++] = add3(poly[i], muls(sub3(poly[nx], poly[i]), t));
                }
            }
            for (int i = 0; i < m; i++) { poly[i] = tmp[i]; }
            n = m;
            if (n == 0) { return box_empty(); }
        }
    }
    box3 r = box_empty();
    for (int i = 0; i < n; i++) { box_pt(r, poly[i]); }
    return r;
}

RT_HD float sel3(float x, float y, float z, int axis) { return axis == 0 ? x : (axis == 1 ? y : z); }

// One Sutherland-Hodgman step (the loop body of clip_triangle_general for one plane) on a
// polygon of at most 4 vertices held in registers; the result has at most 5.
RT_HD void clip_step4(float (&px)[5], float (&py)[5], float (&pz)[5], int& n, int axis, int side, float plane)
{
    float qx[5] = { 0.f, 0.f, 0.f, 0.f, 0.f }, qy[5] = { 0.f, 0.f, 0.f, 0.f, 0.f }, qz[5] = { 0.f, 0.f, 0.f, 0.f, 0.f };
    int m = 0;
    auto push = [&](float x, float y, float z) {
#pragma unroll
        for (int k = 0; k < 5; k++)
        {
            if (k == m) { qx[k] = x; qy[k] = y; qz[k] = z; }
        }
        m++;
    };
#pragma unroll
    for (int i = 0; i < 4; i++)
    {
        if (i < n)
        {
            const bool last = i + 1 == n;
            const f3 a = mk3(px[i], py[i], pz[i]);
            const f3 b = last ? mk3(px[0], py[0], pz[0]) : mk3(px[i + 1], py[i + 1], pz[i + 1]);
            const float pi = sel3(a.x, a.y, a.z, axis), pn = sel3(b.x, b.y, b.z, axis);
            const bool cin = side == 0 ? (pi >= plane) : (pi <= plane);
            const bool nin = side == 0 ? (pn >= plane) : (pn <= plane);
            if (cin) { push(a.x, a.y, a.z); }
            if (cin != nin)
            {
                const float t = (plane - pi) / (pn - pi);
                const f3 r = add3(a, muls(sub3(b, a), t));
                push(r.x, r.y, r.z);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 5; k++) { px[k] = qx[k]; py[k] = qy[k]; pz[k] = qz[k]; }
    n = m;
}

// clip_triangle_general's result with the polygon in registers: a plane every vertex lies
// inside leaves the polygon as it is (no vertex dropped, no crossing), so it is skipped; the
// planes that cut are applied while the polygon has at most 4 vertices (so at most 5 after),
// and anything larger is handed to the general form.
RT_HD box3 clip_triangle(f3 v0, f3 v1, f3 v2, const box3& region)
{
    float px[5] = { v0.x, v1.x, v2.x, 0.f, 0.f }, py[5] = { v0.y, v1.y, v2.y, 0.f, 0.f },
          pz[5] = { v0.z, v1.z, v2.z, 0.f, 0.f };
    int n = 3;
    for (int pl = 0; pl < 6; pl++)
    {
        const int axis = pl >> 1, side = pl & 1;
        const float plane = side == 0 ? sel3(region.mn[0], region.mn[1], region.mn[2], axis)
                                      : sel3(region.mx[0], region.mx[1], region.mx[2], axis);
        bool allin = true;
#pragma unroll
        for (int i = 0; i < 5; i++)
        {
            if (i < n)
            {
                const float c = sel3(px[i], py[i], pz[i], axis);
                allin = allin && (side == 0 ? (c >= plane) : (c <= plane));
            }
        }
        if (allin) { continue; }
        if (n > 4) { return clip_triangle_general(v0, v1, v2, region); }
        clip_step4(px, py, pz, n, axis, side, plane);
        if (n == 0) { return box_empty(); }
    }
    box3 r = box_empty();
#pragma unroll
    for (int i = 0; i < 5; i++)
    {
        if (i < n) { box_pt(r, mk3(px[i], py[i], pz[i])); }
    }
    return r;
}

// Order-preserving float <-> uint32 map for atomicMin / atomicMax reductions of boxes.
// It orders -0 below +0; the reference's order-dependent choice between them is
// value-equal, and the .bvh comparisons of this library treat them as equal.
RT_HD uint32_t f2ord(float f)
{
    uint32_t u = f2bits(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
RT_HD float ord2f(uint32_t u)
{
    return bits2f((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

} // namespace rtd
