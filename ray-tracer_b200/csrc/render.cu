// render.cu -- the per-sample path loop: pathTrace and the pixel loop of the reference
// (src/main.cpp:69-204, 323-365), with a counter-based per-pixel RNG instead of the one global
// std::mt19937 stream, and the material extensions the benchmark scenes need (per-triangle
// albedo, emitters, mirrors; the reference has albedo 0.8 and no emitters).
//
// Two schedules compute the same samples from the same random numbers:
//  RT_RENDER_PLAIN      one thread per pixel runs all its samples (the reference's loop order,
//                       so the per-pixel sums add up in sample order);
//  RT_RENDER_WAVEFRONT  generate / extend / shade queues: all paths of a chunk of samples advance
//                       one bounce per step; extend is the persistent trace kernel over the
//                       compacted ray queue, shade writes the next queue and retires finished
//                       paths into the image with atomics.
// The wavefront also renders the scenes of a batched build together (rt_render_batch): a path
// carries its scene, extend traces it from that scene's root, and each scene has its own
// camera and seed, so scene s of a batch gets the samples a render of scene s alone gets. Its
// launch sequence is replayed from a CUDA graph captured once per configuration, and its
// block size, queue chunk and stack depth can be chosen by rt_autotune_wavefront.
//
// Random numbers: Philox4x32-10 (Salmon et al., SC'11) keyed by (seed, 0x5EED), counter
// (pixel, sample, 0, 0) for the pixel jitter and (pixel, sample, bounce + 1, 0) for the
// bounce's direction and Russian roulette draws.
//
// Adjoint (no counterpart in the reference): gradients of sum(dL/dI * I) with respect to the
// albedo used at each triangle and each material's emission, by path-replay backpropagation
// (Vicini, Speierer, Jakob: "Path Replay Backpropagation", SIGGRAPH 2021). Per sample, a first
// pass computes the path's radiance L; a second pass re-traces the same path from the same
// counter-based random numbers, and at vertex k the radiance still to come,
// L - sum_{i<=k} T_i E_i, divided by the albedo there is dL/dalbedo_k. The RNG is recomputed,
// not stored, so memory stays O(pixels). Russian-roulette probabilities are held constant.
#include "trace_core.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace rtb
{

// camera basis and RNG key of one scene (src/main.cpp:43-83)
struct Cam
{
    float    pos[3], fwd[3], right[3], up[3];
    float    th;
    uint32_t seed;
};

namespace
{

struct RP
{
    uint32_t W, H, spp, max_bounce;
    int32_t  rr_after;
    uint32_t env_kind;
    float    env[3];
    Cam      cam;
    uint32_t sample_offset;
    uint32_t env_w, env_h;
    const float* env_map;
};

__device__ __forceinline__ uint4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++)
    {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return make_uint4(c0, c1, c2, c3);
}
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// Shading inputs (all optional): materials, the material of each baked triangle, and an RGB
// albedo per baked triangle that replaces the material's.
struct Shade
{
    const rt_material* mats;
    const uint32_t*    mot;
    const float*       talb;
    uint32_t           n_mats;
};

struct Surf
{
    f3       albedo, emission;
    uint32_t kind, mat;
};

__device__ __forceinline__ Surf surface(const Shade& S, uint32_t tri)
{
    Surf r;
    r.albedo = mk3(0.8f, 0.8f, 0.8f);
    r.emission = mk3(0.f, 0.f, 0.f);
    r.kind = 0; r.mat = 0;
    if (S.mats)
    {
        const uint32_t m = min(S.mot ? S.mot[tri] : 0u, S.n_mats - 1u);
        const rt_material M = S.mats[m];
        r.albedo = mk3(M.albedo[0], M.albedo[1], M.albedo[2]);
        r.emission = mk3(M.emission[0], M.emission[1], M.emission[2]);
        r.kind = M.kind; r.mat = m;
    }
    if (S.talb) { r.albedo = mk3(S.talb[3 * tri], S.talb[3 * tri + 1], S.talb[3 * tri + 2]); }
    return r;
}

constexpr float kPi = 3.14159265358979323846f;

// primaryRay, src/main.cpp:69-83
__device__ __forceinline__ void primary(const RP& P, const Cam& C, uint32_t x, uint32_t y, uint32_t pix, uint32_t sidx,
                                        f3& o, f3& d)
{
    const uint4 r = philox(pix, sidx, 0u, 0u, C.seed, 0x5EEDu);
    const float aspect = (float)P.W / (float)P.H;
    const float u = (((float)x + u01(r.x)) / (float)P.W * 2.f - 1.f) * aspect;
    const float v = ((float)y + u01(r.y)) / (float)P.H * 2.f - 1.f;
    const f3 fwd = mk3(C.fwd[0], C.fwd[1], C.fwd[2]);
    const f3 rgt = mk3(C.right[0], C.right[1], C.right[2]);
    const f3 up = mk3(C.up[0], C.up[1], C.up[2]);
    o = mk3(C.pos[0], C.pos[1], C.pos[2]);
    d = norm3(add3(add3(fwd, muls(rgt, u * C.th)), muls(up, v * C.th)));
}

// background (src/main.cpp:162-173); env_kind 2: IBL::sample (main.cpp:107-117), the
// nearest texel of an equirectangular map
__device__ __forceinline__ f3 environment(const RP& P, f3 d)
{
    if (P.env_kind == 0)
    {
        const float t = d.y * 0.5f + 0.5f;
        return add3(muls(mk3(1.0f, 1.0f, 1.0f), 1.f - t), muls(mk3(0.5f, 0.7f, 1.0f), t));
    }
    if (P.env_kind == 2)
    {
        const float phi = atan2f(d.z, d.x);
        const float y = d.y < -1.f ? -1.f : (1.f < d.y ? 1.f : d.y);  // std::clamp
        const float theta = acosf(y);
        const float u = (phi + kPi) / (2.f * kPi);
        const float v = theta / kPi;
        const int px = min((int)(u * (float)P.env_w), (int)P.env_w - 1);
        const int py = min((int)(v * (float)P.env_h), (int)P.env_h - 1);
        const float* p = P.env_map + ((size_t)py * P.env_w + px) * 3;
        return mk3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
    }
    return mk3(P.env[0], P.env[1], P.env[2]);
}

// One bounce at a hit (src/main.cpp:178-200) after the emission of the surface was added:
// the next direction (cosine hemisphere about the shading normal, or the mirror direction),
// throughput update and Russian roulette. Returns false when roulette ends the path.
__device__ __forceinline__ bool scatter(const RP& P, uint32_t seed, const Surf& sf, f3 n, f3 din, uint32_t pix,
                                        uint32_t sidx, uint32_t bounce, f3& tp, f3& dout)
{
    const uint4 r = philox(pix, sidx, bounce + 1u, 0u, seed, 0x5EEDu);
    if (sf.kind == 1)
    {
        dout = sub3(din, muls(n, 2.f * dot3(din, n)));
    }
    else
    {
        // sampleCosineHemisphere + toWorld, src/main.cpp:123-141
        const float u1 = u01(r.x), u2 = u01(r.y);
        const float rr = sqrtf(u1);
        const float theta = 2.f * kPi * u2;
        const f3 ld = mk3(rr * cosf(theta), sqrtf(std_max(0.f, 1.f - u1)), rr * sinf(theta));
        const f3 axis = fabsf(n.x) < 0.9f ? mk3(1.f, 0.f, 0.f) : mk3(0.f, 1.f, 0.f);
        const f3 t = norm3(cross3(n, axis));
        const f3 b = cross3(n, t);
        dout = add3(add3(muls(t, ld.x), muls(n, ld.y)), muls(b, ld.z));
    }
    tp = mul3(tp, sf.albedo);
    if (P.rr_after >= 0 && (int32_t)bounce > P.rr_after)
    {
        const float p = std_max(std_max(tp.x, tp.y), tp.z);
        if (u01(r.z) > p) { return false; }
        tp = divs(tp, p);
    }
    return true;
}

// The radiance of one sample of one pixel (primaryRay + pathTrace).
__device__ __forceinline__ f3 path_sample(const TraceCtx& T, const RP& P, const Shade& S, uint32_t x, uint32_t y,
                                          uint32_t pix, uint32_t sidx)
{
    f3 o, d;
    primary(P, P.cam, x, y, pix, sidx, o, d);
    float tmin = 1e-3f;
    f3 tp = mk3(1.f, 1.f, 1.f), L = mk3(0.f, 0.f, 0.f);
    for (uint32_t bounce = 0; bounce <= P.max_bounce; bounce++)
    {
        const THit H = trace_ray<0>(T, o, d, tmin, bits2f(0x7f800000u));
        if (!H.hit)
        {
            L = add3(L, mul3(tp, environment(P, d)));
            break;
        }
        const Surf sf = surface(S, H.tri);
        L = add3(L, mul3(tp, sf.emission));
        const f3 n = hit_normal(T, H.tri, H.u, H.v);
        f3 nd;
        if (!scatter(P, P.cam.seed, sf, n, d, pix, sidx, bounce, tp, nd)) { break; }
        o = add3(o, muls(d, H.t));
        d = nd;
        tmin = 1e-4f;
    }
    return L;
}

__global__ void __launch_bounds__(128)
k_render_plain(TraceCtx T, RP P, Shade S, float* __restrict__ rgb, float* __restrict__ rgb2)
{
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= P.W || y >= P.H) { return; }
    const uint32_t pix = y * P.W + x;
    f3 acc = mk3(0.f, 0.f, 0.f), acc2 = mk3(0.f, 0.f, 0.f);
    for (uint32_t s = 0; s < P.spp; s++)
    {
        const f3 L = path_sample(T, P, S, x, y, pix, P.sample_offset + s);
        acc = add3(acc, L);
        acc2 = add3(acc2, mul3(L, L));
    }
    const float fs = (float)P.spp;
    rgb[3 * pix] = acc.x / fs; rgb[3 * pix + 1] = acc.y / fs; rgb[3 * pix + 2] = acc.z / fs;
    if (rgb2) { rgb2[3 * pix] = acc2.x / fs; rgb2[3 * pix + 1] = acc2.y / fs; rgb2[3 * pix + 2] = acc2.z / fs; }
}

// dst[3 key + c] += v.c for every lane with `valid`, lanes of the warp with equal keys summed
// first so each distinct key costs one set of atomics per warp. All 32 lanes must call it.
__device__ __forceinline__ void warp_add3(float* __restrict__ dst, uint32_t key, bool valid, f3 v)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t k = valid ? key : 0xFFFFFFFFu;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, k);
    bool pending = valid && __popc(peers) > 1;
    if (valid && !pending)
    {
        atomicAdd(&dst[3 * (size_t)key], v.x); atomicAdd(&dst[3 * (size_t)key + 1], v.y); atomicAdd(&dst[3 * (size_t)key + 2], v.z);
    }
    uint32_t pend = __ballot_sync(0xFFFFFFFFu, pending);
    while (pend)
    {
        const int ldr = __ffs(pend) - 1;
        const uint32_t lk = __shfl_sync(0xFFFFFFFFu, k, ldr);
        const bool in = pending && k == lk;
        float sx = in ? v.x : 0.f, sy = in ? v.y : 0.f, sz = in ? v.z : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            sx += __shfl_xor_sync(0xFFFFFFFFu, sx, o);
            sy += __shfl_xor_sync(0xFFFFFFFFu, sy, o);
            sz += __shfl_xor_sync(0xFFFFFFFFu, sz, o);
        }
        if ((int)lane == ldr)
        {
            atomicAdd(&dst[3 * (size_t)key], sx); atomicAdd(&dst[3 * (size_t)key + 1], sy); atomicAdd(&dst[3 * (size_t)key + 2], sz);
        }
        if (in) { pending = false; }
        pend = __ballot_sync(0xFFFFFFFFu, pending);
    }
}

// Path-replay adjoint, one thread per pixel (the plain schedule). Lanes run the replay's
// bounce loop in step so the gradient adds can be combined per warp; pixels whose dL/dI is
// zero are skipped.
__global__ void __launch_bounds__(128)
k_adjoint(TraceCtx T, RP P, Shade S, const float* __restrict__ dimg, float* __restrict__ g_alb, float* __restrict__ g_em)
{
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 4);
    const bool in_img = x < P.W && y < P.H;
    const uint32_t pix = in_img ? y * P.W + x : 0u;
    const float fs = (float)P.spp;
    f3 dl = mk3(0.f, 0.f, 0.f);
    if (in_img) { dl = mk3(dimg[3 * pix] / fs, dimg[3 * pix + 1] / fs, dimg[3 * pix + 2] / fs); }
    const bool act = in_img && (dl.x != 0.f || dl.y != 0.f || dl.z != 0.f);
    if (!__any_sync(0xFFFFFFFFu, act)) { return; }
    for (uint32_t s = 0; s < P.spp; s++)
    {
        const uint32_t sidx = P.sample_offset + s;
        f3 Ltot = mk3(0.f, 0.f, 0.f);
        if (act) { Ltot = path_sample(T, P, S, x, y, pix, sidx); }
        // replay
        f3 o = mk3(0.f, 0.f, 0.f), d = mk3(0.f, 0.f, 1.f);
        if (act) { primary(P, P.cam, x, y, pix, sidx, o, d); }
        float tmin = 1e-3f;
        f3 tp = mk3(1.f, 1.f, 1.f), Ssum = mk3(0.f, 0.f, 0.f);
        bool alive = act;
        for (uint32_t bounce = 0; bounce <= P.max_bounce; bounce++)
        {
            if (!__any_sync(0xFFFFFFFFu, alive)) { break; }
            bool hv = false;
            uint32_t tri = 0, mat = 0;
            f3 ga = mk3(0.f, 0.f, 0.f), ge = mk3(0.f, 0.f, 0.f);
            if (alive)
            {
                const THit H = trace_ray<0>(T, o, d, tmin, bits2f(0x7f800000u));
                if (!H.hit) { alive = false; }
                else
                {
                    const Surf sf = surface(S, H.tri);
                    hv = true; tri = H.tri; mat = sf.mat;
                    ge = mul3(dl, tp);
                    Ssum = add3(Ssum, mul3(tp, sf.emission));
                    const f3 rest = sub3(Ltot, Ssum);
                    ga = mk3(sf.albedo.x != 0.f ? dl.x * rest.x / sf.albedo.x : 0.f,
                             sf.albedo.y != 0.f ? dl.y * rest.y / sf.albedo.y : 0.f,
                             sf.albedo.z != 0.f ? dl.z * rest.z / sf.albedo.z : 0.f);
                    const f3 n = hit_normal(T, H.tri, H.u, H.v);
                    f3 nd;
                    if (!scatter(P, P.cam.seed, sf, n, d, pix, sidx, bounce, tp, nd) || bounce >= P.max_bounce)
                    {
                        alive = false;
                    }
                    o = add3(o, muls(d, H.t));
                    d = nd;
                    tmin = 1e-4f;
                }
            }
            if (g_alb) { warp_add3(g_alb, tri, hv, ga); }
            if (g_em) { warp_add3(g_em, mat, hv && S.mats != nullptr, ge); }
        }
    }
}

// ---- wavefront ----
// ray queue: rt_ray records (o, tmin, d, tmax); path state: (tp.xyz, image pixel), (L.xyz,
// sample); scene queue: the scene of each ray (batched renders). Image pixel = scene * W * H
// + pixel of the scene. Paths are numbered sample-major: g = (sample * S + scene) * W * H + pixel.

__global__ void __launch_bounds__(256)
k_wf_generate(RP P, const Cam* __restrict__ cams, uint32_t S, uint64_t g0, uint32_t n_paths, float4* __restrict__ rays,
              float4* __restrict__ state, uint32_t* __restrict__ rscene, uint32_t* __restrict__ count)
{
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i == 0) { *count = n_paths; }
    if (i >= n_paths) { return; }
    const uint64_t npix = (uint64_t)P.W * P.H;
    const uint64_t g = g0 + i;
    const uint32_t s = (uint32_t)(g / (npix * S));
    const uint64_t rem = g - (uint64_t)s * npix * S;
    const uint32_t sc = (uint32_t)(rem / npix);
    const uint32_t pix = (uint32_t)(rem - (uint64_t)sc * npix);
    const uint32_t x = pix % P.W, y = pix / P.W;
    const Cam C = cams ? cams[sc] : P.cam;
    f3 o, d;
    primary(P, C, x, y, pix, P.sample_offset + s, o, d);
    rays[2 * i] = make_float4(o.x, o.y, o.z, 1e-3f);
    rays[2 * i + 1] = make_float4(d.x, d.y, d.z, bits2f(0x7f800000u));
    state[2 * i] = make_float4(1.f, 1.f, 1.f, __uint_as_float((uint32_t)(sc * npix + pix)));
    state[2 * i + 1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(P.sample_offset + s));
    if (rscene) { rscene[i] = sc; }
}

__device__ __forceinline__ void retire(float* acc, float* acc2, uint32_t gpix, f3 L)
{
    atomicAdd(&acc[3 * (size_t)gpix], L.x); atomicAdd(&acc[3 * (size_t)gpix + 1], L.y); atomicAdd(&acc[3 * (size_t)gpix + 2], L.z);
    if (acc2)
    {
        atomicAdd(&acc2[3 * (size_t)gpix], L.x * L.x); atomicAdd(&acc2[3 * (size_t)gpix + 1], L.y * L.y);
        atomicAdd(&acc2[3 * (size_t)gpix + 2], L.z * L.z);
    }
}

__global__ void __launch_bounds__(256)
k_wf_shade(TraceCtx T, RP P, Shade S, const Cam* __restrict__ cams, uint32_t bounce, const uint32_t* __restrict__ count_in,
           const float4* __restrict__ rays, const float4* __restrict__ state, const float4* __restrict__ hits,
           float4* __restrict__ rays_out, float4* __restrict__ state_out, uint32_t* __restrict__ rscene_out,
           uint32_t* __restrict__ count_out, float* __restrict__ acc, float* __restrict__ acc2)
{
    const uint32_t n = *count_in;
    const uint32_t npix = P.W * P.H;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const float4 r0 = rays[2 * i], r1 = rays[2 * i + 1];
        const float4 s0 = state[2 * i], s1 = state[2 * i + 1];
        const float4 h0 = hits[2 * i], h1 = hits[2 * i + 1];
        const uint32_t gpix = __float_as_uint(s0.w), sidx = __float_as_uint(s1.w);
        f3 tp = mk3(s0.x, s0.y, s0.z), L = mk3(s1.x, s1.y, s1.z);
        const f3 o = mk3(r0.x, r0.y, r0.z), d = mk3(r1.x, r1.y, r1.z);
        const uint32_t flags = __float_as_uint(h1.w);
        if (!(flags & RT_HIT_FLAG_HIT))
        {
            L = add3(L, mul3(tp, environment(P, d)));
            retire(acc, acc2, gpix, L);
            continue;
        }
        const uint32_t sc = gpix / npix, pix = gpix - sc * npix;
        const uint32_t seed = cams ? cams[sc].seed : P.cam.seed;
        const f3 nrm = mk3(h1.x, h1.y, h1.z);
        const Surf sf = surface(S, __float_as_uint(h0.w));
        L = add3(L, mul3(tp, sf.emission));
        f3 nd;
        const bool alive = scatter(P, seed, sf, nrm, d, pix, sidx, bounce, tp, nd);
        if (!alive || bounce >= P.max_bounce)
        {
            retire(acc, acc2, gpix, L);
            continue;
        }
        const f3 no = add3(o, muls(d, h0.x));
        const uint32_t j = atomicAdd(count_out, 1u);
        rays_out[2 * j] = make_float4(no.x, no.y, no.z, 1e-4f);
        rays_out[2 * j + 1] = make_float4(nd.x, nd.y, nd.z, bits2f(0x7f800000u));
        state_out[2 * j] = make_float4(tp.x, tp.y, tp.z, s0.w);
        state_out[2 * j + 1] = make_float4(L.x, L.y, L.z, s1.w);
        if (rscene_out) { rscene_out[j] = sc; }
    }
}

__global__ void k_wf_finish(const float* __restrict__ acc, const float* __restrict__ acc2, uint64_t n, float spp,
                            float* __restrict__ rgb, float* __restrict__ rgb2)
{
    const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) { return; }
    rgb[i] = acc[i] / spp;
    if (rgb2) { rgb2[i] = acc2[i] / spp; }
}

Cam make_cam(const rt_render_cfg& c)
{
    Cam C;
    for (int k = 0; k < 3; k++) { C.pos[k] = c.cam_pos[k]; C.fwd[k] = c.cam_fwd[k]; C.right[k] = c.cam_right[k]; C.up[k] = c.cam_up[k]; }
    C.th = c.tan_half_fov_y;
    C.seed = c.seed;
    return C;
}

RP make_rp(const rt_render_cfg& c, const rt_shading& sh)
{
    RP P;
    std::memset(&P, 0, sizeof(P));
    P.env_map = sh.env_map; P.env_w = sh.env_w; P.env_h = sh.env_h;
    P.W = c.width; P.H = c.height; P.spp = c.spp; P.max_bounce = c.max_bounce; P.rr_after = c.rr_after;
    P.env_kind = c.env_kind;
    for (int k = 0; k < 3; k++) { P.env[k] = c.env_color[k]; }
    P.cam = make_cam(c);
    P.sample_offset = c.sample_offset;
    return P;
}

// One wavefront render: S scenes (1 for a plain handle), per-scene cameras on the device
// (nullptr: P.cam) and subtree roots (nullptr: the handle's root).
struct WfJob
{
    RP              P;
    const Cam*      cams;
    uint32_t        S;
    Shade           sh;
    const TraceRoot* roots;
    float*          rgb;
    float*          rgb2;
};

constexpr uint32_t kMaxBounceQueues = 64;

int wf_buffers(rt_bvh* B, const WfJob& J, const rt_wavefront_params& W)
{
    const uint64_t chunk = W.chunk_paths;
    const uint64_t nimg = (uint64_t)J.S * J.P.W * J.P.H * 3;
    for (int k = 0; k < 2; k++)
    {
        if (B->wf_rays[k].ensure(chunk * 32) || B->wf_state[k].ensure(chunk * 32) ||
            (J.S > 1 && B->wf_scene[k].ensure(chunk * 4)))
        {
            return RT_E_CUDA;
        }
    }
    if (B->wf_hits.ensure(chunk * 32) || B->wf_acc.ensure(nimg * 4 * 2) ||
        B->wf_ctr.ensure((size_t)kMaxBounceQueues * 16 + 64) || B->trace_status.ensure(64))
    {
        return RT_E_CUDA;
    }
    return RT_OK;
}

// Issues every launch of the render on st: no host synchronisation and no allocation, so the
// sequence can be captured into a CUDA graph. Returns the kernel launches issued via *n_kernels.
int wf_issue(rt_bvh* B, const WfJob& J, const rt_wavefront_params& W, cudaStream_t st, uint32_t* n_kernels)
{
    const TraceCtx T = make_trace_ctx(B);
    const RP& P = J.P;
    const uint64_t npix = (uint64_t)P.W * P.H;
    const uint64_t total = npix * J.S * P.spp;
    const uint64_t nimg = npix * J.S * 3;
    const uint32_t nb = P.max_bounce + 2;
    float* acc = B->wf_acc.as<float>();
    float* acc2 = J.rgb2 ? acc + nimg : nullptr;
    uint32_t* counts = B->wf_ctr.as<uint32_t>();  // per bounce queue length
    unsigned long long* tctr = reinterpret_cast<unsigned long long*>(counts + 2 * kMaxBounceQueues);  // per bounce trace counter
    uint32_t* status = B->trace_status.as<uint32_t>() + 4;
    const int sms = device_sm_count();
    const int sblk = W.shade_block ? (int)W.shade_block : 256;
    uint32_t nk = 0;
    RT_CUDA(cudaMemsetAsync(acc, 0, nimg * 4 * (J.rgb2 ? 2 : 1), st));
    TraceLaunch tl;
    tl.block = (int)W.trace_block;
    tl.stack = (int)W.stack_depth;
    tl.roots = J.roots;
    for (uint64_t g0 = 0; g0 < total; g0 += W.chunk_paths)
    {
        const uint32_t n_paths = (uint32_t)std::min<uint64_t>(W.chunk_paths, total - g0);
        RT_CUDA(cudaMemsetAsync(counts, 0, (size_t)kMaxBounceQueues * 16, st));
        k_wf_generate<<<(n_paths + 255) / 256, 256, 0, st>>>(P, J.cams, J.S, g0, n_paths, B->wf_rays[0].as<float4>(),
                                                              B->wf_state[0].as<float4>(),
                                                              J.S > 1 ? B->wf_scene[0].as<uint32_t>() : nullptr, counts);
        nk++;
        int cur = 0;
        for (uint32_t b = 0; b <= P.max_bounce; b++)
        {
            tl.rscene = J.S > 1 ? B->wf_scene[cur].as<uint32_t>() : nullptr;
            if (int e = trace_launch(B, B->wf_rays[cur].p, B->wf_hits.p, 0, counts + b, 0u, st, status, tctr + b, tl)) { return e; }
            k_wf_shade<<<sms * 2048 / sblk, sblk, 0, st>>>(T, P, J.sh, J.cams, b, counts + b, B->wf_rays[cur].as<float4>(),
                                                         B->wf_state[cur].as<float4>(), B->wf_hits.as<float4>(),
                                                         B->wf_rays[cur ^ 1].as<float4>(), B->wf_state[cur ^ 1].as<float4>(),
                                                         J.S > 1 ? B->wf_scene[cur ^ 1].as<uint32_t>() : nullptr,
                                                         counts + b + 1, acc, acc2);
            nk += 2;
            cur ^= 1;
        }
        if (int e = check_launch("wavefront")) { return e; }
        (void)nb;
    }
    k_wf_finish<<<(uint32_t)((nimg + 255) / 256), 256, 0, st>>>(acc, acc2, nimg, (float)P.spp, J.rgb, J.rgb2);
    nk++;
    if (n_kernels) { *n_kernels = nk; }
    return check_launch("wavefront finish");
}

rt_wavefront_params default_params()
{
    rt_wavefront_params W;
    W.trace_block = 128;
    W.chunk_paths = 1u << 22;
    W.stack_depth = 64;
    W.shade_block = 256;
    return W;
}

int check_params(const rt_wavefront_params& W)
{
    if (W.trace_block == 0 || W.trace_block % 32 || W.trace_block > 256) { return fail(RT_E_INVALID, "trace_block must be 32..256, a multiple of 32"); }
    if (W.shade_block == 0 || W.shade_block % 32 || W.shade_block > 1024) { return fail(RT_E_INVALID, "shade_block must be 32..1024, a multiple of 32"); }
    if (W.chunk_paths < 1024 || W.chunk_paths > (1u << 26)) { return fail(RT_E_INVALID, "chunk_paths must be in [1024, 2^26]"); }
    if (W.stack_depth != 32 && W.stack_depth != 64) { return fail(RT_E_INVALID, "stack_depth must be 32 or 64"); }
    return RT_OK;
}

// Replays the job from the handle's cached CUDA graph (captured on first use of a
// configuration) on the handle's own stream, ordered after / before the caller's stream.
int wf_run_graph(rt_bvh* B, const WfJob& J, const rt_wavefront_params& W, cudaStream_t st)
{
    if (int e = wf_buffers(B, J, W)) { return e; }
    // the graph bakes in kernel arguments and buffer addresses: all of them form its key
    // (and the traversal form: binary one-loop / while-while, or the 8-wide layout)
    const void* ptrs[] = { B->wf_rays[0].p, B->wf_rays[1].p, B->wf_state[0].p, B->wf_state[1].p, B->wf_scene[0].p,
                           B->wf_scene[1].p, B->wf_hits.p, B->wf_acc.p, B->wf_ctr.p, B->trace_status.p, B->gnodes.p,
                           B->tripos.p, B->tris.p, B->verts.p, B->rootbuf.p, B->scene_roots.p, B->wnodes.p, B->wid.p };
    const uint32_t form[2] = { B->trace_ww ? 1u : 0u, B->trace_wide ? 1u : 0u };
    std::vector<unsigned char> key(sizeof(WfJob) + sizeof(W) + sizeof(ptrs) + sizeof(form));
    std::memset(key.data(), 0, key.size());
    std::memcpy(key.data(), &J, sizeof(WfJob));
    std::memcpy(key.data() + sizeof(WfJob), &W, sizeof(W));
    std::memcpy(key.data() + sizeof(WfJob) + sizeof(W), ptrs, sizeof(ptrs));
    std::memcpy(key.data() + sizeof(WfJob) + sizeof(W) + sizeof(ptrs), form, sizeof(form));
    if (!B->wf_stream)
    {
        RT_CUDA(cudaStreamCreateWithFlags(&B->wf_stream, cudaStreamNonBlocking));
        RT_CUDA(cudaEventCreateWithFlags(&B->wf_ev[0], cudaEventDisableTiming));
        RT_CUDA(cudaEventCreateWithFlags(&B->wf_ev[1], cudaEventDisableTiming));
    }
    if (!B->wf_exec || key != B->wf_key)
    {
        if (B->wf_exec) { cudaGraphExecDestroy(B->wf_exec); B->wf_exec = nullptr; }
        RT_CUDA(cudaStreamBeginCapture(B->wf_stream, cudaStreamCaptureModeThreadLocal));
        uint32_t nk = 0;
        const int e = wf_issue(B, J, W, B->wf_stream, &nk);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(B->wf_stream, &g);
        if (e) { if (g) { cudaGraphDestroy(g); } return e; }
        if (ce != cudaSuccess) { return fail(RT_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce)); }
        const cudaError_t ie = cudaGraphInstantiate(&B->wf_exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) { B->wf_exec = nullptr; return fail(RT_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie)); }
        B->wf_key = key;
        B->wf_kernels = nk;
    }
    RT_CUDA(cudaEventRecord(B->wf_ev[0], st));
    RT_CUDA(cudaStreamWaitEvent(B->wf_stream, B->wf_ev[0], 0));
    RT_CUDA(cudaGraphLaunch(B->wf_exec, B->wf_stream));
    count_launch(B->wf_kernels);
    RT_CUDA(cudaEventRecord(B->wf_ev[1], B->wf_stream));
    RT_CUDA(cudaStreamWaitEvent(st, B->wf_ev[1], 0));
    return RT_OK;
}

// A valid parameter set for this handle: the tuned one, else the defaults (with the
// stack the tree needs).
rt_wavefront_params pick_params(const rt_bvh* B, const rt_wavefront_params* W)
{
    if (W) { return *W; }
    if (B->wf_tuned_valid) { return B->wf_tuned; }
    return default_params();
}

} // namespace

int render(const rt_bvh* B, const rt_render_cfg& cfg, const rt_shading& sh, int mode, float* rgb, float* rgb2,
           cudaStream_t st)
{
    const TraceCtx T = make_trace_ctx(B);
    const RP P = make_rp(cfg, sh);
    const Shade S{ sh.mats, sh.mat_of_tri, sh.tri_albedo, sh.n_mats };
    if (mode == RT_RENDER_PLAIN)
    {
        const dim3 grid((cfg.width + 15) / 16, (cfg.height + 7) / 8);
        k_render_plain<<<grid, 128, 0, st>>>(T, P, S, rgb, rgb2);
        count_launch();
        return check_launch("render plain");
    }
    if (mode != RT_RENDER_WAVEFRONT) { return fail(RT_E_INVALID, "unknown render mode"); }
    if (cfg.max_bounce + 2 > kMaxBounceQueues) { return fail(RT_E_INVALID, "max_bounce must be below 62 for the wavefront"); }
    rt_bvh* Bm = const_cast<rt_bvh*>(B);
    WfJob J;
    std::memset(&J, 0, sizeof(J));
    J.P = P; J.cams = nullptr; J.S = 1; J.sh = S; J.roots = nullptr; J.rgb = rgb; J.rgb2 = rgb2;
    rt_wavefront_params W = pick_params(B, nullptr);
    if (W.stack_depth < 64) { W.stack_depth = 64; }  // tuned for a batch; a plain handle keeps the full stack
    return wf_run_graph(Bm, J, W, st);
}

int render_batch(rt_bvh* B, const rt_render_cfg* cfgs, uint32_t S, const rt_shading& sh, const rt_wavefront_params* params,
                 float* rgb, float* rgb2, cudaStream_t st)
{
    const rt_render_cfg& c0 = cfgs[0];
    if (c0.max_bounce + 2 > kMaxBounceQueues) { return fail(RT_E_INVALID, "max_bounce must be below 62 for the wavefront"); }
    const rt_wavefront_params W = pick_params(B, params);
    if (int e = check_params(W)) { return e; }
    if (W.stack_depth < 64)
    {
        uint32_t depth = 0;
        if (int e = tree_depth(B, st, &depth)) { return e; }
        if (depth + 1 > W.stack_depth) { return fail(RT_E_INVALID, "stack_depth is smaller than the tree needs"); }
    }
    std::vector<Cam> cams(S);
    for (uint32_t s = 0; s < S; s++) { cams[s] = make_cam(cfgs[s]); }
    if (B->wf_cams.ensure((size_t)S * sizeof(Cam))) { return RT_E_CUDA; }
    RT_CUDA(cudaMemcpyAsync(B->wf_cams.p, cams.data(), (size_t)S * sizeof(Cam), cudaMemcpyHostToDevice, st));
    WfJob J;
    std::memset(&J, 0, sizeof(J));
    J.P = make_rp(c0, sh);
    J.cams = B->wf_cams.as<Cam>();
    J.S = S;
    J.sh = Shade{ sh.mats, sh.mat_of_tri, sh.tri_albedo, sh.n_mats };
    J.roots = S > 1 ? B->scene_roots.as<TraceRoot>() : nullptr;  // one scene: the whole tree
    J.rgb = rgb; J.rgb2 = rgb2;
    if (S == 1) { J.cams = nullptr; J.P.cam = cams[0]; }
    // (an upload from pageable memory has left the host vector when cudaMemcpyAsync returns)
    return wf_run_graph(B, J, W, st);
}

int autotune_wavefront(rt_bvh* B, const rt_render_cfg* cfgs, uint32_t S, const rt_shading& sh, rt_wavefront_params* best,
                       float* scratch_rgb, cudaStream_t st)
{
    uint32_t depth = 0;
    if (int e = tree_depth(B, st, &depth)) { return e; }
    const uint32_t blocks[] = { 64, 128, 256 };
    const uint32_t chunks[] = { 1u << 20, 1u << 21, 1u << 22, 1u << 23 };
    // trial renders with enough samples per pixel that the largest chunk fills (a one-sample
    // trial of a small image cannot tell the chunk sizes apart), at most the configs' own
    uint64_t px = 0;
    for (uint32_t k = 0; k < S; k++) { px += (uint64_t)cfgs[k].width * cfgs[k].height; }
    const uint64_t want = px ? (((uint64_t)chunks[3] + px - 1) / px) : 1;
    std::vector<rt_render_cfg> c1(cfgs, cfgs + S);
    for (auto& c : c1)
    {
        c.spp = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, c.spp));
        c.sample_offset = 0;
    }
    const uint32_t stacks[] = { 32, 64 };
    cudaEvent_t a, b;
    RT_CUDA(cudaEventCreate(&a));
    RT_CUDA(cudaEventCreate(&b));
    float best_ms = 1e30f;
    rt_wavefront_params bw = default_params();
    int err = RT_OK;
    for (uint32_t stack : stacks)
    {
        if (stack < 64 && depth + 1 > stack) { continue; }
        for (uint32_t blk : blocks)
        {
            for (uint32_t ch : chunks)
            {
                rt_wavefront_params W = default_params();
                W.trace_block = blk; W.chunk_paths = ch; W.stack_depth = stack;
                float ms = 0.f;
                for (int rep = 0; rep < 2 && !err; rep++)  // the first run captures the graph
                {
                    if (cudaEventRecord(a, st) != cudaSuccess) { err = fail(RT_E_CUDA, "event"); break; }
                    err = render_batch(B, c1.data(), S, sh, &W, scratch_rgb, nullptr, st);
                    if (err) { break; }
                    if (cudaEventRecord(b, st) != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess)
                    {
                        err = fail(RT_E_CUDA, "event"); break;
                    }
                    cudaEventElapsedTime(&ms, a, b);
                }
                if (err) { break; }
                if (ms < best_ms) { best_ms = ms; bw = W; }
            }
            if (err) { break; }
        }
        if (err) { break; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (err) { return err; }
    B->wf_tuned = bw;
    B->wf_tuned_valid = true;
    if (best) { *best = bw; }
    return RT_OK;
}

int adjoint(const rt_bvh* B, const rt_render_cfg& cfg, const rt_shading& sh, const float* d_rgb, float* g_alb,
            float* g_em, cudaStream_t st)
{
    const TraceCtx T = make_trace_ctx(B);
    const RP P = make_rp(cfg, sh);
    const Shade S{ sh.mats, sh.mat_of_tri, sh.tri_albedo, sh.n_mats };
    const dim3 grid((cfg.width + 15) / 16, (cfg.height + 7) / 8);
    k_adjoint<<<grid, 128, 0, st>>>(T, P, S, d_rgb, g_alb, sh.mats ? g_em : nullptr);
    count_launch();
    return check_launch("adjoint");
}

} // namespace rtb
