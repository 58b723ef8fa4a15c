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

namespace rtb
{

namespace
{

struct RP
{
    uint32_t W, H, spp, max_bounce;
    int32_t  rr_after;
    uint32_t env_kind;
    float    env[3];
    float    pos[3], fwd[3], right[3], up[3];
    float    th;
    uint32_t seed, sample_offset;
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
__device__ __forceinline__ void primary(const RP& P, uint32_t x, uint32_t y, uint32_t pix, uint32_t sidx, f3& o, f3& d)
{
    const uint4 r = philox(pix, sidx, 0u, 0u, P.seed, 0x5EEDu);
    const float aspect = (float)P.W / (float)P.H;
    const float u = (((float)x + u01(r.x)) / (float)P.W * 2.f - 1.f) * aspect;
    const float v = ((float)y + u01(r.y)) / (float)P.H * 2.f - 1.f;
    const f3 fwd = mk3(P.fwd[0], P.fwd[1], P.fwd[2]);
    const f3 rgt = mk3(P.right[0], P.right[1], P.right[2]);
    const f3 up = mk3(P.up[0], P.up[1], P.up[2]);
    o = mk3(P.pos[0], P.pos[1], P.pos[2]);
    d = norm3(add3(add3(fwd, muls(rgt, u * P.th)), muls(up, v * P.th)));
}

// background (src/main.cpp:162-173)
__device__ __forceinline__ f3 environment(const RP& P, f3 d)
{
    if (P.env_kind == 0)
    {
        const float t = d.y * 0.5f + 0.5f;
        return add3(muls(mk3(1.0f, 1.0f, 1.0f), 1.f - t), muls(mk3(0.5f, 0.7f, 1.0f), t));
    }
    return mk3(P.env[0], P.env[1], P.env[2]);
}

// One bounce at a hit (src/main.cpp:178-200) after the emission of the surface was added:
// the next direction (cosine hemisphere about the shading normal, or the mirror direction),
// throughput update and Russian roulette. Returns false when roulette ends the path.
__device__ __forceinline__ bool scatter(const RP& P, const Surf& sf, f3 n, f3 din, uint32_t pix, uint32_t sidx,
                                        uint32_t bounce, f3& tp, f3& dout)
{
    const uint4 r = philox(pix, sidx, bounce + 1u, 0u, P.seed, 0x5EEDu);
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
    primary(P, x, y, pix, sidx, o, d);
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
        if (!scatter(P, sf, n, d, pix, sidx, bounce, tp, nd)) { break; }
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
        if (act) { primary(P, x, y, pix, sidx, o, d); }
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
                    if (!scatter(P, sf, n, d, pix, sidx, bounce, tp, nd) || bounce >= P.max_bounce) { alive = false; }
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
// ray queue: rt_ray records (o, tmin, d, tmax); path state: (tp.xyz, pixel), (L.xyz, sample)

__global__ void __launch_bounds__(256)
k_wf_generate(RP P, uint32_t s0, uint32_t n_paths, float4* __restrict__ rays, float4* __restrict__ state,
              uint32_t* __restrict__ count)
{
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i == 0) { *count = n_paths; }
    if (i >= n_paths) { return; }
    const uint32_t npix = P.W * P.H;
    const uint32_t pix = i % npix, s = s0 + i / npix;
    const uint32_t x = pix % P.W, y = pix / P.W;
    f3 o, d;
    primary(P, x, y, pix, P.sample_offset + s, o, d);
    rays[2 * i] = make_float4(o.x, o.y, o.z, 1e-3f);
    rays[2 * i + 1] = make_float4(d.x, d.y, d.z, bits2f(0x7f800000u));
    state[2 * i] = make_float4(1.f, 1.f, 1.f, __uint_as_float(pix));
    state[2 * i + 1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(P.sample_offset + s));
}

__device__ __forceinline__ void retire(float* acc, float* acc2, uint32_t pix, f3 L)
{
    atomicAdd(&acc[3 * pix], L.x); atomicAdd(&acc[3 * pix + 1], L.y); atomicAdd(&acc[3 * pix + 2], L.z);
    if (acc2)
    {
        atomicAdd(&acc2[3 * pix], L.x * L.x); atomicAdd(&acc2[3 * pix + 1], L.y * L.y); atomicAdd(&acc2[3 * pix + 2], L.z * L.z);
    }
}

__global__ void __launch_bounds__(256)
k_wf_shade(TraceCtx T, RP P, Shade S, uint32_t bounce,
           const uint32_t* __restrict__ count_in, const float4* __restrict__ rays, const float4* __restrict__ state,
           const float4* __restrict__ hits, float4* __restrict__ rays_out, float4* __restrict__ state_out,
           uint32_t* __restrict__ count_out, float* __restrict__ acc, float* __restrict__ acc2)
{
    const uint32_t n = *count_in;
    for (uint32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
    {
        const float4 r0 = rays[2 * i], r1 = rays[2 * i + 1];
        const float4 s0 = state[2 * i], s1 = state[2 * i + 1];
        const float4 h0 = hits[2 * i], h1 = hits[2 * i + 1];
        const uint32_t pix = __float_as_uint(s0.w), sidx = __float_as_uint(s1.w);
        f3 tp = mk3(s0.x, s0.y, s0.z), L = mk3(s1.x, s1.y, s1.z);
        const f3 o = mk3(r0.x, r0.y, r0.z), d = mk3(r1.x, r1.y, r1.z);
        const uint32_t flags = __float_as_uint(h1.w);
        if (!(flags & RT_HIT_FLAG_HIT))
        {
            L = add3(L, mul3(tp, environment(P, d)));
            retire(acc, acc2, pix, L);
            continue;
        }
        const f3 nrm = mk3(h1.x, h1.y, h1.z);
        const Surf sf = surface(S, __float_as_uint(h0.w));
        L = add3(L, mul3(tp, sf.emission));
        f3 nd;
        const bool alive = scatter(P, sf, nrm, d, pix, sidx, bounce, tp, nd);
        if (!alive || bounce >= P.max_bounce)
        {
            retire(acc, acc2, pix, L);
            continue;
        }
        const f3 no = add3(o, muls(d, h0.x));
        const uint32_t j = atomicAdd(count_out, 1u);
        rays_out[2 * j] = make_float4(no.x, no.y, no.z, 1e-4f);
        rays_out[2 * j + 1] = make_float4(nd.x, nd.y, nd.z, bits2f(0x7f800000u));
        state_out[2 * j] = make_float4(tp.x, tp.y, tp.z, s0.w);
        state_out[2 * j + 1] = make_float4(L.x, L.y, L.z, s1.w);
    }
}

__global__ void k_wf_finish(const float* __restrict__ acc, const float* __restrict__ acc2, uint32_t n, float spp,
                            float* __restrict__ rgb, float* __restrict__ rgb2)
{
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) { return; }
    rgb[i] = acc[i] / spp;
    if (rgb2) { rgb2[i] = acc2[i] / spp; }
}

RP make_rp(const rt_render_cfg& c)
{
    RP P;
    P.W = c.width; P.H = c.height; P.spp = c.spp; P.max_bounce = c.max_bounce; P.rr_after = c.rr_after;
    P.env_kind = c.env_kind;
    for (int k = 0; k < 3; k++)
    {
        P.env[k] = c.env_color[k]; P.pos[k] = c.cam_pos[k]; P.fwd[k] = c.cam_fwd[k];
        P.right[k] = c.cam_right[k]; P.up[k] = c.cam_up[k];
    }
    P.th = c.tan_half_fov_y;
    P.seed = c.seed;
    P.sample_offset = c.sample_offset;
    return P;
}

} // namespace

int render(const rt_bvh* B, const rt_render_cfg& cfg, const rt_shading& sh, int mode, float* rgb, float* rgb2,
           cudaStream_t st)
{
    const TraceCtx T = make_trace_ctx(B);
    RP P = make_rp(cfg);
    const Shade S{ sh.mats, sh.mat_of_tri, sh.tri_albedo, sh.n_mats };
    if (mode == RT_RENDER_PLAIN)
    {
        const dim3 grid((cfg.width + 15) / 16, (cfg.height + 7) / 8);
        k_render_plain<<<grid, 128, 0, st>>>(T, P, S, rgb, rgb2);
        count_launch();
        return check_launch("render plain");
    }
    if (mode != RT_RENDER_WAVEFRONT) { return fail(RT_E_INVALID, "unknown render mode"); }
    rt_bvh* Bm = const_cast<rt_bvh*>(B);
    const uint64_t npix = (uint64_t)cfg.width * cfg.height;
    const uint64_t max_paths = 1ull << 22;  // paths in flight per chunk
    uint32_t spc = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(cfg.spp, max_paths / std::max<uint64_t>(npix, 1)));
    const uint64_t chunk = npix * spc;
    const uint32_t nb = cfg.max_bounce + 2;
    for (int k = 0; k < 2; k++)
    {
        if (Bm->wf_rays[k].ensure(chunk * 32) || Bm->wf_state[k].ensure(chunk * 32)) { return RT_E_CUDA; }
    }
    if (Bm->wf_hits.ensure(chunk * 32) || Bm->wf_acc.ensure(npix * 3 * 4 * 2) || Bm->wf_ctr.ensure((size_t)nb * 16 + 64) ||
        Bm->trace_status.ensure(64))
    {
        return RT_E_CUDA;
    }
    float* acc = Bm->wf_acc.as<float>();
    float* acc2 = rgb2 ? acc + npix * 3 : nullptr;
    RT_CUDA(cudaMemsetAsync(acc, 0, npix * 3 * 4 * 2, st));
    uint32_t* counts = Bm->wf_ctr.as<uint32_t>();                                   // per bounce queue length
    unsigned long long* tctr = reinterpret_cast<unsigned long long*>(counts + 2 * nb + 2);  // per bounce trace counter
    uint32_t* status = Bm->trace_status.as<uint32_t>() + 4;
    const int sms = device_sm_count();
    for (uint32_t s0 = 0; s0 < cfg.spp; s0 += spc)
    {
        const uint32_t ns = std::min(spc, cfg.spp - s0);
        const uint32_t n_paths = (uint32_t)(npix * ns);
        RT_CUDA(cudaMemsetAsync(counts, 0, (size_t)nb * 16 + 64 - 0, st));
        k_wf_generate<<<(n_paths + 255) / 256, 256, 0, st>>>(P, s0, n_paths, Bm->wf_rays[0].as<float4>(),
                                                              Bm->wf_state[0].as<float4>(), counts);
        count_launch();
        int cur = 0;
        for (uint32_t b = 0; b <= cfg.max_bounce; b++)
        {
            if (int e = trace_launch(B, Bm->wf_rays[cur].p, Bm->wf_hits.p, 0, counts + b, 0u, st, status, tctr + b)) { return e; }
            k_wf_shade<<<sms * 8, 256, 0, st>>>(T, P, S, b, counts + b, Bm->wf_rays[cur].as<float4>(),
                                                Bm->wf_state[cur].as<float4>(), Bm->wf_hits.as<float4>(),
                                                Bm->wf_rays[cur ^ 1].as<float4>(), Bm->wf_state[cur ^ 1].as<float4>(),
                                                counts + b + 1, acc, acc2);
            count_launch();
            cur ^= 1;
        }
        if (int e = check_launch("wavefront")) { return e; }
    }
    const uint32_t nv = (uint32_t)(npix * 3);
    k_wf_finish<<<(nv + 255) / 256, 256, 0, st>>>(acc, acc2, nv, (float)cfg.spp, rgb, rgb2);
    count_launch();
    return check_launch("wavefront finish");
}

int adjoint(const rt_bvh* B, const rt_render_cfg& cfg, const rt_shading& sh, const float* d_rgb, float* g_alb,
            float* g_em, cudaStream_t st)
{
    const TraceCtx T = make_trace_ctx(B);
    const RP P = make_rp(cfg);
    const Shade S{ sh.mats, sh.mat_of_tri, sh.tri_albedo, sh.n_mats };
    const dim3 grid((cfg.width + 15) / 16, (cfg.height + 7) / 8);
    k_adjoint<<<grid, 128, 0, st>>>(T, P, S, d_rgb, g_alb, sh.mats ? g_em : nullptr);
    count_launch();
    return check_launch("adjoint");
}

} // namespace rtb
