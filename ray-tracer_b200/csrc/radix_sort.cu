// radix_sort.cu -- stable LSD radix sort of (key, uint32 value) pairs, one kernel per 8-bit
// digit in the "onesweep" style (Adinets & Merrill, 2022): every tile ranks its keys in
// shared memory, publishes its digit counts, and learns the counts of all earlier tiles by a
// decoupled look-back, so each pass reads and writes the data exactly once. The digit
// histograms of all passes come precomputed from the kernel that produced the keys.
//
// This replaces the reference's serial 8-pass LSD sort (src/bvh/bvh_morton.cpp:109-159);
// stability keeps equal Morton codes in ascending triangle order, as there.
#include <atomic>
#include "rt_internal.h"

namespace rtb
{
namespace
{

constexpr int      RS_BLOCK   = 256;
constexpr int      RS_WARPS   = RS_BLOCK / 32;
// Two tile shapes: up to 2^21 keys, tiles of 16 keys per thread (4096) with 2 resident blocks
// per SM; above, 8 keys per thread (2048) with 5 resident blocks per SM (48 registers), whose
// extra occupancy hides the memory latency of the long passes.
constexpr uint32_t RS_SMALL_MAX = RS_SMALL_MAX_KEYS;
constexpr uint32_t LB_AGG     = 1u << 30;           // tile aggregate published
constexpr uint32_t LB_PRE     = 2u << 30;           // inclusive prefix published
constexpr uint32_t LB_VAL     = (1u << 30) - 1u;
constexpr uint32_t SPIN_LIMIT = 1u << 22;           // bounded wait per look-back step
constexpr int      LB_WIN     = 32;                 // predecessors read per look-back step

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ void     st_volatile(uint32_t* p, uint32_t v) { *(volatile uint32_t*)p = v; }

// Exclusive scan of one value per thread over a 256-thread block; also returns the total.
__device__ __forceinline__ uint32_t block_excl_scan_256(uint32_t v, uint32_t* warp_sums, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) { x += y; }
    }
    if (lane == 31) { warp_sums[warp] = x; }
    __syncthreads();
    if (warp == 0)
    {
        uint32_t w = lane < RS_WARPS ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) { w += y; }
        }
        if (lane < RS_WARPS) { warp_sums[lane] = w; }
    }
    __syncthreads();
    uint32_t base = warp > 0 ? warp_sums[warp - 1] : 0u;
    if (total) { *total = warp_sums[RS_WARPS - 1]; }
    uint32_t r = base + x - v;
    __syncthreads();
    return r;
}

// Lanes of the warp holding the same 8-bit digit as this one (d = 0xffffffff: no key; such
// lanes match only each other): the set __match_any_sync returns, built from one ballot per
// digit bit plus one for the key's presence. The per-bucket sort below ranks with it (faster
// there than the match instruction; the onesweep passes keep the instruction, which is faster
// for them at 16M keys).
__device__ __forceinline__ uint32_t match_digit8(uint32_t d)
{
    const bool valid = d != 0xffffffffu;
    const uint32_t vm = __ballot_sync(0xffffffffu, valid);
    uint32_t m = valid ? vm : ~vm;
#pragma unroll
    for (int b = 0; b < 8; b++)
    {
        const bool bit = (d >> b) & 1u;
        const uint32_t bm = __ballot_sync(0xffffffffu, bit);
        m &= bit ? bm : ~bm;
    }
    return m;
}

template <typename K, int RS_IPT, int MINB>
__global__ void __launch_bounds__(RS_BLOCK, MINB)
k_onesweep(const K* __restrict__ kin, const uint32_t* __restrict__ vin, int vals_identity, K* __restrict__ kout,
           uint32_t* __restrict__ vout, uint32_t n, uint32_t tiles, int shift, const uint32_t* __restrict__ hist,
           uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ lookback, uint32_t* __restrict__ status,
           const uint32_t* __restrict__ skip, uint32_t skip_if)
{
    if (skip && *skip == skip_if) { return; }  // the other sort path runs (radix_sort_pairs)
    constexpr int RS_TILE = RS_BLOCK * RS_IPT;
    extern __shared__ __align__(16) unsigned char smem[];
    K*        sk     = reinterpret_cast<K*>(smem);
    uint32_t* sv     = reinterpret_cast<uint32_t*>(sk + RS_TILE);
    uint32_t* whist  = sv + RS_TILE;            // [warp][digit]
    uint32_t* tstart = whist + RS_WARPS * 256;  // tile-local digit start
    uint32_t* gbase  = tstart + 256;            // global position of digit d minus tstart[d]
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_sums[RS_WARPS];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) { s_tile = atomicAdd(tile_counter, 1u); }
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_BLOCK) { whist[i] = 0u; }
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t tile_base = tile * (uint32_t)RS_TILE;
    const uint32_t tile_n = min((uint32_t)RS_TILE, n - tile_base);

    // load: warp w owns the contiguous run [w*32*IPT, (w+1)*32*IPT) of the tile, item j of
    // lane l is element w*32*IPT + j*32 + l, so (warp, j, lane) order is input order.
    K        key[RS_IPT];
    uint32_t val[RS_IPT];
    uint32_t dig[RS_IPT];
    uint32_t off[RS_IPT];
#pragma unroll
    for (int j = 0; j < RS_IPT; j++)
    {
        const uint32_t li = (uint32_t)warp * (32u * RS_IPT) + (uint32_t)j * 32u + (uint32_t)lane;
        if (li < tile_n)
        {
            key[j] = kin[tile_base + li];
            val[j] = vals_identity ? tile_base + li : vin[tile_base + li];
            dig[j] = (uint32_t)(key[j] >> shift) & 255u;
        }
        else
        {
            key[j] = 0; val[j] = 0; dig[j] = 0xffffffffu;
        }
    }
    // stable rank inside the warp: peers with the same digit, counted in lane order
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t* wh = whist + warp * 256;
#pragma unroll
    for (int j = 0; j < RS_IPT; j++)
    {
        const uint32_t d = dig[j];
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & lt);
        const bool valid = d != 0xffffffffu;
        uint32_t cnt = valid ? wh[d] : 0u;
        __syncwarp();
        if (valid && before == 0u) { wh[d] = cnt + __popc(peers); }
        __syncwarp();
        off[j] = cnt + before;
    }
    __syncthreads();

    // per digit: tile count, and exclusive offsets of each warp
    const uint32_t d = threadIdx.x;  // RS_BLOCK == 256 digits
    uint32_t run = 0u;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++)
    {
        uint32_t c = whist[w * 256 + d];
        whist[w * 256 + d] = run;
        run += c;
    }
    const uint32_t my = run;
    // publish this tile's count at once so later tiles can proceed. Status words are
    // [tile][digit], so a block reads one predecessor's 256 words as one coalesced row.
    uint32_t* lb = lookback + d;
    st_volatile(&lb[(size_t)tile * 256u], (tile == 0 ? LB_PRE : LB_AGG) | (my & LB_VAL));

    // scatter into shared memory in digit order; it needs only tile-local offsets, so it runs
    // before the look-back and frees the item registers
    const uint32_t ts = block_excl_scan_256(my, s_warp_sums, nullptr);
    const uint32_t hs = block_excl_scan_256(hist[d], s_warp_sums, nullptr);
    tstart[d] = ts;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RS_IPT; j++)
    {
        if (dig[j] != 0xffffffffu)
        {
            const uint32_t pos = tstart[dig[j]] + whist[warp * 256 + dig[j]] + off[j];
            sk[pos] = key[j];
            sv[pos] = val[j];
        }
    }

    // decoupled look-back over earlier tiles: each step reads the status words of up to
    // LB_WIN predecessors with independent loads and folds them newest first until an
    // inclusive prefix is met. A word not yet published is waited on alone (bounded, with a
    // short sleep), then the walk resumes there.
    uint32_t excl = 0u;
    if (tile > 0)
    {
        int p = (int)tile - 1;
        uint32_t spins = 0u;
        bool done = false;
        while (!done && p >= 0)
        {
            uint32_t w[LB_WIN];
#pragma unroll
            for (int k = 0; k < LB_WIN; k++) { w[k] = (p - k >= 0) ? ld_volatile(&lb[(size_t)(p - k) * 256u]) : LB_PRE; }
            int used = 0;
#pragma unroll
            for (int k = 0; k < LB_WIN; k++)
            {
                if (done || used != k) { continue; }
                if ((w[k] & ~LB_VAL) == 0u) { continue; }  // not published yet: resume here
                excl += w[k] & LB_VAL;
                used = k + 1;
                if (w[k] & LB_PRE) { done = true; }
            }
            p -= used;
            if (!done && used == 0)
            {
                // wait for tile p alone
                while ((ld_volatile(&lb[(size_t)p * 256u]) & ~LB_VAL) == 0u)
                {
                    if (++spins > SPIN_LIMIT) { break; }
                    __nanosleep(32);
                }
                if (spins > SPIN_LIMIT) { atomicOr(status, ST_TIMEOUT); break; }
            }
        }
        st_volatile(&lb[(size_t)tile * 256u], LB_PRE | ((excl + my) & LB_VAL));
    }
    gbase[d] = hs + excl - ts;
    __syncthreads();

    // write out with contiguous runs per digit
    for (uint32_t i = threadIdx.x; i < tile_n; i += RS_BLOCK)
    {
        const K k = sk[i];
        const uint32_t g = gbase[(uint32_t)(k >> shift) & 255u] + i;
        if (g >= n) { atomicOr(status, ST_CAPACITY); continue; }
        kout[g] = k;
        vout[g] = sv[i];
    }
}

template <typename K, int IPT>
constexpr size_t onesweep_smem()
{
    return (size_t)RS_BLOCK * IPT * sizeof(K) + (size_t)RS_BLOCK * IPT * 4 + (size_t)RS_WARPS * 256 * 4 + 2 * 256 * 4;
}

// All passes of one tile shape on the given scratch. skip (device, optional): the passes do
// nothing when *skip == skip_if (the MSD path of radix_sort_pairs sorted the keys instead).
template <typename K, int IPT, int MINB>
int onesweep_passes(K* keys, uint32_t* vals, bool vals_identity, uint32_t n, int passes, const uint32_t* hist, K* keys_alt,
                    uint32_t* vals_alt, uint32_t* lookback, uint32_t* tile_counters, uint32_t* status, cudaStream_t st,
                    K** keys_out, uint32_t** vals_out, const uint32_t* skip = nullptr, uint32_t skip_if = 0,
                    bool zeroed = false)
{
    constexpr uint32_t tile = RS_BLOCK * IPT;
    const uint32_t tiles = (n + tile - 1) / tile;
    if (!zeroed)
    {
        RT_CUDA(cudaMemsetAsync(lookback, 0, (size_t)passes * tiles * 256 * 4, st));
        RT_CUDA(cudaMemsetAsync(tile_counters, 0, 64 * 4, st));
    }
    constexpr size_t smem = onesweep_smem<K, IPT>();
    static PerDeviceOnce attr;  // per instantiation and device (bakes may run on several host threads and GPUs)
    if (int e = attr.once([] {
            RT_CUDA(cudaFuncSetAttribute(k_onesweep<K, IPT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            return (int)RT_OK;
        }))
    {
        return e;
    }
    K* kin = keys;
    K* kalt = keys_alt;
    uint32_t* vin = vals;
    uint32_t* valt = vals_alt;
    for (int p = 0; p < passes; p++)
    {
        k_onesweep<K, IPT, MINB><<<tiles, RS_BLOCK, smem, st>>>(kin, vin, (vals_identity && p == 0) ? 1 : 0, kalt, valt, n,
                                                                tiles, 8 * p, hist + 256 * p, tile_counters + p,
                                                                lookback + (size_t)p * tiles * 256, status, skip, skip_if);
        count_launch();
        if (int e = check_launch("onesweep")) { return e; }
        K* tk = kin; kin = kalt; kalt = tk;
        uint32_t* tv = vin; vin = valt; valt = tv;
    }
    *keys_out = kin;
    *vals_out = vin;
    return RT_OK;
}

// ---- MSD path: one onesweep pass on the most significant digit, then every bucket of that
// digit sorted by the lower digits inside one block's shared memory. Used when no bucket holds
// more keys than one block takes (decided on the device from the top digit's histogram, which
// the key producer already built); otherwise those kernels return at once and the LSD passes
// run. Both paths are stable and give the same order.
// Per-bucket block shapes: LB threads x LI keys (capacity LB * LI keys per bucket).
constexpr int LS_SMALL_B = 256, LS_SMALL_I = 18;  // 4,608 keys, two blocks per SM
constexpr int LS_LARGE_B = 512, LS_LARGE_I = 16;  // 8,192 keys, one block per SM

// bstart[d] = first position of top digit d (exclusive scan of its histogram), bstart[256] = n;
// *flag = 1 when a bucket exceeds cap (the LSD passes must run), else 0.
__global__ void __launch_bounds__(256)
k_msd_check(const uint32_t* __restrict__ hist_top, uint32_t n, uint32_t cap, uint32_t* __restrict__ bstart,
            uint32_t* __restrict__ flag, uint32_t* __restrict__ flag_copy)
{
    __shared__ uint32_t ws[RS_WARPS];
    __shared__ uint32_t s_big;
    const uint32_t h = hist_top[threadIdx.x];
    if (threadIdx.x == 0) { s_big = 0u; }
    __syncthreads();
    if (h > cap) { atomicOr(&s_big, 1u); }
    const uint32_t ex = block_excl_scan_256(h, ws, nullptr);
    bstart[threadIdx.x] = ex;
    if (threadIdx.x == 0)
    {
        bstart[256] = n;
        *flag = s_big;
        if (flag_copy) { *flag_copy = s_big; }
    }
}

template <typename K, int LB, int LI>
constexpr size_t local_sort_smem()
{
    return (size_t)LB * LI * sizeof(K) + (size_t)LB * LI * 4 + (size_t)(LB / 32) * 256 * 4 + 256 * 4;
}

// Compare-exchange partner order of the (key, position) pairs of a sub-bucket sort.
template <typename K>
__device__ __forceinline__ bool pair_less(K ka, uint32_t pa, K kb, uint32_t pb)
{
    return ka < kb || (ka == kb && pa < pb);
}

// Bitonic sort (Batcher, 1968) of one sub-bucket of cnt <= 64 keys in shared memory by one warp:
// lane L holds elements L and L + 32 as (key, position in the sub-bucket, value); padding sorts
// last. Ties on the key keep the position order, so the sort is stable.
template <typename K>
__device__ __forceinline__ void warp_sort64(K* sk, uint32_t* sv, uint32_t start, uint32_t cnt, int lane)
{
    K key[2];
    uint32_t pos[2], val[2];
#pragma unroll
    for (int h = 0; h < 2; h++)
    {
        const uint32_t e = (uint32_t)lane + 32u * h;
        const bool v = e < cnt;
        key[h] = v ? sk[start + e] : (K)~(K)0;
        val[h] = v ? sv[start + e] : 0u;
        pos[h] = v ? e : 64u + e;
    }
#pragma unroll
    for (int k = 2; k <= 64; k <<= 1)
    {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            if (j == 32)
            {
                // elements L and L + 32 of one lane (k = 64: ascending)
                if (pair_less<K>(key[1], pos[1], key[0], pos[0]))
                {
                    const K tk = key[0]; key[0] = key[1]; key[1] = tk;
                    const uint32_t tp = pos[0]; pos[0] = pos[1]; pos[1] = tp;
                    const uint32_t tv = val[0]; val[0] = val[1]; val[1] = tv;
                }
                continue;
            }
#pragma unroll
            for (int h = 0; h < 2; h++)
            {
                const uint32_t idx = (uint32_t)lane + 32u * h;
                const K ok = __shfl_xor_sync(0xffffffffu, key[h], j);
                const uint32_t op = __shfl_xor_sync(0xffffffffu, pos[h], j);
                const uint32_t ov = __shfl_xor_sync(0xffffffffu, val[h], j);
                const bool lower = (idx & (uint32_t)j) == 0;
                const bool asc = (idx & (uint32_t)k) == 0;
                const bool other_less = pair_less<K>(ok, op, key[h], pos[h]);
                // the lower index of an ascending pair (and the upper of a descending one) keeps the smaller
                if (other_less == (lower == asc)) { key[h] = ok; pos[h] = op; val[h] = ov; }
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; h++)
    {
        const uint32_t e = (uint32_t)lane + 32u * h;
        if (e < cnt) { sk[start + e] = key[h]; sv[start + e] = val[h]; }
    }
}

// The same network on N = 16 or 32 elements, one per lane: the lanes of each group of N (idx =
// lane mod N) sort the sub-bucket [start, start + cnt) they were given (cnt <= N; groups of 16
// lanes in one warp may sort different sub-buckets).
template <typename K, int N>
__device__ __forceinline__ void warp_sort_n(K* sk, uint32_t* sv, uint32_t start, uint32_t cnt, uint32_t idx)
{
    const bool v = idx < cnt;
    K key = v ? sk[start + idx] : (K)~(K)0;
    uint32_t val = v ? sv[start + idx] : 0u;
    uint32_t pos = v ? idx : 64u + idx;
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
    {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            const K ok = __shfl_xor_sync(0xffffffffu, key, j);
            const uint32_t op = __shfl_xor_sync(0xffffffffu, pos, j);
            const uint32_t ov = __shfl_xor_sync(0xffffffffu, val, j);
            const bool lower = (idx & (uint32_t)j) == 0;
            const bool asc = (idx & (uint32_t)k) == 0;
            if (pair_less<K>(ok, op, key, pos) == (lower == asc)) { key = ok; pos = op; val = ov; }
        }
    }
    if (v) { sk[start + idx] = key; sv[start + idx] = val; }
}

// One block per bucket of the top digit: keys[bstart[b], bstart[b+1]) sorted stably by the
// digits below the top one, kin/vin -> kout/vout (may be the same buffers: the block holds its
// bucket in registers and shared memory before writing). With sub_shift >= 0 the block first
// takes one counting pass on the 8 bits below the top digit (bits sub_shift .. sub_shift + 7),
// which splits the bucket into 256 sub-buckets, and, when none holds more than 64 keys, sorts
// each with a warp's bitonic network on the whole key; otherwise (and with sub_shift < 0) it
// takes npass 8-bit LSD passes, ranked as in k_onesweep.
template <typename K, int LB, int LI, int MINB>
__global__ void __launch_bounds__(LB, MINB)
k_local_sort(const K* kin, const uint32_t* vin, K* kout, uint32_t* vout, const uint32_t* __restrict__ bstart,
             const uint32_t* __restrict__ flag, int npass, int sub_shift, uint32_t* __restrict__ tab)
{
    constexpr uint32_t CAP = (uint32_t)LB * LI;
    if (*flag) { return; }
    extern __shared__ __align__(16) unsigned char smem[];
    K*        sk     = reinterpret_cast<K*>(smem);
    uint32_t* sv     = reinterpret_cast<uint32_t*>(sk + CAP);
    uint32_t* whist  = sv + CAP;                 // [warp][digit]
    uint32_t* tstart = whist + (LB / 32) * 256;  // block-local digit start
    __shared__ uint32_t s_warp_sums[8];
    __shared__ uint32_t s_tot[256];
    __shared__ uint32_t s_max;
    const uint32_t b0 = bstart[blockIdx.x], m = bstart[blockIdx.x + 1] - b0;
    // tab (with sub-buckets): the bucket table of the top 16 key bits -- tab[v] = the first
    // sorted index whose top 16 bits are >= v -- for this bucket's 256 values, from the
    // sub-bucket starts; the last bucket also writes tab[65536] = n
    if (tab && blockIdx.x == 255 && threadIdx.x == 0) { tab[65536] = bstart[256]; }
    if (m == 0)
    {
        if (tab && threadIdx.x < 256) { tab[blockIdx.x * 256u + threadIdx.x] = b0; }
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (int)((m + 32u * LI - 1) / (32u * LI));  // warps holding keys
    // element (warp, j, lane) = warp * 32 * LI + j * 32 + lane, so that order is input order
    K        key[LI];
    uint32_t val[LI];
    auto load = [&]() {
#pragma unroll
        for (int j = 0; j < LI; j++)
        {
            const uint32_t e = (uint32_t)warp * (32u * LI) + (uint32_t)j * 32u + (uint32_t)lane;
            if (e < m) { key[j] = kin[b0 + e]; val[j] = vin[b0 + e]; } else { key[j] = 0; val[j] = 0; }
        }
    };
    load();
    const uint32_t lt = (1u << lane) - 1u;
    // one stable counting pass of the registers' keys by bits shift .. shift + 7 into sk / sv;
    // leaves the digit totals in s_tot and their exclusive scan in tstart
    auto pass = [&](int shift) {
        for (int i = threadIdx.x; i < nw * 256; i += LB) { whist[i] = 0u; }
        __syncthreads();
        uint32_t* wh = whist + warp * 256;
        uint32_t dig[LI], off[LI];
#pragma unroll
        for (int j = 0; j < LI; j++) { dig[j] = 0xffffffffu; }
        if (warp < nw)  // warps wholly past the bucket's end have nothing to rank
        {
#pragma unroll
            for (int j = 0; j < LI; j++)
            {
                const uint32_t e = (uint32_t)warp * (32u * LI) + (uint32_t)j * 32u + (uint32_t)lane;
                const bool valid = e < m;
                const uint32_t d = valid ? (uint32_t)(key[j] >> shift) & 255u : 0xffffffffu;
                dig[j] = d;
                const uint32_t peers = match_digit8(d);
                const uint32_t before = __popc(peers & lt);
                uint32_t cnt = valid ? wh[d] : 0u;
                __syncwarp();
                if (valid && before == 0u) { wh[d] = cnt + __popc(peers); }
                __syncwarp();
                off[j] = cnt + before;
            }
        }
        __syncthreads();
        // per digit (threads 0..255): warps' exclusive offsets and the digit's total
        uint32_t total = 0u;
        if (threadIdx.x < 256)
        {
            for (int w = 0; w < nw; w++)
            {
                const uint32_t c = whist[w * 256 + threadIdx.x];
                whist[w * 256 + threadIdx.x] = total;
                total += c;
            }
            s_tot[threadIdx.x] = total;
        }
        __syncthreads();
        // exclusive scan of the 256 digit totals (warps 0..7 hold them; the others scan zeros)
        uint32_t x = total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) { x += y; }
        }
        if (lane == 31 && warp < 8) { s_warp_sums[warp] = x; }
        __syncthreads();
        if (warp == 0)
        {
            uint32_t w = lane < 8 ? s_warp_sums[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1)
            {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) { w += y; }
            }
            if (lane < 8) { s_warp_sums[lane] = w; }
        }
        __syncthreads();
        if (threadIdx.x < 256) { tstart[threadIdx.x] = (warp > 0 ? s_warp_sums[warp - 1] : 0u) + x - total; }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < LI; j++)
        {
            if (dig[j] != 0xffffffffu)
            {
                const uint32_t pos = tstart[dig[j]] + whist[warp * 256 + dig[j]] + off[j];
                sk[pos] = key[j];
                sv[pos] = val[j];
            }
        }
        __syncthreads();
    };
    bool sorted = false;
    if (sub_shift >= 0)
    {
        if (threadIdx.x == 0) { s_max = 0u; }
        pass(sub_shift);
        if (threadIdx.x < 256)
        {
            atomicMax(&s_max, s_tot[threadIdx.x]);
            if (tab) { tab[blockIdx.x * 256u + threadIdx.x] = b0 + tstart[threadIdx.x]; }
        }
        __syncthreads();
        if (s_max <= 64u)
        {
            // warp w owns digits w, w + LB/32, ...: one per lane; small sub-buckets two at a time
            // with 16-lane networks, then 32- and 64-element networks for the larger ones
            constexpr int NWARP = LB / 32;
            const int myd = warp + NWARP * lane;
            const uint32_t myc = myd < 256 ? s_tot[myd] : 0u;
            uint32_t small = __ballot_sync(0xffffffffu, myc > 1u && myc <= 16u);
            uint32_t mid = __ballot_sync(0xffffffffu, myc > 16u && myc <= 32u);
            uint32_t big = __ballot_sync(0xffffffffu, myc > 32u);
            while (small)
            {
                const int l1 = __ffs(small) - 1;
                small &= small - 1u;
                const int l2 = small ? __ffs(small) - 1 : -1;
                if (l2 >= 0) { small &= small - 1u; }
                const int mine = lane < 16 ? l1 : l2;
                const uint32_t d = mine >= 0 ? (uint32_t)(warp + NWARP * mine) : 0u;
                warp_sort_n<K, 16>(sk, sv, tstart[d], mine >= 0 ? s_tot[d] : 0u, (uint32_t)lane & 15u);
            }
            while (mid)
            {
                const int l1 = __ffs(mid) - 1;
                mid &= mid - 1u;
                const uint32_t d = (uint32_t)(warp + NWARP * l1);
                warp_sort_n<K, 32>(sk, sv, tstart[d], s_tot[d], (uint32_t)lane);
            }
            while (big)
            {
                const int l1 = __ffs(big) - 1;
                big &= big - 1u;
                const uint32_t d = (uint32_t)(warp + NWARP * l1);
                warp_sort64<K>(sk, sv, tstart[d], s_tot[d], lane);
            }
            __syncthreads();
            sorted = true;
        }
        // else a crowded sub-bucket: the LSD passes below, from the registers (still in input order)
    }
    if (!sorted)
    {
        for (int p = 0; p < npass; p++)
        {
            pass(8 * p);
            if (p + 1 < npass)
            {
#pragma unroll
                for (int j = 0; j < LI; j++)
                {
                    const uint32_t e = (uint32_t)warp * (32u * LI) + (uint32_t)j * 32u + (uint32_t)lane;
                    if (e < m) { key[j] = sk[e]; val[j] = sv[e]; }
                }
                __syncthreads();
            }
        }
        if (npass == 0)  // nothing below the top digit: the bucket as it is
        {
#pragma unroll
            for (int j = 0; j < LI; j++)
            {
                const uint32_t e = (uint32_t)warp * (32u * LI) + (uint32_t)j * 32u + (uint32_t)lane;
                if (e < m) { sk[e] = key[j]; sv[e] = val[j]; }
            }
            __syncthreads();
        }
    }
    for (uint32_t i = threadIdx.x; i < m; i += LB)
    {
        kout[b0 + i] = sk[i];
        vout[b0 + i] = sv[i];
    }
}

} // namespace

// Look-back words the sort of n keys needs (passes x tiles x 256).
size_t sort_lookback_words(uint32_t n, int passes)
{
    const uint32_t tile = n <= RS_SMALL_MAX ? RS_BLOCK * 16 : RS_BLOCK * 8;
    return (size_t)passes * ((n + tile - 1) / tile) * 256;
}

template <typename K>
int radix_sort_pairs(K* keys, uint32_t* vals, bool vals_identity, uint32_t n, int key_bits, const uint32_t* hist,
                     const uint32_t* msd_hist, SortScratch& s, uint32_t* status, cudaStream_t st, K** keys_out,
                     uint32_t** vals_out, bool scratch_zeroed, uint32_t* msd_only_flag, uint32_t* msd_table,
                     const uint32_t** table_flag)
{
    *keys_out = keys;
    *vals_out = vals;
    if (table_flag) { *table_flag = nullptr; }
    if (n == 0) { return RT_OK; }
    if (n > LB_VAL) { return fail(RT_E_CAPACITY, "radix sort: more than 2^30 keys"); }
    const int passes = sort_passes(key_bits);
    const size_t lbw = sort_lookback_words(n, passes);
    // tile_counters: 64 pass counters, then the MSD path's 257 bucket starts and its flag
    if (s.keys_alt.ensure((size_t)n * sizeof(K)) || s.vals_alt.ensure((size_t)n * 4) || s.lookback.ensure(lbw * 4) ||
        s.tile_counters.ensure((64 + 260) * 4))
    {
        return RT_E_CUDA;
    }
    if (n <= RS_SMALL_MAX)
    {
        // per-bucket shape: the smaller one while an even spread leaves it 8% headroom
        constexpr uint32_t cap_small = (uint32_t)LS_SMALL_B * LS_SMALL_I, cap_large = (uint32_t)LS_LARGE_B * LS_LARGE_I;
        const bool msd = msd_hist != nullptr && key_bits > 8 && n <= 256u * cap_large;
        const bool small = (uint64_t)n * 108 <= (uint64_t)256 * cap_small * 100;
        uint32_t* bstart = s.tile_counters.as<uint32_t>() + 64;
        uint32_t* flag = bstart + 257;
        if (msd)
        {
            // top digit (bits key_bits-8 .. key_bits-1) by one onesweep pass keys -> alt, then the
            // buckets by the lower digits in shared memory, alt -> the buffer the LSD passes end in
            constexpr uint32_t tile = RS_BLOCK * 16;
            const uint32_t tiles = (n + tile - 1) / tile;
            constexpr size_t smem = onesweep_smem<K, 16>();
            constexpr size_t sm_small = local_sort_smem<K, LS_SMALL_B, LS_SMALL_I>();
            constexpr size_t sm_large = local_sort_smem<K, LS_LARGE_B, LS_LARGE_I>();
            static PerDeviceOnce attr;  // per key type and device
            if (int e = attr.once([] {
                    RT_CUDA(cudaFuncSetAttribute(k_onesweep<K, 16, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                    RT_CUDA(cudaFuncSetAttribute(k_local_sort<K, LS_SMALL_B, LS_SMALL_I, 2>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_small));
                    RT_CUDA(cudaFuncSetAttribute(k_local_sort<K, LS_LARGE_B, LS_LARGE_I, 1>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_large));
                    return (int)RT_OK;
                }))
            {
                return e;
            }
            K* kalt = s.keys_alt.as<K>();
            uint32_t* valt = s.vals_alt.as<uint32_t>();
            K* kfin = (passes & 1) ? kalt : keys;
            uint32_t* vfin = (passes & 1) ? valt : vals;
            const int npass = sort_passes(key_bits - 8);
            // more than 8 bits below the top digit: sub-buckets by the next 8 bits, sorted whole
            const int sub_shift = key_bits - 8 > 8 ? key_bits - 16 : -1;
            // the sub-buckets are the top 16 bits' values: the per-bucket sort writes their table
            uint32_t* ltab = sub_shift >= 0 ? msd_table : nullptr;
            if (table_flag) { *table_flag = ltab ? flag : nullptr; }
            // either this pass or the LSD passes use the look-back words (the flag picks one), so
            // one zeroing serves both
            if (!scratch_zeroed)
            {
                RT_CUDA(cudaMemsetAsync(s.lookback.as<uint32_t>(), 0, (size_t)tiles * 256 * 4, st));
                RT_CUDA(cudaMemsetAsync(s.tile_counters.as<uint32_t>() + 63, 0, 4, st));
            }
            k_msd_check<<<1, 256, 0, st>>>(msd_hist, n, small ? cap_small : cap_large, bstart, flag, msd_only_flag);
            k_onesweep<K, 16, 2><<<tiles, RS_BLOCK, smem, st>>>(keys, vals, vals_identity ? 1 : 0, kalt, valt, n, tiles,
                                                                key_bits - 8, msd_hist, s.tile_counters.as<uint32_t>() + 63,
                                                                s.lookback.as<uint32_t>(), status, flag, 1u);
            if (small)
            {
                k_local_sort<K, LS_SMALL_B, LS_SMALL_I, 2><<<256, LS_SMALL_B, sm_small, st>>>(kalt, valt, kfin, vfin, bstart,
                                                                                           flag, npass, sub_shift, ltab);
            }
            else
            {
                k_local_sort<K, LS_LARGE_B, LS_LARGE_I, 1><<<256, LS_LARGE_B, sm_large, st>>>(kalt, valt, kfin, vfin, bstart,
                                                                                           flag, npass, sub_shift, ltab);
            }
            count_launch(3);
            RT_CUDA(cudaGetLastError());
            if (msd_only_flag)  // no LSD fallback: the caller reads *msd_only_flag and sorts again if set
            {
                *keys_out = kfin;
                *vals_out = vfin;
                return RT_OK;
            }
        }
        return onesweep_passes<K, 16, 2>(keys, vals, vals_identity, n, passes, hist, s.keys_alt.as<K>(), s.vals_alt.as<uint32_t>(),
                                         s.lookback.as<uint32_t>(), s.tile_counters.as<uint32_t>(), status, st, keys_out,
                                         vals_out, msd ? flag : nullptr, 0u, scratch_zeroed);
    }
    return onesweep_passes<K, 8, 5>(keys, vals, vals_identity, n, passes, hist, s.keys_alt.as<K>(), s.vals_alt.as<uint32_t>(),
                                    s.lookback.as<uint32_t>(), s.tile_counters.as<uint32_t>(), status, st, keys_out, vals_out,
                                    nullptr, 0u, scratch_zeroed);
}

template int radix_sort_pairs<uint64_t>(uint64_t*, uint32_t*, bool, uint32_t, int, const uint32_t*, const uint32_t*,
                                        SortScratch&, uint32_t*, cudaStream_t, uint64_t**, uint32_t**, bool, uint32_t*,
                                        uint32_t*, const uint32_t**);
template int radix_sort_pairs<uint32_t>(uint32_t*, uint32_t*, bool, uint32_t, int, const uint32_t*, const uint32_t*,
                                        SortScratch&, uint32_t*, cudaStream_t, uint32_t**, uint32_t**, bool, uint32_t*,
                                        uint32_t*, const uint32_t**);

} // namespace rtb

namespace rtb
{

// The same passes on caller-provided scratch (no allocation): keys_alt / vals_alt hold n
// entries, lookback passes * tiles * 256 words, tile_counters 64 words. Used by the
// allocation-free entry point; the sort itself is the one above.
template <typename K>
int radix_sort_pairs_raw(K* keys, uint32_t* vals, uint32_t n, int key_bits, const uint32_t* hist, K* keys_alt,
                         uint32_t* vals_alt, uint32_t* lookback, uint32_t* tile_counters, uint32_t* status,
                         cudaStream_t st, K** keys_out, uint32_t** vals_out)
{
    *keys_out = keys;
    *vals_out = vals;
    if (n == 0) { return RT_OK; }
    const int passes = sort_passes(key_bits);
    if (n > RS_SMALL_MAX) { return fail(RT_E_CAPACITY, "radix sort on fixed scratch: at most 2^21 keys"); }
    static_assert(RS_BLOCK * 16 == RS_SMALL_TILE_KEYS, "fixed-scratch callers size the look-back words by this tile");
    return onesweep_passes<K, 16, 2>(keys, vals, true, n, passes, hist, keys_alt, vals_alt, lookback, tile_counters, status, st,
                                     keys_out, vals_out);
}

template int radix_sort_pairs_raw<uint64_t>(uint64_t*, uint32_t*, uint32_t, int, const uint32_t*, uint64_t*, uint32_t*,
                                            uint32_t*, uint32_t*, uint32_t*, cudaStream_t, uint64_t**, uint32_t**);
template int radix_sort_pairs_raw<uint32_t>(uint32_t*, uint32_t*, uint32_t, int, const uint32_t*, uint32_t*, uint32_t*,
                                            uint32_t*, uint32_t*, uint32_t*, cudaStream_t, uint32_t**, uint32_t**);

} // namespace rtb
