// Block-level sort of one tile's bucket in shared memory, for CTAs of NT
// threads (32..256).  Used by the rasterisers (tiles of up to
// NT * kFusedIpt keys are sorted by the raster CTA itself, right before
// blending) and by the stand-alone sort of the larger tiles.
//
// Keys are (depth << 32 | slot).  The order produced is depth first and,
// among equal depths, the (view * n + i) index of the slot -- the order of
// a stable sort of the reference's (tile | depth) keys emitted in Gaussian
// order (core/gaussian_render.cu:591-632 sorts with CUB's stable radix
// sort).  LSD radix passes run only over the 8-bit windows covering the
// depth bits that vary inside the tile; equal-depth runs are then put in
// index order by a short insertion sort (the depth key has float resolution,
// so short runs are common), or, when some run is longer than kMaxTieRun,
// the whole tile is sorted again on (depth, index).
#pragma once

#include "gs_kernels.h"

namespace gs {
namespace tilesort {

constexpr int kMaxTieRun = 32;

// Views into the CTA's shared memory.
struct Smem {
    uint64_t* k;      // [capacity] keys; the warp histograms alias it while ranking
    int32_t* v;       // [capacity] values (slots) carried with the keys
    uint32_t* whist;  // [NT / 32][256], aliases k (needs capacity * 8 >= NT * 32 bytes)
    int32_t* bexcl;   // [256] digit start inside the ranked chunk
    int32_t* dcount;  // [256] digit count of the ranked chunk
    int32_t* scan;    // [NT / 32]
    uint64_t* red;    // [2 * NT / 32]
    int32_t* run;     // [256] running digit start (global-memory passes only)
};

// Exclusive scan of one int per thread over the NT threads; every thread
// must call it.
template <int NT>
__device__ __forceinline__ int excl_scan(const int v, int32_t* tmp)
{
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    if (NW == 1) return incl - v;
    if (lane == 31) tmp[warp] = incl;
    __syncthreads();
    int prefix = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) prefix += w < warp ? tmp[w] : 0;
    __syncthreads();
    return prefix + incl - v;
}

// Bits that differ between the values of the block (pads: or_v = 0,
// and_v = ~0); every thread must call it.
template <int NT>
__device__ __forceinline__ uint64_t varying_bits(uint64_t or_v, uint64_t and_v, uint64_t* tmp)
{
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        or_v |= __shfl_xor_sync(kFull, or_v, o);
        and_v &= __shfl_xor_sync(kFull, and_v, o);
    }
    if (NW == 1) return or_v ^ and_v;
    if (lane == 0) {
        tmp[warp] = or_v;
        tmp[NW + warp] = and_v;
    }
    __syncthreads();
    uint64_t o = 0, n = ~0ull;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        o |= tmp[w];
        n &= tmp[NW + w];
    }
    __syncthreads();
    return o ^ n;
}

// Stable rank of IPT keys per thread by the digit (key >> shift) & 0xFF.
// Item order: p = warp * 32 * IPT + i * 32 + lane.  pos[i] = rank of item
// i; sm.bexcl / sm.dcount hold each digit's start and count.  Thread t
// owns digits [t * D, (t + 1) * D), D = 256 / NT.  Every thread must call
// it; it ends with a barrier.
template <int NT, int IPT>
__device__ __forceinline__ void block_rank(const uint64_t (&key)[IPT], const int shift, int (&pos)[IPT],
                                           const Smem& sm)
{
    constexpr int NW = NT / 32;
    constexpr int D = NT >= 256 ? 1 : 256 / NT;  // digits per owning thread
    const bool owner = NT <= 256 || (int)threadIdx.x < 256;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* wh = sm.whist + warp * 256;
#pragma unroll
    for (int k = 0; k < 8; ++k) wh[lane + 32 * k] = 0;
    __syncwarp();
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const unsigned d = (unsigned)(key[i] >> shift) & 0xFFu;
        const unsigned peers = __match_any_sync(kFull, d);
        const uint32_t before = wh[d];
        const int below = __popc(peers & lt);
        __syncwarp();
        if (below == 0) wh[d] = before + __popc(peers);
        __syncwarp();
        pos[i] = (int)before + below;
    }
    __syncthreads();
    int cnt[D];
    int mine = 0;
    if (owner) {
#pragma unroll
        for (int dd = 0; dd < D; ++dd) {
            const int d = threadIdx.x * D + dd;
            int run = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                const uint32_t c = sm.whist[w * 256 + d];
                sm.whist[w * 256 + d] = (uint32_t)run;
                run += (int)c;
            }
            cnt[dd] = run;
            mine += run;
        }
    }
    int ex = excl_scan<NT>(mine, sm.scan);
    if (owner) {
#pragma unroll
        for (int dd = 0; dd < D; ++dd) {
            const int d = threadIdx.x * D + dd;
            sm.bexcl[d] = ex;
            sm.dcount[d] = cnt[dd];
            ex += cnt[dd];
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const unsigned dd = (unsigned)(key[i] >> shift) & 0xFFu;
        pos[i] += sm.bexcl[dd] + (int)sm.whist[warp * 256 + dd];
    }
    __syncthreads();  // whist (aliasing k) may be overwritten from here on
}

// LSD passes over the 8-bit windows covering `mask`, lowest first; the data
// lives in registers (p order) and goes through shared memory between
// passes.  Returns true (registers and sm.k / sm.v in sorted p order) when
// at least one pass ran.  Without CARRY_V the values stay where they are
// (the keys carry the slot themselves) and sm.v is not touched.
template <int NT, int IPT, bool CARRY_V = true>
__device__ __forceinline__ bool radix_passes(uint64_t (&k)[IPT], int32_t (&v)[IPT], uint64_t mask, const Smem& sm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool any = false;
    while (mask) {
        const int shift = __ffsll((long long)mask) - 1;
        mask &= ~(0xFFull << shift);
        int pos[IPT];
        block_rank<NT, IPT>(k, shift, pos, sm);
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            sm.k[pos[i]] = k[i];
            if (CARRY_V) sm.v[pos[i]] = v[i];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int p = warp * 32 * IPT + i * 32 + lane;
            k[i] = sm.k[p];
            if (CARRY_V) v[i] = sm.v[p];
        }
        __syncthreads();
        any = true;
    }
    return any;
}

__device__ __forceinline__ uint32_t depth_of(const uint64_t key) { return (uint32_t)(key >> 32); }

// Puts every run of equal depths that starts at one of this thread's items
// (p = first_p + i * stride) of `keys` (sorted by depth, slot in the low
// 32 bits) in index order.  Returns true when a run is too long to fix.
template <int IPT>
__device__ __forceinline__ bool fix_tie_runs(uint64_t* keys, const int m, const int first_p, const int stride,
                                             const int32_t* __restrict__ slot_gi)
{
    bool too_long = false;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const int p = first_p + i * stride;
        if (p >= m) continue;
        const uint32_t d = depth_of(keys[p]);
        if ((p > 0 && depth_of(keys[p - 1]) == d) || p + 1 >= m || depth_of(keys[p + 1]) != d) continue;
        int len = 2;
        while (p + len < m && depth_of(keys[p + len]) == d && len <= kMaxTieRun) ++len;
        if (len > kMaxTieRun) {
            too_long = true;
            continue;
        }
        for (int x = 1; x < len; ++x) {
            const uint64_t kx = keys[p + x];
            const int32_t gx = __ldg(&slot_gi[(uint32_t)kx]);
            int y = x - 1;
            while (y >= 0 && __ldg(&slot_gi[(uint32_t)keys[p + y]]) > gx) {
                keys[p + y + 1] = keys[p + y];
                --y;
            }
            keys[p + y + 1] = kx;
        }
    }
    return too_long;
}

// Sorts the m <= NT * IPT keys at `keys` into sm.k (p order, depth << 32 |
// slot).  Every thread of the CTA must call it; it ends with a barrier.
template <int NT, int IPT>
__device__ void sort_tile(const uint64_t* __restrict__ keys, const int m, const int32_t* __restrict__ slot_gi,
                          const Smem& sm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t k[IPT];
    int32_t v[IPT];
    uint64_t o = 0, n = ~0ull;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const int p = warp * 32 * IPT + i * 32 + lane;
        if (p < m) {
            k[i] = keys[p];
            v[i] = (int32_t)(uint32_t)k[i];
            o |= k[i];
            n &= k[i];
        } else {
            k[i] = ~0ull;  // pads rank last and are never read
            v[i] = 0;
        }
    }
    const uint64_t vary = varying_bits<NT>(o, n, sm.red) & 0xFFFFFFFF00000000ull;
    // the keys carry their slots: no values through these passes
    if (!radix_passes<NT, IPT, false>(k, v, vary, sm)) {
        // one depth for the whole tile: to shared memory as they are
#pragma unroll
        for (int i = 0; i < IPT; ++i) sm.k[warp * 32 * IPT + i * 32 + lane] = k[i];
        __syncthreads();
    }
    const bool too_long = fix_tie_runs<IPT>(sm.k, m, warp * 32 * IPT + lane, 32, slot_gi);
    if (__syncthreads_or(too_long)) {
        // a long run of equal depths: sort again on (depth, index)
        o = 0;
        n = ~0ull;
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int p = warp * 32 * IPT + i * 32 + lane;
            if (p < m) {
                v[i] = (int32_t)(uint32_t)k[i];  // the slot, carried through this sort
                k[i] = (k[i] & 0xFFFFFFFF00000000ull) | (uint32_t)__ldg(&slot_gi[v[i]]);
                o |= k[i];
                n &= k[i];
            }
        }
        radix_passes<NT, IPT>(k, v, varying_bits<NT>(o, n, sm.red), sm);
        // back to (depth << 32 | slot)
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int p = warp * 32 * IPT + i * 32 + lane;
            sm.k[p] = (k[i] & 0xFFFFFFFF00000000ull) | (uint32_t)v[i];
        }
        __syncthreads();
    }
}

}  // namespace tilesort
}  // namespace gs
