// Block-level sort of one tile's bucket in shared memory, for CTAs of NT
// threads (32..256).  sort_tile is used by the rasterisers (tiles of up to
// NT * kFusedIpt keys are sorted by the raster CTA itself, right before
// blending); the stand-alone sort of the larger tiles uses count_sort_tile
// (below) and falls back on sort_tile.
//
// Keys are (depth << 32 | slot).  The order produced is depth first and,
// among equal depths, the (view * n + i) index of the slot -- the order of
// a stable sort of the reference's (tile | depth) keys emitted in Gaussian
// order (core/gaussian_render.cu:591-632 sorts with CUB's stable radix
// sort).  LSD radix passes run only over the top `prefix_bits` (16 by
// default, the autotuner's sort-bit-width knob: 8 to 32) of the depth bits
// that vary inside the tile, two 8-bit passes at 16; the keys
// are then in order of that prefix, and each run of equal prefixes is put
// in (depth, index) order by a short insertion sort.  On the benchmark's
// views no run is longer than 8 keys (the 16-bit prefix of the depth spread
// inside a tile is nearly unique); when some run is longer than
// kMaxTieRun, the whole tile is sorted again on (depth, index).
#pragma once

#include "gs_kernels.h"

namespace gs {
namespace tilesort {

constexpr int kMaxTieRun = 32;
constexpr int kDefaultPrefixBits = 16;

// The part of the varying depth bits that the radix passes sort: the top
// `bits` of them (8..32; anything else means the default).  *shift receives
// the lowest bit of that window; keys with the same key >> *shift form the
// runs left to the insertion sort.
__device__ __forceinline__ uint64_t prefix_window(const uint64_t vary_depth, int bits, int* shift)
{
    if (bits < 8 || bits > 32) bits = kDefaultPrefixBits;
    if (!vary_depth) {
        *shift = 32;
        return 0;
    }
    const int hi = 64 - __clzll((long long)vary_depth);  // one past the highest varying bit
    const int lo = hi - bits > 32 ? hi - bits : 32;
    *shift = lo;
    return vary_depth & (~0ull << lo);
}

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

// (depth, index) order of two keys of one tile: a before b?
__device__ __forceinline__ bool key_before(const uint64_t a, const uint64_t b, const int32_t* __restrict__ slot_gi)
{
    const uint32_t da = depth_of(a), db = depth_of(b);
    if (da != db) return da < db;
    return __ldg(&slot_gi[(uint32_t)a]) < __ldg(&slot_gi[(uint32_t)b]);
}

// If position p of `keys` (m keys sorted by the prefix key >> shift, slot in
// the low 32 bits) starts a run of equal prefixes, puts that run in (depth,
// index) order.  Returns true when the run is too long to fix this way.
// Runs are disjoint and every key of a run has the run's prefix, so the
// threads that fix different runs never disturb one another's tests.
__device__ __forceinline__ bool fix_run_at(uint64_t* keys, const int m, const int p, const int shift,
                                           const int32_t* __restrict__ slot_gi)
{
    const uint64_t pre = keys[p] >> shift;
    if ((p > 0 && (keys[p - 1] >> shift) == pre) || p + 1 >= m || (keys[p + 1] >> shift) != pre) return false;
    int len = 2;
    while (p + len < m && (keys[p + len] >> shift) == pre && len <= kMaxTieRun) ++len;
    if (len > kMaxTieRun) return true;
    for (int x = 1; x < len; ++x) {
        const uint64_t kx = keys[p + x];
        int y = x - 1;
        while (y >= 0 && key_before(kx, keys[p + y], slot_gi)) {
            keys[p + y + 1] = keys[p + y];
            --y;
        }
        keys[p + y + 1] = kx;
    }
    return false;
}

// fix_run_at for every item of this thread (p = first_p + i * stride).
template <int IPT>
__device__ __forceinline__ bool fix_prefix_runs(uint64_t* keys, const int m, const int first_p, const int stride,
                                                const int shift, const int32_t* __restrict__ slot_gi)
{
    bool too_long = false;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const int p = first_p + i * stride;
        if (p < m) too_long |= fix_run_at(keys, m, p, shift, slot_gi);
    }
    return too_long;
}

// Sorts the m <= NT * IPT keys at `keys` into sm.k (p order, depth << 32 |
// slot).  Every thread of the CTA must call it; it ends with a barrier.
template <int NT, int IPT>
__device__ void sort_tile(const uint64_t* __restrict__ keys, const int m, const int32_t* __restrict__ slot_gi,
                          const Smem& sm, const int prefix_bits)
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
    int shift;
    const uint64_t window =
        prefix_window(varying_bits<NT>(o, n, sm.red) & 0xFFFFFFFF00000000ull, prefix_bits, &shift);
    // the keys carry their slots: no values through these passes
    if (!radix_passes<NT, IPT, false>(k, v, window, sm)) {
        // one depth for the whole tile: to shared memory as they are
#pragma unroll
        for (int i = 0; i < IPT; ++i) sm.k[warp * 32 * IPT + i * 32 + lane] = k[i];
        __syncthreads();
    }
    const bool too_long = fix_prefix_runs<IPT>(sm.k, m, warp * 32 * IPT + lane, 32, shift, slot_gi);
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

// Counting-sort form of sort_tile for the stand-alone sort of the larger
// tiles (m keys, as many as sm.k holds; NT threads), writing the tile's
// slots in (depth, index) order to `out`.  One pass places every key in
// shared memory by the top BITS varying depth bits: a histogram of 16-bit
// counters packed two to a word (`hist`, 2^(BITS - 1) words; counts and
// offsets stay below 2^16, so m < 2^16), its exclusive scan, then each key
// takes the next position of its bin with a shared-memory atomic, so
// inside a bin the keys land in no particular order.  After the placement
// the histogram holds every bin's end, and each key's bin is the run
// [end(d - 1), end(d)) of the keys with its prefix: the key's rank among
// them in (depth, index) order, counted by the key's own thread, is its
// offset in the run.  That is the whole order (keys of different bins are
// ordered by the bin), so the pass need not be stable, and a run of L keys
// costs L comparisons per key, in parallel.  The callers keep about two
// bins per key (13 bits for up to 4096 keys, 15 for up to 16384); at 13
// bits no run on the benchmark's views is longer than 25 keys.
// IPT > 0: m <= NT * IPT, each thread holds its IPT keys in registers
// across the passes; IPT = 0: every pass reads the keys from global memory.
// Returns true when some run is longer than kMaxRankRun (`out` then holds
// only part of the order); the caller then sorts the tile another way.
// Every thread of the CTA must call it; it ends with a barrier.
constexpr int kCountBits = 13;
constexpr int kMaxRankRun = 64;

template <int NT, int IPT, int BITS = kCountBits>
__device__ bool count_sort_tile(const uint64_t* __restrict__ keys, const int m, const int32_t* __restrict__ slot_gi,
                                const Smem& sm, uint32_t* hist, int32_t* __restrict__ out)
{
    constexpr int NW = NT / 32;
    constexpr int kBins = 1 << BITS;
    constexpr int kWords = kBins / 2;
    constexpr int WPW = kWords / NW;  // histogram words scanned by each warp
    static_assert(WPW % 32 == 0, "histogram words per warp");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t o = 0, n = ~0ull;
    uint64_t kr[IPT > 0 ? IPT : 1];
    if constexpr (IPT > 0) {
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int p = i * NT + threadIdx.x;
            kr[i] = p < m ? keys[p] : 0ull;
            if (p < m) {
                o |= kr[i];
                n &= kr[i];
            }
        }
    } else {
        for (int p = threadIdx.x; p < m; p += NT) {
            const uint64_t k = keys[p];
            o |= k;
            n &= k;
        }
    }
    for (int w = threadIdx.x; w < kWords; w += NT) hist[w] = 0u;
    int shift;
    prefix_window(varying_bits<NT>(o, n, sm.red) & 0xFFFFFFFF00000000ull, BITS, &shift);
    // (varying_bits ends with a barrier: the cleared histogram is visible)
    auto count = [&](const uint64_t k) {
        const uint32_t d = (uint32_t)(k >> shift) & (kBins - 1);
        atomicAdd(&hist[d >> 1], 1u << ((d & 1u) << 4));
    };
    if constexpr (IPT > 0) {
#pragma unroll
        for (int i = 0; i < IPT; ++i)
            if (i * NT + (int)threadIdx.x < m) count(kr[i]);
    } else {
        for (int p = threadIdx.x; p < m; p += NT) count(keys[p]);
    }
    __syncthreads();
    // exclusive scan over the bins in order: word w holds bins 2w (low
    // half) and 2w + 1 (high half); each warp scans its WPW words
    int carry = 0;
    for (int r = 0; r < WPW / 32; ++r) {
        const int w = warp * WPW + r * 32 + lane;
        const uint32_t h = hist[w];
        const int lo = (int)(h & 0xFFFFu), c = lo + (int)(h >> 16);
        int incl = c;
#pragma unroll
        for (int of = 1; of < 32; of <<= 1) {
            const int t = __shfl_up_sync(kFull, incl, of);
            if (lane >= of) incl += t;
        }
        const int ex = carry + incl - c;
        hist[w] = (uint32_t)ex | ((uint32_t)(ex + lo) << 16);
        carry += __shfl_sync(kFull, incl, 31);
    }
    if (lane == 0) sm.scan[warp] = carry;
    __syncthreads();
    int wbase = 0;
#pragma unroll
    for (int w2 = 0; w2 < NW; ++w2) wbase += w2 < warp ? sm.scan[w2] : 0;
    if (wbase)
        for (int r = 0; r < WPW / 32; ++r) hist[warp * WPW + r * 32 + lane] += (uint32_t)wbase | ((uint32_t)wbase << 16);
    __syncthreads();
    auto place = [&](const uint64_t k) {
        const uint32_t d = (uint32_t)(k >> shift) & (kBins - 1);
        const uint32_t half = (d & 1u) << 4;
        const uint32_t old = atomicAdd(&hist[d >> 1], 1u << half);
        sm.k[(old >> half) & 0xFFFFu] = k;
    };
    if constexpr (IPT > 0) {
#pragma unroll
        for (int i = 0; i < IPT; ++i)
            if (i * NT + (int)threadIdx.x < m) place(kr[i]);
    } else {
        for (int p = threadIdx.x; p < m; p += NT) place(keys[p]);
    }
    __syncthreads();
    bool too_long = false;
    for (int p = threadIdx.x; p < m; p += NT) {
        const uint64_t k = sm.k[p];
        const uint32_t d = (uint32_t)(k >> shift) & (kBins - 1);
        const uint32_t e = (hist[d >> 1] >> ((d & 1u) << 4)) & 0xFFFFu;
        const uint32_t s0 = d ? (hist[(d - 1) >> 1] >> (((d - 1) & 1u) << 4)) & 0xFFFFu : 0u;
        if (e - s0 > (uint32_t)kMaxRankRun) {
            too_long = true;
            continue;
        }
        uint32_t rank = 0;
        for (uint32_t q = s0; q < e; ++q) rank += key_before(sm.k[q], k, slot_gi) ? 1u : 0u;
        out[s0 + rank] = (int32_t)(uint32_t)k;
    }
    return __syncthreads_or(too_long) != 0;
}

}  // namespace tilesort
}  // namespace gs
