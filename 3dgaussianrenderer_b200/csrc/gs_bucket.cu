// Tile-bucket ordering of the frame pipeline: the whole-frame replacement
// for the reference's buildTileList + sortTileList + evaluateTileRanges
// (core/gaussian_render.cu:312-677).
//
// The reference emits (tile << 32 | depth, index) keys, radix-sorts all of
// them on tile and depth bits, then finds each tile's range.  Here the frame
// kernel has already counted every tile's keys, so:
//   1. tile scan   -- exclusive scan of the tile counts = each tile's range;
//   2. bucket emit -- every overlap is written straight into its tile's
//                     range, at a position claimed with one atomic, as
//                     (depth << 32 | slot);
//   3. tile sort   -- each tile's keys are ordered by depth in shared
//                     memory (LSD radix over only the depth bits that vary
//                     inside the tile), equal depths by view * n + i; small
//                     tiles by the raster CTA right before it blends them,
//                     larger ones by a separate kernel.
// The result per tile is exactly the order of a stable sort of the
// reference's keys emitted in Gaussian order: depth first, index among equal
// depths.  Each key crosses HBM about three times (emit, sort read, sorted
// index write) instead of twice per radix pass.
#include "gs_kernels.h"
#include "gs_tilesort.cuh"

#include <algorithm>

namespace gs {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Exclusive block scan of one int64 per thread; every thread must call it.
__device__ __forceinline__ int64_t excl_scan_block(const int64_t v, int64_t* s_tmp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_tmp[warp] = incl;
    __syncthreads();
    int64_t prefix = 0;
    for (int w = 0; w < warp; ++w) prefix += s_tmp[w];
    __syncthreads();
    return prefix + incl - v;
}

// OR and AND of one 64-bit value per thread over the block (pads pass
// or_v = 0, and_v = ~0); every thread must call it.
__device__ __forceinline__ uint64_t varying_bits_block(uint64_t or_v, uint64_t and_v, uint64_t* s_tmp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        or_v |= __shfl_xor_sync(kFull, or_v, o);
        and_v &= __shfl_xor_sync(kFull, and_v, o);
    }
    if (lane == 0) {
        s_tmp[warp] = or_v;
        s_tmp[kWarps + warp] = and_v;
    }
    __syncthreads();
    uint64_t o = 0, n = ~0ull;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        o |= s_tmp[w];
        n &= s_tmp[kWarps + w];
    }
    __syncthreads();
    return o ^ n;
}

}  // namespace

// ---- 1. tile scan -------------------------------------------------------------

__global__ void __launch_bounds__(kThreads) tile_scan_kernel(TileScanArgs a)
{
    constexpr int IPT = kTileScanItems / kThreads;
    __shared__ int64_t s_tmp[kWarps];
    __shared__ int64_t s_base;
    __shared__ int64_t s_blk;
    if (threadIdx.x == 0) s_blk = (int64_t)atomicAdd(a.block_counter, 1ull);
    __syncthreads();
    const int64_t blk = s_blk;
    const int64_t nblk = (a.tiles + kTileScanItems - 1) / kTileScanItems;
    if (blk >= nblk) return;
    const uint32_t epoch = a.epoch_dev ? *a.epoch_dev : a.epoch;

    // thread t owns tiles [first, first + IPT) of this block
    const int64_t first = blk * kTileScanItems + (int64_t)threadIdx.x * IPT;
    uint32_t c[IPT];
    int64_t sum = 0;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        c[j] = first + j < a.tiles ? a.count[first + j] : 0u;
        sum += c[j];
    }
    // leave the counts zeroed for the next frame (saves a clear per frame)
#pragma unroll
    for (int j = 0; j < IPT; ++j)
        if (first + j < a.tiles && c[j]) a.count[first + j] = 0u;
    const int64_t excl = excl_scan_block(sum, s_tmp);
    if (threadIdx.x == kThreads - 1) {
        const uint64_t agg = (uint64_t)(excl + sum);
        uint64_t prev = 0;
        uint64_t* st = a.status + blk;
        if (blk == 0) {
            store_status(st, status_word(kFlagP, epoch, agg));
        } else {
            store_status(st, status_word(kFlagA, epoch, agg));
            prev = look_back(a.status, blk, 1, epoch, a.err, kErrTimeout);
            store_status(st, status_word(kFlagP, epoch, prev + agg));
        }
        s_base = (int64_t)prev;
        if (blk == nblk - 1) {
            const int64_t total = (int64_t)(prev + agg);
            *a.total = total;
            if (a.sort_n) {
                *a.sort_n = total < a.capacity ? total : a.capacity;
                *a.overflow = total > a.capacity ? 1 : 0;
            }
        }
    }
    __syncthreads();
    int64_t run = s_base + excl;
    const int64_t cap = a.capacity;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const int64_t t = first + j;
        if (t < a.tiles) {
            if (c[j] > (uint32_t)kTileSortSmemKeys)
                a.big_list[a.tiles + atomicAdd(a.huge_count, 1u)] = (int32_t)t;
            else if (c[j] > (uint32_t)a.fused_cap)
                a.big_list[atomicAdd(a.big_count, 1u)] = (int32_t)t;
            a.cursor[t] = (unsigned long long)run;
            const int64_t lo = run < cap ? run : cap;
            const int64_t hi = run + c[j] < cap ? run + c[j] : cap;
            a.ranges[2 * t] = (int32_t)lo;
            a.ranges[2 * t + 1] = (int32_t)hi;
        }
        run += c[j];
    }
}

void launch_tile_scan(const TileScanArgs& a, cudaStream_t st)
{
    const int64_t blocks = (a.tiles + kTileScanItems - 1) / kTileScanItems;
    if (blocks <= 0) return;
    tile_scan_kernel<<<(unsigned)blocks, kThreads, 0, st>>>(a);
}

// ---- 1b. raster order of the tiles --------------------------------------------
//
// Tiles with more than 1.5x the average key count go first, so the longest
// raster CTAs start in the first wave instead of stretching the last one;
// the others follow (in reverse order, filled from the end).  One atomic
// per warp and class.
__global__ void __launch_bounds__(kThreads) tile_order_kernel(const int32_t* __restrict__ ranges, int64_t tiles,
                                                             const int64_t* __restrict__ total,
                                                             int32_t* __restrict__ order, unsigned int* heads)
{
    const int64_t t = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    const bool valid = t < tiles;
    const int64_t cnt = valid ? (int64_t)(__ldg(&ranges[2 * t + 1]) - __ldg(&ranges[2 * t])) : 0;
    const bool heavy = valid && 2 * cnt * tiles > 3 * *total;
    const unsigned bh = __ballot_sync(kFull, heavy), bl = __ballot_sync(kFull, valid && !heavy);
    const int lane = threadIdx.x & 31;
    unsigned int h0 = 0, l0 = 0;
    if (lane == 0) {
        if (bh) h0 = atomicAdd(&heads[0], (unsigned)__popc(bh));
        if (bl) l0 = atomicAdd(&heads[1], (unsigned)__popc(bl));
    }
    h0 = __shfl_sync(kFull, h0, 0);
    l0 = __shfl_sync(kFull, l0, 0);
    const unsigned below = lanemask_lt();
    if (heavy)
        order[h0 + __popc(bh & below)] = (int32_t)t;
    else if (valid)
        order[tiles - 1 - (int64_t)(l0 + __popc(bl & below))] = (int32_t)t;
}

void launch_tile_order(const int32_t* ranges, int64_t tiles, const int64_t* total, int32_t* order,
                       unsigned int* heads, cudaStream_t st)
{
    if (tiles <= 0) return;
    tile_order_kernel<<<(unsigned)((tiles + kThreads - 1) / kThreads), kThreads, 0, st>>>(ranges, tiles, total, order,
                                                                                         heads);
}

// ---- 2. bucket emit -----------------------------------------------------------

__device__ __forceinline__ uint32_t depth_bits(const float depth)
{
    return (uint32_t)(make_key(0, depth) & 0xFFFFFFFFull);
}

// Called by the whole warp: each lane with `has` writes one key into tile
// `gtile`'s bucket.  With `a.aggregate`, lanes of the same tile claim their
// positions with one atomic (see warp_count_hits for when that pays); the
// order inside a bucket is irrelevant, the tile sort orders it.
__device__ __forceinline__ void put_keys(const BucketEmitArgs& a, const bool has, const int64_t gtile,
                                         const uint32_t depth, const int64_t slot)
{
if (!a.aggregate) {
        if (!has) return;
        const unsigned long long pos = atomicAdd(&a.cursor[gtile], 1ull);
        if ((int64_t)pos < a.capacity) a.keys[pos] = ((uint64_t)depth << 32) | (uint32_t)slot;
        return;
    }
    const unsigned act = __ballot_sync(kFull, has);
    if (!has) return;
    const unsigned grp = __match_any_sync(act, (unsigned long long)gtile);
    const int leader = __ffs(grp) - 1;
    unsigned long long base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&a.cursor[gtile], (unsigned long long)__popc(grp));
    base = __shfl_sync(grp, base, leader);
    const unsigned long long pos = base + __popc(grp & lanemask_lt());
    if ((int64_t)pos < a.capacity) a.keys[pos] = ((uint64_t)depth << 32) | (uint32_t)slot;
}

// Grid-strided over the slots in 256-slot steps (the slot count is only
// known on the device).  Rectangles of at most 32 candidates expand the hit
// mask the frame kernel recorded; larger ones are re-tested by the whole
// warp, 32 candidates at a time.
__global__ void __launch_bounds__(kThreads) emit_bucket_kernel(BucketEmitArgs a)
{
    const int64_t nslots = (int64_t)*a.slot_count;
    const int lane = threadIdx.x & 31;
    for (int64_t base = (int64_t)blockIdx.x * kThreads; base < nslots; base += (int64_t)gridDim.x * kThreads) {
        const int64_t slot = base + threadIdx.x;
        int cand = 0, view = 0;
        int4 r = make_int4(0, 0, 0, 0);
        Ell e = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        uint32_t depth = 0;
        uint32_t m = 0;  // hit mask still to emit (rectangles of at most 32 candidates)
        int64_t toff = 0;
        int tiles_x = 0;
        if (slot < nslots) {
            // view * n + i < 2^31 (checked when the frame is planned): a
            // 32-bit division
            view = (int)((uint32_t)__ldg(&a.slot_gi[slot]) / (uint32_t)a.n);
            r = unpack_rect(__ldg(&a.rect[slot]));
            cand = rect_candidates(r);
            depth = depth_bits(__ldg(&a.z[slot]));
            if (cand <= 32) {
                const ViewParams& v = a.views[view];
                m = __ldg(&a.hitmask[slot]);
                toff = v.tile_offset;
                tiles_x = v.tiles_x;
                cand = 0;
            } else {
                const float2 c = __ldg(&a.xy[slot]);
                const float4 el = __ldg(&a.ell[slot]);
                e = {c.x, c.y, el.x, el.y, el.z, el.w};
            }
        }
        if (a.aggregate) {
            // one overlap per lane and step, the warp converged
            while (__any_sync(kFull, m != 0)) {
                const bool has = m != 0;
                int64_t gt = 0;
                if (has) {
                    const int c = __ffs(m) - 1;
                    m &= m - 1;
                    int cy, cx;
                    divmod_small(c, r.z, cy, cx);
                    gt = toff + (int64_t)(r.y + cy) * tiles_x + (r.x + cx);
                }
                put_keys(a, has, gt, depth, slot);
            }
        } else {
            // up to 4 overlaps per step: their cursor atomics are in flight
            // together, then the keys are written
            const uint64_t lo = (uint32_t)slot;
            while (m) {
                int64_t gt[4];
                unsigned long long pos[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    gt[u] = -1;
                    if (m) {
                        const int c = __ffs(m) - 1;
                        m &= m - 1;
                        int cy, cx;
                        divmod_small(c, r.z, cy, cx);
                        gt[u] = toff + (int64_t)(r.y + cy) * tiles_x + (r.x + cx);
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (gt[u] >= 0) pos[u] = atomicAdd(&a.cursor[gt[u]], 1ull);
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (gt[u] >= 0 && (int64_t)pos[u] < a.capacity) a.keys[pos[u]] = ((uint64_t)depth << 32) | lo;
            }
        }
        if (__ballot_sync(kFull, cand > 0) == 0) continue;
        // warp-cooperative walk over the large rectangles
        int incl = cand;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        const int excl = incl - cand;
        const int total = __shfl_sync(kFull, incl, 31);
        for (int cb = 0; cb < total; cb += 32) {
            const int c = cb + lane;
            int o = 0;
#pragma unroll
            for (int b = 16; b >= 1; b >>= 1) {
                const int t = __shfl_sync(kFull, incl, o + b - 1);
                if (t <= c) o += b;
            }
            Ell oe;
            oe.cx = __shfl_sync(kFull, e.cx, o);
            oe.cy = __shfl_sync(kFull, e.cy, o);
            oe.cs = __shfl_sync(kFull, e.cs, o);
            oe.sn = __shfl_sync(kFull, e.sn, o);
            oe.ex = __shfl_sync(kFull, e.ex, o);
            oe.ey = __shfl_sync(kFull, e.ey, o);
            int4 orr;
            orr.x = __shfl_sync(kFull, r.x, o);
            orr.y = __shfl_sync(kFull, r.y, o);
            orr.z = __shfl_sync(kFull, r.z, o);
            orr.w = __shfl_sync(kFull, r.w, o);
            const int oexcl = __shfl_sync(kFull, excl, o);
            const int oview = __shfl_sync(kFull, view, o);
            const uint32_t od = __shfl_sync(kFull, depth, o);
            bool hit = false;
            int64_t gt = 0;
            if (c < total) {
                int tile = 0;
                const ViewParams& v = a.views[oview];
                hit = candidate_hit(oe, orr, c - oexcl, v, tile);
                gt = v.tile_offset + tile;
            }
            put_keys(a, hit, gt, od, base + (threadIdx.x & ~31) + o);
        }
    }
}

void launch_emit_bucket(const BucketEmitArgs& a, int num_sms, cudaStream_t st)
{
    const int64_t blocks = std::min<int64_t>((a.max_slots + kThreads - 1) / kThreads, (int64_t)num_sms * 16);
    if (blocks <= 0) return;
    emit_bucket_kernel<<<(unsigned)blocks, kThreads, 0, st>>>(a);
}

// ---- 3. sort of the tiles too large for the raster CTAs -------------------------------
//
// Tiles up to the fused capacity are sorted by the raster CTA itself
// (gs_tilesort.cuh).  The larger ones, listed by the tile scan, are sorted
// here beforehand -- up to kTileSortSmemKeys keys by one counting pass in
// shared memory and ranks inside its runs (tilesort::count_sort_tile; the
// radix form of the raster CTA when a run is too long), up to
// kTileSortHugeKeys the same in one 1024-thread CTA, else by stable LSD
// passes through global memory -- and their order is written to `vals` for
// the rasteriser to read.  On the 64-view batch (57k such tiles, 92M keys)
// the counting form takes 1.98 ms against 2.33 ms for the radix form.

namespace {

using tilesort::Smem;

constexpr int kBigThreads = kThreads;

// One stable LSD pass of a tile too large for shared memory, by one CTA:
// digit histogram of the segment, then 4096-key chunks in order, each
// ranked in the block and written at its digits' running starts.
__device__ void global_pass(const uint64_t* in_k, const int32_t* in_v, uint64_t* out_k, int32_t* out_v, const int m,
                            const int shift, const Smem& sm)
{
    constexpr int NT = kBigThreads;
    constexpr int IPT = kTileSortSmemKeys / NT;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool owner = threadIdx.x < 256;
    uint32_t* hist = reinterpret_cast<uint32_t*>(sm.v);  // the value buffer is unused on this path
    if (owner) hist[threadIdx.x] = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < m; p += NT) atomicAdd(&hist[(unsigned)(in_k[p] >> shift) & 0xFFu], 1u);
    __syncthreads();
    const int ex = tilesort::excl_scan<NT>(owner ? (int)hist[threadIdx.x] : 0, sm.scan);
    if (owner) sm.run[threadIdx.x] = ex;
    __syncthreads();
    for (int c0 = 0; c0 < m; c0 += kTileSortSmemKeys) {
        uint64_t k[IPT];
        int32_t v[IPT];
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int p = c0 + warp * 32 * IPT + i * 32 + lane;
            if (p < m) {
                k[i] = in_k[p];
                v[i] = in_v ? in_v[p] : (int32_t)(uint32_t)k[i];
            } else {
                k[i] = ~0ull;
                v[i] = 0;
            }
        }
        int pos[IPT];
        tilesort::block_rank<NT, IPT>(k, shift, pos, sm);
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int p = c0 + warp * 32 * IPT + i * 32 + lane;
            if (p < m) {
                const unsigned d = (unsigned)(k[i] >> shift) & 0xFFu;
                const int dst = sm.run[d] + (pos[i] - sm.bexcl[d]);
                out_k[dst] = k[i];
                out_v[dst] = v[i];
            }
        }
        __syncthreads();
        if (owner) sm.run[threadIdx.x] += sm.dcount[threadIdx.x];
        __syncthreads();
    }
}

__device__ void sort_tile_global(const TileSortArgs& a, const int64_t start, const int m, const Smem& sm)
{
    constexpr int NT = kBigThreads;
    uint64_t* bk[2] = {a.keys + start, a.keys_alt + start};
    int32_t* bv[2] = {a.vals + start, a.vals_alt + start};
    int cur = 0;
    bool have_v = false;  // values not yet materialised: slot = low key bits

    auto vary_of = [&](const uint64_t hi_mask) {
        uint64_t o = 0, n = ~0ull;
        for (int p = threadIdx.x; p < m; p += NT) {
            const uint64_t x = bk[cur][p];
            o |= x;
            n &= x;
        }
        return tilesort::varying_bits<NT>(o, n, sm.red) & hi_mask;
    };
    auto run_passes = [&](uint64_t mask) {
        while (mask) {
            const int shift = __ffsll((long long)mask) - 1;
            mask &= ~(0xFFull << shift);
            global_pass(bk[cur], have_v ? bv[cur] : nullptr, bk[cur ^ 1], bv[cur ^ 1], m, shift, sm);
            cur ^= 1;
            have_v = true;
        }
    };

    // passes over the top 16 varying depth bits, then the runs of equal
    // prefixes into (depth, index) order (as in the shared-memory sort); the
    // keys keep their slots in the low bits throughout
    int shift;
    run_passes(tilesort::prefix_window(vary_of(0xFFFFFFFF00000000ull), a.prefix_bits, &shift));
    bool too_long = false;
    for (int p = threadIdx.x; p < m; p += NT) too_long |= tilesort::fix_run_at(bk[cur], m, p, shift, a.slot_gi);
    if (!__syncthreads_or(too_long)) {
        // result into a.vals
        for (int p = threadIdx.x; p < m; p += NT) bv[0][p] = (int32_t)(uint32_t)bk[cur][p];
        return;
    }
    // a long run of equal prefixes: sort again on (depth, index), the slots
    // carried as values
    for (int p = threadIdx.x; p < m; p += NT) {
        const uint64_t x = bk[cur][p];
        const int32_t s = (int32_t)(uint32_t)x;
        bv[cur][p] = s;
        bk[cur][p] = (x & 0xFFFFFFFF00000000ull) | (uint32_t)__ldg(&a.slot_gi[s]);
    }
    have_v = true;
    __syncthreads();
    run_passes(vary_of(~0ull));
    if (cur == 1)
        for (int p = threadIdx.x; p < m; p += NT) bv[0][p] = bv[1][p];
}

template <int IPT>
__device__ void sort_big_smem(const TileSortArgs& a, const int64_t start, const int m, const Smem& sm)
{
    tilesort::sort_tile<kBigThreads, IPT>(a.keys + start, m, a.slot_gi, sm, a.prefix_bits);
    for (int p = threadIdx.x; p < m; p += kBigThreads) a.vals[start + p] = (int32_t)(uint32_t)sm.k[p];
}

// The counting form (one placement pass, ranks inside the runs), the
// histogram in the values' part of shared memory; a tile with a long run of
// equal prefixes takes the radix form.
__device__ void sort_big_count(const TileSortArgs& a, const int64_t start, const int m, const Smem& sm)
{
    uint32_t* hist = reinterpret_cast<uint32_t*>(sm.v);
    const bool long_run =
        m <= kBigThreads * 8
            ? tilesort::count_sort_tile<kBigThreads, 8>(a.keys + start, m, a.slot_gi, sm, hist, a.vals + start)
            : tilesort::count_sort_tile<kBigThreads, 0>(a.keys + start, m, a.slot_gi, sm, hist, a.vals + start);
    if (!long_run) return;
    if (m <= 2048)
        sort_big_smem<8>(a, start, m, sm);
    else
        sort_big_smem<16>(a, start, m, sm);
}

}  // namespace

// Persistent CTAs over the big-tile list.
// 4 blocks per SM (64 registers; the spills are in the radix fallback)
constexpr int kBigBlocksPerSm = 4;
__global__ void __launch_bounds__(kBigThreads, kBigBlocksPerSm) tile_sort_big_kernel(TileSortArgs a)
{
    constexpr int NW = kBigThreads / 32;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t s_bexcl[256];
    __shared__ int32_t s_dcount[256];
    __shared__ int32_t s_run[256];
    __shared__ int32_t s_scan[NW];
    __shared__ uint64_t s_red[2 * NW];
    Smem sm;
    sm.k = reinterpret_cast<uint64_t*>(smem);
    sm.v = reinterpret_cast<int32_t*>(smem + kTileSortSmemKeys * 8);
    sm.whist = reinterpret_cast<uint32_t*>(smem);
    sm.bexcl = s_bexcl;
    sm.dcount = s_dcount;
    sm.scan = s_scan;
    sm.red = s_red;
    sm.run = s_run;
    const int nbig = (int)*a.big_count;
    for (int j = blockIdx.x; j < nbig; j += gridDim.x) {
        const int64_t t = a.big_list[j];
        const int64_t start = __ldg(&a.ranges[2 * t]);
        const int m = __ldg(&a.ranges[2 * t + 1]) - (int)start;
        if (m <= kTileSortSmemKeys)
            sort_big_count(a, start, m, sm);
        else
            sort_tile_global(a, start, m, sm);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// The tiles above kTileSortSmemKeys keys, by persistent 1024-thread CTAs
// (one per SM: 128 KB of keys and a 64 KB histogram of 2^15 bins in shared
// memory), in the counting form over 15 depth bits.  A tile above
// kTileSortHugeKeys keys, or with a run longer than kMaxRankRun, is handed
// to tile_sort_big_kernel: appended to its list, which that kernel, launched
// after this one on the same stream, reads when it starts.
constexpr int kHugeThreads = 1024;
constexpr int kHugeBits = 15;
__global__ void __launch_bounds__(kHugeThreads, 1) tile_sort_huge_kernel(TileSortArgs a)
{
    constexpr int NW = kHugeThreads / 32;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t s_scan[NW];
    __shared__ uint64_t s_red[2 * NW];
    Smem sm{};
    sm.k = reinterpret_cast<uint64_t*>(smem);
    sm.scan = s_scan;
    sm.red = s_red;
    uint32_t* hist = reinterpret_cast<uint32_t*>(smem + kTileSortHugeKeys * 8);
    const int nhuge = (int)*a.huge_count;
    for (int j = blockIdx.x; j < nhuge; j += gridDim.x) {
        const int64_t t = a.big_list[a.tiles + j];
        const int64_t start = __ldg(&a.ranges[2 * t]);
        const int m = __ldg(&a.ranges[2 * t + 1]) - (int)start;
        bool handed = m > kTileSortHugeKeys;
        if (!handed)
            handed = tilesort::count_sort_tile<kHugeThreads, 0, kHugeBits>(a.keys + start, m, a.slot_gi, sm, hist,
                                                                          a.vals + start);
        if (handed && threadIdx.x == 0) a.big_list[atomicAdd(a.big_count, 1u)] = (int32_t)t;
        __syncthreads();  // shared memory is reused by the next tile
    }
}

void launch_tile_sort(const TileSortArgs& a, int num_sms, cudaStream_t st)
{
    constexpr int big_smem = kTileSortSmemKeys * 12;
    constexpr int huge_smem = kTileSortHugeKeys * 12;
    static PerDeviceOnce attr;
    attr.run([] {
        cudaFuncSetAttribute(tile_sort_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big_smem);
        cudaFuncSetAttribute(tile_sort_huge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, huge_smem);
    });
    if (a.tiles <= 0) return;
    tile_sort_huge_kernel<<<(unsigned)num_sms, kHugeThreads, huge_smem, st>>>(a);
    tile_sort_big_kernel<<<(unsigned)(kBigBlocksPerSm * num_sms), kBigThreads, big_smem, st>>>(a);
}

}  // namespace gs
