// Onesweep LSD radix sort of (tile|depth key, index) pairs and tile-range
// identification (replaces the reference's CUB DeviceRadixSort::SortPairs
// call at core/gaussian_render.cu:591-632 and evaluateTileRangesKernel at
// :634-660).
//
// One upfront pass builds the 8-bit digit histograms of every sort pass;
// then each pass is a single kernel: a block takes the next 4096-item tile
// (tiles are handed out by an atomic counter, so a block only ever waits on
// blocks that are already running), ranks its keys by digit with warp-level
// multi-split, publishes its per-digit counts, obtains the counts of all
// earlier tiles by decoupled look-back, reorders the tile in shared memory
// and writes each digit's run contiguously.  Only the significant key bits
// are sorted (32 depth bits plus the tile bits), in ceil(bits/8) passes.
#include "gs_kernels.h"

#include <algorithm>

namespace gs {

namespace {

__device__ __forceinline__ int64_t item_count(const int64_t host_n, const int64_t* dev_n)
{
    return dev_n ? *dev_n : host_n;
}

}  // namespace

// Digit histograms of all passes in one read of the keys.  Warp-private
// shared-memory histograms keep the atomics on the high (tile) digits,
// where many keys share a bin, from serialising a whole block.
__global__ void __launch_bounds__(256) sort_hist_kernel(const uint64_t* __restrict__ keys, int64_t host_n,
                                                        const int64_t* dev_n, int passes, uint32_t* __restrict__ hist)
{
    extern __shared__ uint32_t s_h[];  // [8 warps][passes][256]
    const int warp = threadIdx.x >> 5;
    for (int j = threadIdx.x; j < 8 * passes * kRadix; j += blockDim.x) s_h[j] = 0;
    __syncthreads();
    const int64_t n = item_count(host_n, dev_n);
    uint32_t* wh = s_h + warp * passes * kRadix;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = __ldg(&keys[i]);
        for (int p = 0; p < passes; ++p) atomicAdd(&wh[p * kRadix + (int)((k >> (8 * p)) & 0xFF)], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < passes * kRadix; j += blockDim.x) {
        uint32_t s = 0;
        for (int w = 0; w < 8; ++w) s += s_h[w * passes * kRadix + j];
        if (s) atomicAdd(&hist[j], s);
    }
}

struct SortPassArgs {
    const uint64_t* keys_in;
    const int32_t* vals_in;
    uint64_t* keys_out;
    int32_t* vals_out;
    int64_t host_n;
    const int64_t* dev_n;
    int shift;
    uint32_t epoch;
    const uint32_t* epoch_dev;  // non-null: epoch = *epoch_dev + pass
    int pass;
    const uint32_t* hist;  // this pass's 256 bins
    uint64_t* status;
    unsigned long long* counter;
    int* err;
};


// Exclusive scan over the block of one value per thread (threads past the
// digits pass 0).  Every thread of the block must call it.
__device__ __forceinline__ int64_t block_excl_scan(const int64_t v, int64_t* s_tmp)
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

// One onesweep pass over THREADS x IPT-key tiles (MINB blocks per SM).
template <int THREADS, int IPT, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) onesweep_kernel(SortPassArgs a)
{
    constexpr int kSortTile = THREADS * IPT;
    constexpr int kSortIpt = IPT;
    constexpr int kSortThreads = THREADS;
    constexpr int kSortWarps = THREADS / 32;
    static_assert(kSortWarps * kRadix * 4 <= kSortTile * 12, "warp histograms alias the tile buffer");
    static_assert(THREADS >= kRadix, "one thread per digit");
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* s_whist = reinterpret_cast<uint32_t*>(smem);                 // [warps][256] while ranking
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(smem);                  // [kSortTile] while scattering
    int32_t* s_vals = reinterpret_cast<int32_t*>(smem + kSortTile * 8);    // [kSortTile]
    __shared__ int64_t s_gstart[kRadix];
    __shared__ int64_t s_dstart[kRadix];
    __shared__ int32_t s_bexcl[kRadix];
    __shared__ int64_t s_scan[kSortWarps];
    __shared__ int64_t s_tile;

    const int64_t n = item_count(a.host_n, a.dev_n);
    const uint32_t epoch = a.epoch_dev ? *a.epoch_dev + (uint32_t)a.pass : a.epoch;
    const int64_t num_tiles = (n + kSortTile - 1) / kSortTile;
    if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(a.counter, 1ull);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= num_tiles) return;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool digit_thread = threadIdx.x < kRadix;
    const int64_t base = tile * kSortTile;
    const int valid = (int)min((int64_t)kSortTile, n - base);

    // global start of every digit (exclusive scan of this pass's histogram)
    {
        const int64_t ds = block_excl_scan(digit_thread ? (int64_t)a.hist[threadIdx.x] : 0, s_scan);
        if (digit_thread) s_dstart[threadIdx.x] = ds;
    }

    // warp w owns items [w * 32 * IPT, (w + 1) * 32 * IPT) of the tile, lane
    // l holds items l, l + 32, ... of that range (coalesced loads)
    uint64_t key[kSortIpt];
    int32_t val[kSortIpt];
    int rank[kSortIpt];
    const int64_t wbase = base + (int64_t)warp * 32 * kSortIpt + lane;
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
        const int64_t idx = wbase + i * 32;
        if (idx < n) {
            key[i] = __ldcs(&a.keys_in[idx]);
            val[i] = __ldcs(&a.vals_in[idx]);
        } else {
            key[i] = ~0ull;  // pads rank last, in digit 255, and are never written
            val[i] = 0;
        }
    }

    uint32_t* wh = s_whist + warp * kRadix;
#pragma unroll
    for (int k = 0; k < kRadix / 32; ++k) wh[lane + 32 * k] = 0;
    __syncwarp();

    // warp-level multi-split ranking: peers = lanes holding the same digit
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
        const unsigned d = (unsigned)(key[i] >> a.shift) & 0xFFu;
        unsigned peers = kFull;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const unsigned bal = __ballot_sync(kFull, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? bal : ~bal;
        }
        const uint32_t before = wh[d];
        const int below = __popc(peers & lt);
        __syncwarp();
        if (below == 0) wh[d] = before + __popc(peers);
        __syncwarp();
        rank[i] = (int)before + below;
    }
    __syncthreads();

    // per digit: warp offsets, block offsets, look-back across tiles
    int run = 0;
    if (digit_thread) {
        const int d = threadIdx.x;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = s_whist[w * kRadix + d];
            s_whist[w * kRadix + d] = (uint32_t)run;
            run += (int)c;
        }
    }
    const int64_t bex = block_excl_scan((int64_t)run, s_scan);
    if (digit_thread) {
        const int d = threadIdx.x;
        s_bexcl[d] = (int32_t)bex;
        uint64_t* st = a.status + tile * kRadix + d;
        uint64_t excl = 0;
        if (tile == 0) {
            store_status(st, status_word(kFlagP, epoch, (uint64_t)run));
        } else {
            store_status(st, status_word(kFlagA, epoch, (uint64_t)run));
            excl = look_back(a.status + d, tile, kRadix, epoch, a.err, kErrTimeout);
            store_status(st, status_word(kFlagP, epoch, excl + (uint64_t)run));
        }
        s_gstart[d] = s_dstart[d] + (int64_t)excl;
    }
    __syncthreads();

#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
        const unsigned d = (unsigned)(key[i] >> a.shift) & 0xFFu;
        rank[i] += s_bexcl[d] + (int)s_whist[warp * kRadix + d];  // position in the tile
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
        s_keys[rank[i]] = key[i];
        s_vals[rank[i]] = val[i];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortIpt; ++j) {
        const int p = j * kSortThreads + threadIdx.x;
        if (p < valid) {
            const uint64_t k = s_keys[p];
            const unsigned d = (unsigned)(k >> a.shift) & 0xFFu;
            const int64_t dst = s_gstart[d] + (p - s_bexcl[d]);
            a.keys_out[dst] = k;
            a.vals_out[dst] = s_vals[p];
        }
    }
}

int sort_passes(int key_bits) { return (key_bits + 7) / 8; }

template <int THREADS, int IPT, int MINB>
static void launch_pass_t(const SortPassArgs& a, int64_t num_items, cudaStream_t st)
{
    constexpr int tile = THREADS * IPT;
    constexpr int smem = tile * 12;
    static PerDeviceOnce attr;
    attr.run([] {
        cudaFuncSetAttribute(onesweep_kernel<THREADS, IPT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    const int64_t tiles = (num_items + tile - 1) / tile;
    onesweep_kernel<THREADS, IPT, MINB><<<(unsigned)tiles, THREADS, smem, st>>>(a);
}

// Tile shapes of the onesweep pass (the autotuner picks one per workload).
static void launch_pass(const SortPassArgs& a, int64_t num_items, int variant, cudaStream_t st)
{
    switch (variant) {
        case 1: launch_pass_t<256, 8, 4>(a, num_items, st); break;    // 2048 keys, 4 blocks/SM
        case 2: launch_pass_t<256, 16, 2>(a, num_items, st); break;   // 4096 keys, 16 keys/thread
        case 3: launch_pass_t<512, 16, 1>(a, num_items, st); break;   // 8192 keys
        default: launch_pass_t<512, 8, 2>(a, num_items, st); break;   // 4096 keys, 2 blocks/SM
    }
}

int sort_tile_items(int variant)
{
    switch (variant) {
        case 1: return 2048;
        case 3: return 8192;
        default: return 4096;
    }
}

int launch_sort(const uint64_t* keys_in, const int32_t* vals_in, uint64_t* keys_alt, int32_t* vals_alt,
                int64_t num_items, const int64_t* d_num_items, int key_bits, const SortScratch& s, uint32_t epoch,
                int num_sms, cudaStream_t st, int variant, const uint32_t* d_epoch)
{
    const int passes = sort_passes(key_bits);
    if (num_items <= 0 || passes == 0) return 0;
    static PerDeviceOnce attr;
    attr.run([] {
        cudaFuncSetAttribute(sort_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             8 * kMaxPasses * kRadix * 4);
    });
    cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * kMaxPasses * kRadix, st);
    cudaMemsetAsync(s.counters, 0, sizeof(unsigned long long) * kMaxPasses, st);
    const int hist_blocks = (int)std::min<int64_t>((int64_t)num_sms * 4, std::max<int64_t>(1, (num_items + 4095) / 4096));
    sort_hist_kernel<<<hist_blocks, 256, 8 * passes * kRadix * 4, st>>>(keys_in, num_items, d_num_items, passes,
                                                                         s.hist);
    // pass p reads A = (keys_in, vals_in) when p is even and B = (keys_alt,
    // vals_alt) when odd, and writes the other pair
    for (int p = 0; p < passes; ++p) {
        const bool even = (p % 2) == 0;
        SortPassArgs a;
        a.keys_in = even ? keys_in : keys_alt;
        a.vals_in = even ? vals_in : vals_alt;
        a.keys_out = even ? keys_alt : const_cast<uint64_t*>(keys_in);
        a.vals_out = even ? vals_alt : const_cast<int32_t*>(vals_in);
        a.host_n = num_items;
        a.dev_n = d_num_items;
        a.shift = 8 * p;
        a.epoch = epoch + (uint32_t)p;
        a.epoch_dev = d_epoch;
        a.pass = p;
        a.hist = s.hist + p * kRadix;
        a.status = s.status;
        a.counter = s.counters + p;
        a.err = s.err;
        launch_pass(a, num_items, variant, st);
    }
    return passes;
}

// ---- tile ranges -------------------------------------------------------------

__global__ void __launch_bounds__(256) ranges_kernel(const uint64_t* __restrict__ keys, int64_t host_n,
                                                     const int64_t* dev_n, int32_t* __restrict__ ranges)
{
    const int64_t n = item_count(host_n, dev_n);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t t = __ldg(&keys[i]) >> 32;
        if (i == 0 || (__ldg(&keys[i - 1]) >> 32) != t) ranges[2 * t] = (int32_t)i;
        if (i == n - 1 || (__ldg(&keys[i + 1]) >> 32) != t) ranges[2 * t + 1] = (int32_t)(i + 1);
    }
}

void launch_ranges(const uint64_t* keys, int64_t num_items, const int64_t* d_num_items, int32_t* ranges,
                   cudaStream_t st)
{
    if (num_items <= 0) return;
    const int64_t blocks = std::min<int64_t>((num_items + 255) / 256, (int64_t)device_sm_count() * 32);
    ranges_kernel<<<(unsigned)blocks, 256, 0, st>>>(keys, num_items, d_num_items, ranges);
}

}  // namespace gs
