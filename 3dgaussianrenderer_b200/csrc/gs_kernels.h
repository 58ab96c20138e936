// Kernel argument blocks and launchers of the gs_b200 pipeline (internal).
#pragma once

#include "gs_common.cuh"

#include <atomic>

namespace gs {

constexpr int kErrTimeout = 4;  // GS_ERR_DEVICE_TIMEOUT

// Runs a set-up step once per device.  Function attributes such as
// cudaFuncAttributeMaxDynamicSharedMemorySize belong to the current
// device's context, so a kernel that needs more than 48 KB of dynamic
// shared memory must be opted in on every device it runs on, not once per
// process.  Devices 0..63 are remembered; higher ones repeat the step on
// every call (it is idempotent).
class PerDeviceOnce {
public:
    template <class F>
    void run(F&& f)
    {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            dev = -1;
        }
        if (dev < 0 || dev >= 64) {
            f();
            return;
        }
        const uint64_t bit = 1ull << dev;
        if (done_.load(std::memory_order_acquire) & bit) return;
        f();
        done_.fetch_or(bit, std::memory_order_acq_rel);
    }

private:
    std::atomic<uint64_t> done_{0};
};

// Multiprocessor count of the current device (queried once per device).
inline int device_sm_count()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 148;
    }
    if (dev >= 0 && dev < 64) {
        const int c = cache[dev].load(std::memory_order_relaxed);
        if (c > 0) return c;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        return 148;
    }
    if (dev >= 0 && dev < 64) cache[dev].store(sms, std::memory_order_relaxed);
    return sms;
}

// Fused SH + projection + count + scan over (view, Gaussian) pairs.  A block
// owns one group of 256 Gaussians for `views_per_block` consecutive views;
// every view has its own look-back chain over the groups, so offsets are
// relative to the view's first key.
struct FrameArgs {
    int64_t n;          // Gaussians per view
    int64_t groups;     // ceil(n / 256)
    int32_t num_views;
    int32_t views_per_block;
    uint32_t epoch;     // look-back epoch of this launch
    const uint32_t* epoch_dev;  // non-null: the epoch is read here (graph replays)
    int64_t num_tiles;  // blocks = ceil(num_views / views_per_block) * groups
    const float4* pos;
    const float4* sr;
    const float* sh;    // grouped [ceil(n/256)][sh_count][256]
    int32_t sh_count;
    const float4* color_in;  // degree-0 scenes: colour from the model
    const ViewParams* views;
    const int32_t* orig;  // caller index of each stored Gaussian (null: stored in caller order)
    // outputs, per view at [view * n + i]; offsets for every Gaussian, the
    // rest only for Gaussians that overlap at least one tile
    int32_t raster_mode;  // GS_TERM_REFERENCE: color/xy/conic; GS_TERM_TMIN: rec
    float4* color;
    float2* xy;         // reference mode, or any mode when the rectangle has > 32 candidates
    float* z;
    float4* ell;        // only when the rectangle has > 32 candidates
    float4* conic;
    float4* rec;        // GS_TERM_TMIN raster record, 3 float4 per item (RasterRec)
    int2* rect;
    uint32_t* hitmask;  // bit c = candidate c overlaps (rectangles with <= 32 candidates)
    int32_t* offsets;   // exclusive key offset inside the view
    // scratch
    uint64_t* status;   // [num_views][groups] look-back words
    unsigned long long* tile_counter;
    int64_t* view_total;  // [num_views] keys per view
    int* err;
    // tile-bucket pipeline (launch_frame_project with bucket = true): the
    // (view, Gaussian) pairs that overlap a tile take slots from
    // `slot_counter` in any order; every per-item output above is written
    // at the slot instead of view * n + i, `offsets[slot]` receives
    // view * n + caller index, and each overlapped tile's key count is added to
    // tile_count[view tile offset + tile].
    uint32_t* tile_count;
    unsigned long long* slot_counter;
    int32_t aggregate;  // group same-tile count atomics of a warp (frames with few tiles)
    // probe outputs (diagnostics and tests; null in ordinary frames): the
    // projection of every Gaussian of every view at [view * n + caller
    // index] -- culled Gaussians as centre (-128, -128), depth -128, zero
    // ellipse and conic -- and the colour of those that reach a tile
    float2* probe_xy;
    float* probe_z;
    float4* probe_ell;
    float4* probe_conic;
    float4* probe_color;
};

// Bucket emission: every overlap of slot s is written as
// (depth bits << 32 | s) at an atomically claimed position of its tile's
// bucket (cursor[tile], preset to the tile's first key by the tile scan).
struct BucketEmitArgs {
    int64_t n;                       // Gaussians per view
    const unsigned long long* slot_count;
    int64_t max_slots;               // grid bound
    const ViewParams* views;
    const int32_t* slot_gi;          // view * n + i of each slot
    const int2* rect;
    const uint32_t* hitmask;
    const float2* xy;
    const float4* ell;
    const float* z;
    unsigned long long* cursor;      // [tiles]
    uint64_t* keys;
    int64_t capacity;
    int32_t aggregate;               // group same-tile cursor atomics of a warp (frames with few tiles)
};

// Frames of at most this many tiles (all views) group the same-tile atomics
// of a warp in the frame kernel's counts and the bucket emission.
constexpr int64_t kAggregateMaxTiles = 32768;

// Exclusive scan of the per-tile key counts into tile ranges and bucket
// cursors; the last block writes the key total.  Ranges are clamped to
// `capacity` (a frame whose keys do not fit is flagged, never overrun).
struct TileScanArgs {
    uint32_t* count;                 // [tiles]; zeroed again after the scan
    int64_t tiles;
    unsigned long long* cursor;      // [tiles] out: first key of the tile
    int32_t* ranges;                 // [2 * tiles] out: first, one past last
    uint64_t* status;                // look-back words, one per 4096 tiles
    unsigned long long* block_counter;
    uint32_t epoch;
    const uint32_t* epoch_dev;       // non-null: epoch read here
    int* err;
    int64_t* total;                  // K
    int64_t capacity;
    int64_t* sort_n;                 // min(K, capacity)
    int* overflow;                   // K > capacity
    int32_t* big_list;               // out: [0, tiles) tiles with more than fused_cap keys, up to
                                     // kTileSortSmemKeys; [tiles, 2 tiles) the larger ones
    unsigned int* big_count;
    unsigned int* huge_count;
    int32_t fused_cap;
};

// Per-tile sort of the buckets: each tile's keys are ordered by depth and,
// among equal depths, by view * n + i, which is the order of a stable sort
// of the reference's (tile | depth) keys emitted in Gaussian order.
struct TileSortArgs {
    const int32_t* ranges;
    int64_t tiles;
    uint64_t* keys;                  // bucketed (depth << 32 | slot); reordered in place
    uint64_t* keys_alt;              // scratch for tiles above the shared-memory capacity
    int32_t* vals;                   // out: slots in blend order
    int32_t* vals_alt;
    const int32_t* slot_gi;
    int32_t* big_list;               // tiles above the fused capacity (from the tile scan; the
                                     // tiles above kTileSortSmemKeys from index `tiles` on)
    unsigned int* big_count;
    const unsigned int* huge_count;
    int32_t prefix_bits;             // depth bits the radix passes sort (8..32; 0 = 16)
};
constexpr int kTileSortSmemKeys = 4096;
// Tiles of up to this many keys are sorted in the shared memory of one
// 1024-thread CTA (tile_sort_huge_kernel); larger ones by passes through
// global memory.
constexpr int kTileSortHugeKeys = 16384;
// Keys a tile may have to be sorted inside its raster CTA (TW * TH / 2
// threads, 8 keys each); larger tiles are sorted ahead of the raster.
constexpr int kFusedIpt = 8;
inline int fused_tile_capacity(int tile_w, int tile_h) { return tile_w * tile_h / 2 * kFusedIpt; }
constexpr int kTileScanItems = 1024;  // tiles per scan block

struct EmitArgs {
    int64_t n;
    int32_t num_views;
    const ViewParams* views;
    const int32_t* offsets;
    const int64_t* view_total;
    const int64_t* view_base;  // exclusive prefix of view_total
    const int2* rect;
    const uint32_t* hitmask;  // null: always re-test candidates
    const float2* xy;
    const float4* ell;
    const float* z;
    uint64_t* keys;
    int32_t* values;
    int64_t capacity;
};

// Raster record of one (view, Gaussian) for GS_TERM_TMIN, written by the
// frame kernel: alpha at an offset (dx, dy) from the centre is
// 2^(A dx^2 + B dx dy + C dy^2 + L) -- the conic scaled by -log2(e)/2 and
// L = log2(opacity), so alpha = opacity * exp(-q/2) with one exp2 -- and
// the cull extents bound the ellipse where alpha = kCullAlpha.  A record
// whose conic is not positive definite (non-finite projections) has
// L = -1e30 and empty extents: it contributes nothing, as the reference's
// saturate(NaN) = 0 makes it.
//   r0 = (x, y, ext_x, ext_y)   r1 = (A, B, C, L)   r2 = (red, green, blue, 0)
// (the cull test reads r0 only; r1 and r2 are read for the kept entries)
constexpr float kCullAlpha = 3.814697265625e-06f;  // 2^-18

// Onesweep LSD radix sort of (uint64 key, int32 value) pairs.  Tiles of
// 2048, 4096 or 8192 keys (sort_tile_items(variant)); kSortTile is the
// default variant's, kSortMinTile sizes the look-back words for all.
constexpr int kSortTile = 4096;
constexpr int kSortMinTile = 2048;
constexpr int kSortVariants = 4;
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;

struct SortScratch {
    uint32_t* hist;                   // [kMaxPasses][kRadix]
    uint64_t* status;                 // [max_tiles][kRadix] look-back words, reused by every pass
    unsigned long long* counters;     // [kMaxPasses] tile counters
    int* err;
    int64_t max_tiles;
};

struct RasterArgs {
    ViewParams view0;                 // single-view kernel: the view, by value
    const ViewParams* views;          // persistent kernel: all views
    int32_t num_views;
    int32_t write_empty;              // 1: tiles without entries are written as (0,0,0,0)
    int64_t num_tiles_total;          // sum of the views' tiles (of this launch's tiles when tile_base is used)
    int64_t tile_base;                // record raster without `order`: CTA b draws global tile tile_base + b
    const int32_t* ranges;            // [2 * num_tiles_total]
    const int32_t* values;
    const float2* xy;                 // indexed by value (reference-mode kernel)
    const float4* conic;
    const float4* color;
    const float4* rec;                // 3 float4 per value (record kernel); null: use xy/conic/color
    float t_min;
    unsigned long long* tile_counter; // persistent variant only
    // tile-bucket frames: a tile of at most fused_cap keys is sorted by its
    // raster CTA from the bucketed (depth << 32 | slot) keys; `values` then
    // only holds the order of the larger tiles.  keys == null: `values`
    // holds every tile's order.
    const uint64_t* keys;
    const int32_t* slot_gi;
    int32_t fused_cap;
    const int32_t* order;             // non-null: CTA (or queue entry) k rasterises tile order[k]
    // record raster (GS_TERM_TMIN) knobs: entries culled and staged per warp
    // step (32 or 64), and a persistent grid over the atomic tile queue
    // (tile_counter, zero at launch) instead of one CTA per tile
    int32_t rec_chunk;
    int32_t rec_persistent;
    int32_t sort_prefix_bits;         // depth bits the fused tile sort radix-sorts (8..32; 0 = 16)
};

void launch_sh_stage(int64_t n, const float4* pos, const float* sh, int sh_count, int deg, const ViewParams& v,
                     float4* color, cudaStream_t st);
void launch_project_stage(int64_t n, const float4* pos, const float4* sr, const ViewParams& v, float2* xy,
                          float* z, float4* ell, float4* conic, cudaStream_t st);
void launch_frame_project(const FrameArgs& a, int deg, cudaStream_t st, bool bucket = false);
void launch_tile_scan(const TileScanArgs& a, cudaStream_t st);
// Raster order of the tiles: those with more than 1.5x the average key count
// (ranges and *total from the tile scan) first.  heads[2] start at zero.
void launch_tile_order(const int32_t* ranges, int64_t tiles, const int64_t* total, int32_t* order,
                       unsigned int* heads, cudaStream_t st);
void launch_emit_bucket(const BucketEmitArgs& a, int num_sms, cudaStream_t st);
void launch_tile_sort(const TileSortArgs& a, int num_sms, cudaStream_t st);
void launch_count_stage(const FrameArgs& a, cudaStream_t st);
// view_base[v] = sum of view_total[u < v]; *total = sum of all.  With a
// non-null `sort_n`, also *sort_n = min(total, capacity) and *overflow = 1
// when the keys do not fit (frames whose key count is not known on the host).
void launch_view_base(const int64_t* view_total, int num_views, int64_t* view_base, int64_t* total, cudaStream_t st,
                      int64_t capacity = 0, int64_t* sort_n = nullptr, int* overflow = nullptr);
void launch_emit(const EmitArgs& a, cudaStream_t st);

// Sorts num_items pairs on bits [0, key_bits).  When d_num_items is non-null
// the item count is read on the device (graph-friendly; num_items is then
// an upper bound used to size the grids); likewise a non-null d_epoch
// replaces `epoch` as the look-back epoch of the first pass.  Returns the
// number of passes; the result is in the alternate buffers when that number
// is odd.
int launch_sort(const uint64_t* keys_in, const int32_t* vals_in, uint64_t* keys_alt, int32_t* vals_alt,
                int64_t num_items, const int64_t* d_num_items, int key_bits, const SortScratch& s, uint32_t epoch,
                int num_sms, cudaStream_t st, int variant = 0, const uint32_t* d_epoch = nullptr);
int sort_tile_items(int variant);
int sort_passes(int key_bits);

void launch_ranges(const uint64_t* keys, int64_t num_items, const int64_t* d_num_items, int32_t* ranges,
                   cudaStream_t st);
void launch_raster(const RasterArgs& a, int tile_w, int tile_h, int termination, bool persistent, int num_sms,
                   cudaStream_t st);

// Scene storage order (gs_scene.cu): 30-bit Morton codes of the centres over
// the box [lo, hi] with values = index, then the gather of every scene array
// through the sorted permutation (orig[j] = caller index of stored j).
void launch_morton(int64_t n, const float4* pos, const float lo[3], const float hi[3], uint64_t* keys, int32_t* vals,
                   cudaStream_t st);
void launch_scene_gather(int64_t n, const int32_t* perm, const float4* pos_in, const float4* sr_in,
                         const float4* col_in, const float* sh_in, int32_t sh_count, float4* pos, float4* sr,
                         float4* col, float* sh, int32_t* orig, cudaStream_t st);

}  // namespace gs
