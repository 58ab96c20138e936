// C-ABI of gs_b200: contexts, resident scenes, whole-frame and stage entry
// points (declared in include/gs_b200.h).
//
// Frame orchestration replaces the reference's frame loop
// (app/main.cpp:326-432) and Renderer::Render (core/renderer.cpp:94-139):
// everything runs on one stream with events between stages; the only host
// synchronisation inside a frame is the read of the exact key count K after
// the fused projection/count kernel (the reference syncs after every stage
// and once more for its tile counter).  Buffers grow on demand and are
// never truncated: the tile list is sized from the exact K.
#include "gs_kernels.h"
#include "../../include/gs_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <new>
#include <string>
#include <vector>

using namespace gs;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* what)
{
    g_last_error = what ? what : "";
    return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return GS_ERR_OOM;
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return GS_ERR_NO_DEVICE;
    return GS_ERR_CUDA;
}

#define GS_CUDA(call)                                            \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return cuda_fail(_e, #call);      \
    } while (0)

// Test hook (gs_test_fail_allocations): after g_alloc_skip more buffer
// allocations, the next g_fail_allocs fail as if the device were out of
// memory.
std::mutex g_alloc_hook_mu;
int g_alloc_skip = 0, g_fail_allocs = 0;
std::atomic<bool> g_alloc_hook{false};

bool injected_alloc_failure()
{
    if (!g_alloc_hook.load(std::memory_order_relaxed)) return false;
    std::lock_guard<std::mutex> lk(g_alloc_hook_mu);
    if (g_alloc_skip > 0) {
        --g_alloc_skip;
        return false;
    }
    if (g_fail_allocs > 0) {
        if (--g_fail_allocs == 0) g_alloc_hook = false;
        return true;
    }
    g_alloc_hook = false;
    return false;
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    // Grows to at least `need` bytes (25% headroom); old contents are lost.
    cudaError_t ensure(size_t need, bool zero = false)
    {
        if (need <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
        const size_t sz = std::max<size_t>(need + need / 4, 256);
        cudaError_t e = cudaMalloc(&p, sz);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return e;
        }
        bytes = sz;
        if (zero) return cudaMemset(p, 0, sz);
        return cudaSuccess;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const
    {
        return reinterpret_cast<T*>(p);
    }
};

// Small per-context device words, reset at the start of every frame (by a
// copy of the pinned `h_init`, which also carries the frame's look-back
// epochs, so a captured frame reads fresh epochs on every replay).
struct Counters {
    unsigned long long frame_tile;                 // frame kernel block queue
    unsigned long long raster_tile;                // persistent raster queue
    unsigned long long sort_tiles[kMaxPasses];     // onesweep tile queues
    unsigned long long scan_block;                 // tile scan block queue
    unsigned long long slots;                      // (view, Gaussian) slots taken by the frame kernel
    int64_t total;                                 // K
    int64_t sort_n;                                // min(K, key capacity)
    unsigned int big_tiles;                        // tiles sorted ahead of the raster (to 4096 keys)
    unsigned int huge_tiles;                       // those above 4096 keys
    unsigned int order_heads[2];                   // raster order: heavy tiles placed, others placed
    int err;
    int overflow;                                  // K > key capacity: the frame must be redone
    uint32_t epoch_scan, epoch_sort;               // look-back epochs of this frame
};

// A frame captured into a CUDA graph, or a frame seen once (no `exec` yet):
// the graph is captured the second time the same key comes along.
struct FrameGraph {
    uint64_t scene_uid = 0;
    gs_render_cfg cfg{};
    std::vector<int32_t> sizes;      // width, height per view
    std::vector<uint8_t*> outs;
    uint64_t layout = 0;             // context buffers the graph has baked in
    cudaGraphExec_t exec = nullptr;
    uint64_t last_use = 0;
    int seen = 0;                    // calls with this key
    int failed = 0;                  // capture failed: run this key without a graph
    int raster_groups = 0;           // raster launched per view group (host-output batches)
    int split = 0;                   // needed 2^31 tile keys or more: render as halves of the views
};
constexpr size_t kMaxGraphs = 8;
// gs_render_batch_host renders batches of more than this many views in
// groups, reading each group back while the next one renders.
constexpr int kHostChunkViews = 16;
constexpr int kHostGroupViews = 8;  // views per raster group of a T_min host batch
constexpr int kMaxRasterGroups = 8;

// Host read-back overlapped with the frame (T_min bucket frames): the
// raster runs one view group after the other, each group's end is marked by
// an event, and the group's images are copied on `copy` after it.
struct HostCopy {
    uint8_t* h_rgba = nullptr;
    cudaStream_t copy = nullptr;
    int groups = 0;
    int first_view[kMaxRasterGroups + 1] = {};  // group g = views [first_view[g], first_view[g + 1])
    size_t first_byte[kMaxRasterGroups + 1] = {};
};

// A tuned bucket of gs_autotune: the batching knobs that were fastest for
// scenes of 2^n_log2 .. 2^(n_log2+1) Gaussians, views of 2^px_log2 ..
// 2^(px_log2+1) pixels and a view count in views_bucket.
struct TuneEntry {
    int32_t n_log2 = 0, px_log2 = 0, views_bucket = 0, termination = 0, ordering = 0;
    int32_t tile_w = 16, tile_h = 16, views_per_block = 0, sort_variant = 0;
    int32_t ordering_picked = 0, raster_chunk = 0, raster_persistent = 0, sort_bits = 0;
    double ms = 0.0;
    uint64_t stamp = 0;  // insertion order: the oldest entry goes when the table is full
};
constexpr size_t kMaxTuneEntries = 256;

std::atomic<uint64_t> g_scene_uid{1};

// Failure-path self-test (gs_test_bounded_wait): a decoupled look-back
// from block 1 whose predecessor never publishes.  The wait gives up after
// `spin_limit` polls, sets the error word and returns, as every look-back of
// the pipeline does when a block it waits on never arrives.
struct WaitWords {
    uint64_t status[2];  // status[0] stays unpublished
    int err;
};

__global__ void wait_selftest_kernel(WaitWords* w, int spin_limit)
{
    if (threadIdx.x == 0) look_back(w->status, 1, 1, 1u, &w->err, kErrTimeout, spin_limit);
}

// Internal status of a frame whose tile lists need 2^31 entries or more
// (list positions are int32): run_frame renders it again as two frames
// over halves of its views.
constexpr int kSplitViews = -2;

}  // namespace

struct gs_scene {
    uint64_t uid = 0;  // never reused, unlike the address: keys the frame graphs
    int device = 0;
    int64_t n = 0;
    int32_t sh_degree = 0;
    int32_t sh_count = 0;
    DevBuf pos, sr, color, sh;
    DevBuf orig;  // int32 caller index of each stored Gaussian; empty: caller order
};

struct gs_ctx {
    int device = 0;
    int num_sms = 148;
    std::mutex mu;
    uint32_t epoch_scan = 1, epoch_sort = 1;
    DevBuf views;                          // ViewParams[]
    DevBuf color, xy, z, ell, conic, rect, offsets;  // per (view, Gaussian)
    DevBuf rec, hitmask;                   // T_min raster records (48 B), candidate hit masks
    DevBuf scan_status;                    // frame kernel look-back words, [view][group]
    DevBuf view_stats;                     // int64 [2][views]: keys per view, first key of view
    DevBuf keys0, vals0, keys1, vals1;     // tile lists
    DevBuf sort_hist, sort_status;
    DevBuf ranges;
    DevBuf tile_count, cursor, big_list;   // tile-bucket ordering: keys per tile, bucket fill cursors, big tiles
    DevBuf tile_order;                     // raster order of the tiles (heavy tiles first)
    DevBuf counters;
    DevBuf image;                          // images of the host-output variants
    Counters* h_counters = nullptr;        // pinned mirror
    Counters* h_init = nullptr;            // pinned per-frame reset image of the counters
    ViewParams* h_views = nullptr;         // pinned staging
    int h_views_cap = 0;
    cudaEvent_t ev[8] = {};
    int64_t key_capacity = 0;
    int64_t per_view_capacity = 0;         // Gaussians * views the splat buffers hold
    cudaStream_t cap_stream = nullptr;     // graph capture
    cudaStream_t copy_stream = nullptr;    // image read-back of the host-output batches
    cudaEvent_t ev_group[kMaxRasterGroups] = {};  // end of each raster view group
    bool tile_count_dirty = true;          // tile counts may be nonzero: clear before the next frame
    std::vector<FrameGraph> graphs;
    uint64_t use_clock = 0;
    std::vector<TuneEntry> tune;           // gs_autotune's table
    uint64_t tune_clock = 0;
    // the last tile-bucket frame (gs_probe_tile_lists); last_tiles < 0: none
    // since the lists last changed
    int64_t last_tiles = -1, last_keys = 0, last_slots = 0;
    int32_t last_fused_cap = 0;
};

namespace {

void make_view_params(const gs_camera& c, const gs_render_cfg& cfg, ViewParams& v)
{
    std::memcpy(v.view, c.view, sizeof(v.view));
    std::memcpy(v.cam, c.position, sizeof(v.cam));
    v.cot[0] = c.fov_cotangent[0];
    v.cot[1] = c.fov_cotangent[1];
    v.dsb[0] = c.depth_scale_bias[0];
    v.dsb[1] = c.depth_scale_bias[1];
    v.aspect = c.aspect;
    v.width = c.width;
    v.height = c.height;
    v.tile_w = cfg.tile_w;
    v.tile_h = cfg.tile_h;
    v.tiles_x = (c.width + cfg.tile_w - 1) / cfg.tile_w;
    v.tiles_y = (c.height + cfg.tile_h - 1) / cfg.tile_h;
    v.tiles_xf = (float)c.width / (float)cfg.tile_w;
    v.tiles_yf = (float)c.height / (float)cfg.tile_h;
    v.tclip_x = ((float)cfg.tile_w / (float)c.width) * 2.0f;
    v.tclip_y = ((float)cfg.tile_h / (float)c.height) * 2.0f;
    v.texel_x = 2.0f / (float)c.width;
    v.texel_y = 2.0f / (float)c.height;
    // gaussian_render.cu:184-186: (1/pi) * texel * texel, per axis
    const float k_Pi = 3.14159265359f;
    v.bump_x = ((1.0f / k_Pi) * v.texel_x) * v.texel_x;
    v.bump_y = ((1.0f / k_Pi) * v.texel_y) * v.texel_y;
    v.tile_offset = 0;
    v.out = nullptr;
}

bool valid_cfg(const gs_render_cfg& c)
{
    const bool shape = (c.tile_w == 16 && c.tile_h == 16) || (c.tile_w == 16 && c.tile_h == 8) ||
                       (c.tile_w == 8 && c.tile_h == 8);
    return shape && c.sh_max_degree >= 0 && c.sh_max_degree <= 3 && c.sort_variant >= 0 &&
           c.sort_variant < kSortVariants && c.views_per_block >= 0 &&
           (c.ordering == GS_ORDER_BUCKETS || c.ordering == GS_ORDER_ONESWEEP || c.ordering == GS_ORDER_AUTO) &&
           (c.graph == 0 || c.graph == 1) && (c.raster_chunk == 0 || c.raster_chunk == 32 || c.raster_chunk == 64) &&
           (c.raster_persistent == 0 || c.raster_persistent == 1) &&
           (c.sort_bits == 0 || (c.sort_bits >= 8 && c.sort_bits <= 32)) &&
           (c.termination == GS_TERM_REFERENCE || c.termination == GS_TERM_TMIN);
}

bool valid_cam(const gs_camera* c)
{
    return c && c->width > 0 && c->height > 0 && c->width <= 16384 && c->height <= 16384;
}

int eval_degree(const gs_scene* s, const gs_render_cfg& cfg) { return std::min(s->sh_degree, cfg.sh_max_degree); }

float ms_between(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();  // not a frame failure: leave no error behind
        ms = 0.f;
    }
    return ms;
}

// Records `ev` on `st`; under stream capture as an event-record node of the
// graph (an ordinary record would only become an internal dependency), so
// replays can still be timed.
cudaError_t record(cudaEvent_t ev, cudaStream_t st, bool capturing)
{
    return capturing ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal) : cudaEventRecord(ev, st);
}

// Onesweep tile shape of the stage sort: 8192-key tiles up to 16M keys (on
// the 2.6M keys of a 1024^2 frame they cut the look-back chain to a wave:
// 0.253 against 0.258 ms with 4096-key tiles), the default shape above
// (17.1 against 17.5 ms on 222M keys).
int stage_sort_variant(int64_t num_keys) { return num_keys <= (1ll << 24) ? 3 : 0; }

int ensure_sort_scratch(gs_ctx* ctx, int64_t num_items)
{
    const int64_t tiles = (num_items + kSortMinTile - 1) / kSortMinTile;
    if (ctx->sort_hist.ensure(sizeof(uint32_t) * kMaxPasses * kRadix) != cudaSuccess) return fail(GS_ERR_OOM, "sort hist");
    const size_t need = sizeof(uint64_t) * (size_t)std::max<int64_t>(tiles, 1) * kRadix;
    if (need > ctx->sort_status.bytes) {
        // fresh words must read as unpublished for every epoch
        if (ctx->sort_status.ensure(need, true) != cudaSuccess) return fail(GS_ERR_OOM, "sort status");
    }
    return GS_OK;
}

// Reserves `count` consecutive epochs of a look-back status array, clearing
// the array when the 16-bit epoch would wrap.
uint32_t take_epochs(uint32_t& epoch, uint32_t count, DevBuf& status, cudaStream_t st)
{
    if (epoch + count > 0xFFFFu) {
        if (status.p) cudaMemsetAsync(status.p, 0, status.bytes, st);
        epoch = 1;
    }
    const uint32_t e = epoch;
    epoch += count;
    return e;
}

int ensure_ctx_host(gs_ctx* ctx, int num_views)
{
    if (num_views > ctx->h_views_cap) {
        if (ctx->h_views) cudaFreeHost(ctx->h_views);
        ctx->h_views = nullptr;
        GS_CUDA(cudaMallocHost(&ctx->h_views, sizeof(ViewParams) * (size_t)num_views));
        ctx->h_views_cap = num_views;
    }
    if (ctx->views.ensure(sizeof(ViewParams) * (size_t)num_views) != cudaSuccess) return fail(GS_ERR_OOM, "views");
    return GS_OK;
}

// Grows the tile lists (both ping-pong pairs: tiles above the shared-memory
// sort capacity use the second) to hold `keys` keys.
int ensure_key_buffers(gs_ctx* ctx, int64_t keys)
{
    if (keys <= ctx->key_capacity && ctx->keys0.p) return GS_OK;
    const size_t k = (size_t)std::max<int64_t>(keys, 1);
    if (ctx->keys0.ensure(8 * k) || ctx->keys1.ensure(8 * k) || ctx->vals0.ensure(4 * k) || ctx->vals1.ensure(4 * k)) {
        ctx->key_capacity = 0;  // some lists were released: regrow them all next time
        return fail(GS_ERR_OOM, "tile lists");
    }
    const int64_t cap = std::min(std::min((int64_t)(ctx->keys0.bytes / 8), (int64_t)(ctx->keys1.bytes / 8)),
                                 std::min((int64_t)(ctx->vals0.bytes / 4), (int64_t)(ctx->vals1.bytes / 4)));
    ctx->key_capacity = std::min<int64_t>(cap, (1ll << 31) - 1);
    return GS_OK;
}

// One frame over `num_views` views of `scene` with GS_ORDER_ONESWEEP: keys
// in Gaussian order at scanned offsets, radix sort, ranges.  The host reads
// the exact key count between the projection and the emission.
int run_frame_onesweep(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int num_views, const gs_render_cfg& cfg,
              uint8_t* const* outs, gs_stats* stats, cudaStream_t st)
{
    if (!valid_cfg(cfg)) return fail(GS_ERR_INVALID, "invalid render cfg");
    if (num_views <= 0) return fail(GS_ERR_INVALID, "no views");
    for (int v = 0; v < num_views; ++v) {
        if (!valid_cam(&cams[v])) return fail(GS_ERR_INVALID, "invalid camera");
        if (!outs[v]) return fail(GS_ERR_INVALID, "null output");
    }
    GS_CUDA(cudaSetDevice(ctx->device));
    int rc = ensure_ctx_host(ctx, num_views);
    if (rc) return rc;

    const int64_t n = scene->n;
    int64_t tiles_total = 0;
    for (int v = 0; v < num_views; ++v) {
        ViewParams& vp = ctx->h_views[v];
        make_view_params(cams[v], cfg, vp);
        vp.tile_offset = tiles_total;
        vp.out = reinterpret_cast<uchar4*>(outs[v]);
        tiles_total += (int64_t)vp.tiles_x * vp.tiles_y;
    }
    if (tiles_total >= (1ll << 31)) return fail(GS_ERR_INVALID, "too many tiles");
    const int64_t items = n * num_views;
    if (items >= (1ll << 31)) return fail(GS_ERR_INVALID, "views x Gaussians exceeds 2^31");
    const int64_t groups = (n + 255) / 256;
    // views per block: the SH chunk of a group is read once per block
    const int vpb = std::min(num_views, cfg.views_per_block > 0 ? cfg.views_per_block : 16);
    const int64_t blocks = groups * ((num_views + vpb - 1) / vpb);
    const int64_t chains = groups * num_views;

    // per-(view, Gaussian) buffers
    if (items > ctx->per_view_capacity) {
        const size_t m = (size_t)items;
        if (ctx->color.ensure(16 * m) || ctx->xy.ensure(8 * m) || ctx->z.ensure(4 * m) || ctx->ell.ensure(16 * m) ||
            ctx->conic.ensure(16 * m) || ctx->rect.ensure(8 * m) || ctx->offsets.ensure(4 * m) ||
            ctx->rec.ensure(48 * m) || ctx->hitmask.ensure(4 * m)) {
            ctx->per_view_capacity = 0;  // some of them were released: re-check them all next time
            return fail(GS_ERR_OOM, "splat buffers");
        }
        ctx->per_view_capacity = items;
    }
    if (sizeof(uint64_t) * (size_t)std::max<int64_t>(chains, 1) > ctx->scan_status.bytes) {
        if (ctx->scan_status.ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(chains, 1), true))
            return fail(GS_ERR_OOM, "scan status");
    }
    if (ctx->view_stats.ensure(sizeof(int64_t) * 2 * (size_t)num_views)) return fail(GS_ERR_OOM, "view stats");
    int64_t* view_total = ctx->view_stats.as<int64_t>();
    int64_t* view_base = view_total + num_views;
    if (ctx->ranges.ensure(sizeof(int32_t) * 2 * (size_t)tiles_total)) return fail(GS_ERR_OOM, "ranges");

    Counters* dc = ctx->counters.as<Counters>();
    GS_CUDA(cudaMemcpyAsync(ctx->views.p, ctx->h_views, sizeof(ViewParams) * num_views, cudaMemcpyHostToDevice, st));
    GS_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), st));
    GS_CUDA(cudaEventRecord(ctx->ev[0], st));

    // 1. SH + projection + exact tile counts + key offsets
    FrameArgs fa{};
    fa.n = n;
    fa.groups = groups;
    fa.num_views = num_views;
    fa.views_per_block = vpb;
    fa.epoch = take_epochs(ctx->epoch_scan, 1, ctx->scan_status, st);
    fa.num_tiles = blocks;
    fa.pos = scene->pos.as<float4>();
    fa.orig = scene->orig.as<int32_t>();
    fa.sr = scene->sr.as<float4>();
    fa.sh = scene->sh.as<float>();
    fa.sh_count = scene->sh_count;
    fa.color_in = scene->color.as<float4>();
    fa.views = ctx->views.as<ViewParams>();
    fa.color = ctx->color.as<float4>();
    fa.xy = ctx->xy.as<float2>();
    fa.z = ctx->z.as<float>();
    fa.ell = ctx->ell.as<float4>();
    fa.conic = ctx->conic.as<float4>();
    fa.rect = ctx->rect.as<int2>();
    fa.rec = ctx->rec.as<float4>();
    fa.hitmask = ctx->hitmask.as<uint32_t>();
    fa.raster_mode = cfg.termination;
    fa.offsets = ctx->offsets.as<int32_t>();
    fa.status = ctx->scan_status.as<uint64_t>();
    fa.tile_counter = &dc->frame_tile;
    fa.view_total = view_total;
    fa.err = &dc->err;
    // degree-0 scenes blend the model colours (ply_parser.cpp:383,389); SH
    // scenes evaluate min(scene degree, cfg degree) (gaussian_render.cu:392)
    if (scene->sh_degree == 0 && !scene->color.p) return fail(GS_ERR_INVALID, "scene has no colour");
    const int deg = scene->sh_degree > 0 ? eval_degree(scene, cfg) : -1;
    if (n > 0) {
        launch_frame_project(fa, deg, st);
        launch_view_base(view_total, num_views, view_base, &dc->total, st);
    }
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaEventRecord(ctx->ev[1], st));
    GS_CUDA(cudaMemcpyAsync(ctx->h_counters, dc, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    GS_CUDA(cudaStreamSynchronize(st));
    if (ctx->h_counters->err) return fail(GS_ERR_DEVICE_TIMEOUT, "projection look-back timed out");
    const int64_t K = n > 0 ? ctx->h_counters->total : 0;
    if (K >= (1ll << 31)) return fail(kSplitViews, "more than 2^31 tile keys");

    // 2. emit keys
    ctx->last_tiles = -1;  // the bucket frame's lists are overwritten from here on
    if (K > ctx->key_capacity) {
        rc = ensure_key_buffers(ctx, K);
        if (rc) return rc;
    }
    rc = ensure_sort_scratch(ctx, K);
    if (rc) return rc;
    GS_CUDA(cudaEventRecord(ctx->ev[2], st));
    EmitArgs ea{};
    ea.n = n;
    ea.num_views = num_views;
    ea.views = ctx->views.as<ViewParams>();
    ea.offsets = ctx->offsets.as<int32_t>();
    ea.view_total = view_total;
    ea.view_base = view_base;
    ea.rect = ctx->rect.as<int2>();
    ea.hitmask = ctx->hitmask.as<uint32_t>();
    ea.xy = ctx->xy.as<float2>();
    ea.ell = ctx->ell.as<float4>();
    ea.z = ctx->z.as<float>();
    ea.keys = ctx->keys0.as<uint64_t>();
    ea.values = ctx->vals0.as<int32_t>();
    ea.capacity = ctx->key_capacity;
    if (K > 0) launch_emit(ea, st);
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaEventRecord(ctx->ev[3], st));

    // 3. sort on the significant bits
    const int key_bits = gs_key_bits(tiles_total);
    SortScratch ss;
    ss.hist = ctx->sort_hist.as<uint32_t>();
    ss.status = ctx->sort_status.as<uint64_t>();
    ss.counters = dc->sort_tiles;
    ss.err = &dc->err;
    ss.max_tiles = (int64_t)(ctx->sort_status.bytes / (8 * kRadix));
    int passes = 0;
    if (K > 0) {
        const uint32_t ep = take_epochs(ctx->epoch_sort, (uint32_t)sort_passes(key_bits), ctx->sort_status, st);
        passes = launch_sort(ctx->keys0.as<uint64_t>(), ctx->vals0.as<int32_t>(), ctx->keys1.as<uint64_t>(),
                             ctx->vals1.as<int32_t>(), K, nullptr, key_bits, ss, ep, ctx->num_sms, st,
                             cfg.sort_variant);
    }
    GS_CUDA(cudaGetLastError());
    const uint64_t* skeys = (passes % 2) ? ctx->keys1.as<uint64_t>() : ctx->keys0.as<uint64_t>();
    const int32_t* svals = (passes % 2) ? ctx->vals1.as<int32_t>() : ctx->vals0.as<int32_t>();
    GS_CUDA(cudaEventRecord(ctx->ev[4], st));

    // 4. tile ranges + raster
    GS_CUDA(cudaMemsetAsync(ctx->ranges.p, 0xFF, sizeof(int32_t) * 2 * (size_t)tiles_total, st));
    if (K > 0) launch_ranges(skeys, K, nullptr, ctx->ranges.as<int32_t>(), st);
    RasterArgs ra{};
    ra.view0 = ctx->h_views[0];
    ra.views = ctx->views.as<ViewParams>();
    ra.num_views = num_views;
    ra.write_empty = 1;
    ra.num_tiles_total = tiles_total;
    ra.ranges = ctx->ranges.as<int32_t>();
    ra.values = svals;
    ra.xy = ctx->xy.as<float2>();
    ra.conic = ctx->conic.as<float4>();
    ra.color = ctx->color.as<float4>();
    ra.rec = cfg.termination == GS_TERM_TMIN ? ctx->rec.as<float4>() : nullptr;
    ra.t_min = cfg.t_min;
    ra.tile_counter = &dc->raster_tile;
    ra.rec_chunk = cfg.raster_chunk;
    ra.rec_persistent = cfg.raster_persistent;
    launch_raster(ra, cfg.tile_w, cfg.tile_h, cfg.termination, num_views > 1, ctx->num_sms, st);
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaEventRecord(ctx->ev[5], st));
    GS_CUDA(cudaMemcpyAsync(&ctx->h_counters->err, &dc->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    GS_CUDA(cudaStreamSynchronize(st));
    if (ctx->h_counters->err) return fail(GS_ERR_DEVICE_TIMEOUT, "sort look-back timed out");

    if (stats) {
        stats->sh_eval_ms = 0.0;  // SH is fused into the projection kernel
        stats->project_ms = ms_between(ctx->ev[0], ctx->ev[1]);
        stats->build_tile_ms = ms_between(ctx->ev[2], ctx->ev[3]);
        stats->sort_ms = ms_between(ctx->ev[3], ctx->ev[4]);
        stats->raster_ms = ms_between(ctx->ev[4], ctx->ev[5]);
        stats->total_ms = ms_between(ctx->ev[0], ctx->ev[5]);
        stats->num_keys = K;
        stats->num_tiles = tiles_total;
        // frame kernel, emit, sort histogram + passes, ranges, raster
        // frame kernel + view bases, emit, sort histogram + passes, ranges, raster
        stats->kernel_launches = (n > 0 ? 2 : 0) + (K > 0 ? 3 + passes : 0) + 1;
    }
    return GS_OK;
}

// ---- GS_ORDER_BUCKETS frames -------------------------------------------------

// What the host decides before a tile-bucket frame is enqueued.
struct FramePlan {
    int num_views = 0;
    int64_t n = 0, groups = 0, blocks = 0, items = 0, tiles_total = 0;
    int vpb = 0, deg = 0;
    const HostCopy* host_copy = nullptr;  // non-null: raster per view group, each group's end marked
    const gs_frame_probe* probe = nullptr;  // non-null: the frame kernel also writes the probe outputs
};

// Validates the frame, fills the pinned view parameters and makes the
// per-(view, Gaussian) and per-tile buffers large enough.
int plan_bucket_frame(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int num_views,
                      const gs_render_cfg& cfg, uint8_t* const* outs, FramePlan& p)
{
    if (!valid_cfg(cfg)) return fail(GS_ERR_INVALID, "invalid render cfg");
    if (num_views <= 0) return fail(GS_ERR_INVALID, "no views");
    for (int v = 0; v < num_views; ++v) {
        if (!valid_cam(&cams[v])) return fail(GS_ERR_INVALID, "invalid camera");
        if (!outs[v]) return fail(GS_ERR_INVALID, "null output");
    }
    if (scene->sh_degree == 0 && !scene->color.p) return fail(GS_ERR_INVALID, "scene has no colour");
    GS_CUDA(cudaSetDevice(ctx->device));
    int rc = ensure_ctx_host(ctx, num_views);
    if (rc) return rc;
    p.num_views = num_views;
    p.n = scene->n;
    p.tiles_total = 0;
    for (int v = 0; v < num_views; ++v) {
        ViewParams& vp = ctx->h_views[v];
        make_view_params(cams[v], cfg, vp);
        vp.tile_offset = p.tiles_total;
        vp.out = reinterpret_cast<uchar4*>(outs[v]);
        p.tiles_total += (int64_t)vp.tiles_x * vp.tiles_y;
    }
    if (p.tiles_total >= (1ll << 31)) return fail(GS_ERR_INVALID, "too many tiles");
    p.items = p.n * num_views;
    if (p.items >= (1ll << 31)) return fail(GS_ERR_INVALID, "views x Gaussians exceeds 2^31");
    p.groups = (p.n + 255) / 256;
    p.vpb = std::min(num_views, cfg.views_per_block > 0 ? cfg.views_per_block : 16);
    p.blocks = p.groups * ((num_views + p.vpb - 1) / p.vpb);
    p.deg = scene->sh_degree > 0 ? eval_degree(scene, cfg) : -1;

    if (p.items > ctx->per_view_capacity) {
        const size_t m = (size_t)p.items;
        if (ctx->color.ensure(16 * m) || ctx->xy.ensure(8 * m) || ctx->z.ensure(4 * m) || ctx->ell.ensure(16 * m) ||
            ctx->conic.ensure(16 * m) || ctx->rect.ensure(8 * m) || ctx->offsets.ensure(4 * m) ||
            ctx->rec.ensure(48 * m) || ctx->hitmask.ensure(4 * m)) {
            ctx->per_view_capacity = 0;  // some of them were released: re-check them all next time
            return fail(GS_ERR_OOM, "splat buffers");
        }
        ctx->per_view_capacity = p.items;
    }
    const size_t tiles = (size_t)std::max<int64_t>(p.tiles_total, 1);
    const size_t scan_blocks = (tiles + kTileScanItems - 1) / kTileScanItems;
    if (sizeof(uint64_t) * scan_blocks > ctx->scan_status.bytes) {
        if (ctx->scan_status.ensure(sizeof(uint64_t) * scan_blocks, true)) return fail(GS_ERR_OOM, "scan status");
    }
    if (sizeof(uint32_t) * tiles > ctx->tile_count.bytes) ctx->tile_count_dirty = true;
    if (ctx->ranges.ensure(sizeof(int32_t) * 2 * tiles) || ctx->tile_count.ensure(sizeof(uint32_t) * tiles) ||
        ctx->cursor.ensure(sizeof(unsigned long long) * tiles) || ctx->big_list.ensure(sizeof(int32_t) * 2 * tiles) ||
        ctx->tile_order.ensure(sizeof(int32_t) * tiles))
        return fail(GS_ERR_OOM, "tile buffers");
    return GS_OK;
}

// Enqueues a whole tile-bucket frame on `st` with no host synchronisation
// (everything a replayed graph needs): counters reset, fused projection,
// tile scan, bucket emit, tile sort, raster, counters read-back into
// ctx->h_counters.  The key count stays on the device; a frame whose keys
// exceed ctx->key_capacity comes back with `overflow` set.
int enqueue_bucket_frame(gs_ctx* ctx, const gs_scene* scene, const gs_render_cfg& cfg, const FramePlan& p,
                         cudaStream_t st, bool capturing)
{
    Counters* dc = ctx->counters.as<Counters>();
    GS_CUDA(cudaMemcpyAsync(ctx->views.p, ctx->h_views, sizeof(ViewParams) * p.num_views, cudaMemcpyHostToDevice, st));
    GS_CUDA(cudaMemcpyAsync(dc, ctx->h_init, sizeof(Counters), cudaMemcpyHostToDevice, st));
    // the tile counts are all zero here: cleared when allocated, re-zeroed
    // by every tile scan, and cleared again after a failed frame
    if (ctx->tile_count_dirty) {
        GS_CUDA(cudaMemsetAsync(ctx->tile_count.p, 0, ctx->tile_count.bytes, st));
        if (!capturing) ctx->tile_count_dirty = false;
    }
    GS_CUDA(record(ctx->ev[0], st, capturing));

    FrameArgs fa{};
    fa.n = p.n;
    fa.groups = p.groups;
    fa.num_views = p.num_views;
    fa.views_per_block = p.vpb;
    fa.num_tiles = p.blocks;
    fa.pos = scene->pos.as<float4>();
    fa.orig = scene->orig.as<int32_t>();
    fa.sr = scene->sr.as<float4>();
    fa.sh = scene->sh.as<float>();
    fa.sh_count = scene->sh_count;
    fa.color_in = scene->color.as<float4>();
    fa.views = ctx->views.as<ViewParams>();
    fa.raster_mode = cfg.termination;
    fa.color = ctx->color.as<float4>();
    fa.xy = ctx->xy.as<float2>();
    fa.z = ctx->z.as<float>();
    fa.ell = ctx->ell.as<float4>();
    fa.conic = ctx->conic.as<float4>();
    fa.rect = ctx->rect.as<int2>();
    fa.rec = ctx->rec.as<float4>();
    fa.hitmask = ctx->hitmask.as<uint32_t>();
    fa.offsets = ctx->offsets.as<int32_t>();  // slot -> view * n + i
    fa.err = &dc->err;
    fa.tile_count = ctx->tile_count.as<uint32_t>();
    fa.slot_counter = &dc->slots;
    fa.aggregate = p.tiles_total <= kAggregateMaxTiles;
    if (p.probe) {
        fa.probe_xy = reinterpret_cast<float2*>(p.probe->d_xy);
        fa.probe_z = p.probe->d_z;
        fa.probe_ell = reinterpret_cast<float4*>(p.probe->d_ellipse);
        fa.probe_conic = reinterpret_cast<float4*>(p.probe->d_conic);
        fa.probe_color = reinterpret_cast<float4*>(p.probe->d_color);
    }
    if (p.n > 0) launch_frame_project(fa, p.deg, st, true);

    TileScanArgs ta{};
    ta.count = ctx->tile_count.as<uint32_t>();
    ta.tiles = p.tiles_total;
    ta.cursor = ctx->cursor.as<unsigned long long>();
    ta.ranges = ctx->ranges.as<int32_t>();
    ta.status = ctx->scan_status.as<uint64_t>();
    ta.block_counter = &dc->scan_block;
    ta.epoch_dev = &dc->epoch_scan;
    ta.err = &dc->err;
    ta.total = &dc->total;
    ta.capacity = ctx->key_capacity;
    ta.sort_n = &dc->sort_n;
    ta.overflow = &dc->overflow;
    ta.big_list = ctx->big_list.as<int32_t>();
    ta.big_count = &dc->big_tiles;
    ta.huge_count = &dc->huge_tiles;
    ta.fused_cap = fused_tile_capacity(cfg.tile_w, cfg.tile_h);
    launch_tile_scan(ta, st);
    launch_tile_order(ctx->ranges.as<int32_t>(), p.tiles_total, &dc->total, ctx->tile_order.as<int32_t>(),
                      dc->order_heads, st);
    GS_CUDA(record(ctx->ev[1], st, capturing));
    GS_CUDA(record(ctx->ev[2], st, capturing));

    BucketEmitArgs ea{};
    ea.n = p.n;
    ea.aggregate = p.tiles_total <= kAggregateMaxTiles;
    ea.slot_count = &dc->slots;
    ea.max_slots = p.items;
    ea.views = ctx->views.as<ViewParams>();
    ea.slot_gi = ctx->offsets.as<int32_t>();
    ea.rect = ctx->rect.as<int2>();
    ea.hitmask = ctx->hitmask.as<uint32_t>();
    ea.xy = ctx->xy.as<float2>();
    ea.ell = ctx->ell.as<float4>();
    ea.z = ctx->z.as<float>();
    ea.cursor = ctx->cursor.as<unsigned long long>();
    ea.keys = ctx->keys0.as<uint64_t>();
    ea.capacity = ctx->key_capacity;
    if (p.n > 0) launch_emit_bucket(ea, ctx->num_sms, st);
    GS_CUDA(record(ctx->ev[3], st, capturing));

    TileSortArgs sa{};
    sa.ranges = ctx->ranges.as<int32_t>();
    sa.tiles = p.tiles_total;
    sa.keys = ctx->keys0.as<uint64_t>();
    sa.keys_alt = ctx->keys1.as<uint64_t>();
    sa.vals = ctx->vals0.as<int32_t>();
    sa.vals_alt = ctx->vals1.as<int32_t>();
    sa.slot_gi = ctx->offsets.as<int32_t>();
    sa.big_list = ctx->big_list.as<int32_t>();
    sa.big_count = &dc->big_tiles;
    sa.huge_count = &dc->huge_tiles;
    sa.prefix_bits = cfg.sort_bits;
    if (p.n > 0) launch_tile_sort(sa, ctx->num_sms, st);
    GS_CUDA(record(ctx->ev[4], st, capturing));

    RasterArgs ra{};
    ra.view0 = ctx->h_views[0];
    ra.views = ctx->views.as<ViewParams>();
    ra.num_views = p.num_views;
    ra.write_empty = 1;
    ra.num_tiles_total = p.tiles_total;
    ra.ranges = ctx->ranges.as<int32_t>();
    ra.values = ctx->vals0.as<int32_t>();
    ra.xy = ctx->xy.as<float2>();
    ra.conic = ctx->conic.as<float4>();
    ra.color = ctx->color.as<float4>();
    ra.rec = cfg.termination == GS_TERM_TMIN ? ctx->rec.as<float4>() : nullptr;
    ra.t_min = cfg.t_min;
    ra.tile_counter = &dc->raster_tile;
    ra.keys = ctx->keys0.as<uint64_t>();  // tiles up to the fused capacity are sorted by the raster CTA
    ra.slot_gi = ctx->offsets.as<int32_t>();
    ra.fused_cap = fused_tile_capacity(cfg.tile_w, cfg.tile_h);
    ra.order = ctx->tile_order.as<int32_t>();
    ra.rec_chunk = cfg.raster_chunk;
    ra.rec_persistent = cfg.raster_persistent;
    ra.sort_prefix_bits = cfg.sort_bits;
    if (p.host_copy && p.host_copy->groups > 1 && ra.rec) {
        // one launch per view group, in view order; a group's images are
        // complete at its event
        const HostCopy& hc = *p.host_copy;
        ra.order = nullptr;
        for (int g = 0; g < hc.groups; ++g) {
            const int v0 = hc.first_view[g], v1 = hc.first_view[g + 1];
            const int64_t t0 = ctx->h_views[v0].tile_offset;
            const int64_t t1 = v1 < p.num_views ? ctx->h_views[v1].tile_offset : p.tiles_total;
            RasterArgs rg = ra;
            rg.tile_base = t0;
            rg.num_tiles_total = t1 - t0;
            // a persistent group launch starts its own queue from zero
            if (rg.rec_persistent) GS_CUDA(cudaMemsetAsync(&dc->raster_tile, 0, sizeof(unsigned long long), st));
            launch_raster(rg, cfg.tile_w, cfg.tile_h, cfg.termination, false, ctx->num_sms, st);
            GS_CUDA(record(ctx->ev_group[g], st, capturing));
        }
    } else {
        launch_raster(ra, cfg.tile_w, cfg.tile_h, cfg.termination, p.num_views > 1, ctx->num_sms, st);
    }
    GS_CUDA(cudaGetLastError());
    GS_CUDA(record(ctx->ev[5], st, capturing));
    GS_CUDA(cudaMemcpyAsync(ctx->h_counters, dc, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    return GS_OK;
}

// Signature of every context buffer a captured frame refers to.
uint64_t layout_of(const gs_ctx* ctx)
{
    const DevBuf* bufs[] = {&ctx->views, &ctx->color, &ctx->xy, &ctx->z, &ctx->ell, &ctx->conic, &ctx->rect,
                            &ctx->offsets, &ctx->rec, &ctx->hitmask, &ctx->scan_status, &ctx->keys0, &ctx->vals0,
                            &ctx->keys1, &ctx->vals1, &ctx->ranges, &ctx->tile_count, &ctx->cursor, &ctx->big_list,
                            &ctx->tile_order, &ctx->counters};
    uint64_t h = 1469598103934665603ull;
    auto mix = [&h](uint64_t x) { h = (h ^ x) * 1099511628211ull; };
    for (const DevBuf* b : bufs) {
        mix((uint64_t)(uintptr_t)b->p);
        mix((uint64_t)b->bytes);
    }
    mix((uint64_t)(uintptr_t)ctx->h_views);
    mix((uint64_t)ctx->key_capacity);
    return h;
}

bool same_frame(const FrameGraph& g, const gs_scene* scene, const gs_render_cfg& cfg, const gs_camera* cams,
                int num_views, uint8_t* const* outs)
{
    if (g.scene_uid != scene->uid || (int)g.outs.size() != num_views) return false;
    if (std::memcmp(&g.cfg, &cfg, sizeof(cfg)) != 0) return false;
    for (int v = 0; v < num_views; ++v)
        if (g.outs[v] != outs[v] || g.sizes[2 * v] != cams[v].width || g.sizes[2 * v + 1] != cams[v].height)
            return false;
    return true;
}

void drop_graph(FrameGraph& g)
{
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
}

// Captures the frame enqueued by enqueue_bucket_frame into g.exec.
bool capture_frame(gs_ctx* ctx, const gs_scene* scene, const gs_render_cfg& cfg, const FramePlan& p, FrameGraph& g)
{
    if (!ctx->cap_stream && cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const int rc = enqueue_bucket_frame(ctx, scene, cfg, p, ctx->cap_stream, true);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->cap_stream, &graph);
    bool ok = rc == GS_OK && e == cudaSuccess && graph;
    if (ok) ok = cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        g.exec = nullptr;
        cudaGetLastError();
    }
    g.layout = layout_of(ctx);
    return ok;
}

// One frame with GS_ORDER_BUCKETS.  The key count never goes to the host
// before the frame ends: the lists are used at the capacity they have, and
// a frame that outgrew them is redone once at 1.25x the count it reported.
// With cfg.graph, the second frame with the same scene, options, view sizes
// and outputs is captured into a CUDA graph and later ones replay it.
int run_frame_bucket(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int num_views, const gs_render_cfg& cfg,
                     uint8_t* const* outs, gs_stats* stats, cudaStream_t st, const HostCopy* hc = nullptr,
                     const gs_frame_probe* probe = nullptr)
{
    FramePlan p;
    int rc = plan_bucket_frame(ctx, scene, cams, num_views, cfg, outs, p);
    if (rc) return rc;
    p.host_copy = hc;
    p.probe = probe;
    const int raster_groups = hc ? hc->groups : 0;
    if (!ctx->keys0.p || ctx->key_capacity == 0) {
        rc = ensure_key_buffers(ctx, std::max<int64_t>(p.items, 1 << 20));
        if (rc) return rc;
    }

    // the graph slot of this frame, if any
    FrameGraph* g = nullptr;
    if (cfg.graph) {
        for (FrameGraph& x : ctx->graphs)
            if (same_frame(x, scene, cfg, cams, num_views, outs) && x.raster_groups == raster_groups) g = &x;
        if (!g) {
            if (ctx->graphs.size() >= kMaxGraphs) {
                auto lru = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                            [](const FrameGraph& a, const FrameGraph& b) { return a.last_use < b.last_use; });
                drop_graph(*lru);
                ctx->graphs.erase(lru);
            }
            ctx->graphs.emplace_back();
            g = &ctx->graphs.back();
            g->scene_uid = scene->uid;
            g->cfg = cfg;
            g->raster_groups = raster_groups;
            g->outs.assign(outs, outs + num_views);
            g->sizes.resize(2 * (size_t)num_views);
            for (int v = 0; v < num_views; ++v) {
                g->sizes[2 * v] = cams[v].width;
                g->sizes[2 * v + 1] = cams[v].height;
            }
        } else if (g->exec && g->layout != layout_of(ctx)) {
            drop_graph(*g);  // buffers moved since the capture
        }
        g->last_use = ++ctx->use_clock;
        ++g->seen;
        if (g->split) return kSplitViews;
    }

    int attempts = 0;
    bool replayed = false;
    for (;;) {
        ++attempts;
        ctx->h_init->epoch_scan = take_epochs(ctx->epoch_scan, 1, ctx->scan_status, st);
        ctx->h_init->epoch_sort = 0;
        // the second call with the same key is captured; a redone frame is not
        const bool use_graph = g && !g->failed && g->seen >= 2 && attempts == 1 && !ctx->tile_count_dirty;
        if (use_graph && !g->exec && !capture_frame(ctx, scene, cfg, p, *g)) g->failed = 1;
        if (use_graph && g->exec) {
            GS_CUDA(cudaGraphLaunch(g->exec, st));
            replayed = true;
        } else {
            rc = enqueue_bucket_frame(ctx, scene, cfg, p, st, false);
            if (rc) return rc;
            replayed = false;
        }
        if (hc && hc->groups > 1 && cfg.termination == GS_TERM_TMIN) {
            // each group's images go to the host once its raster is done,
            // while the next group renders (a redone frame copies again)
            for (int gi = 0; gi < hc->groups; ++gi) {
                GS_CUDA(cudaStreamWaitEvent(hc->copy, ctx->ev_group[gi], 0));
                const size_t b0 = hc->first_byte[gi], b1 = hc->first_byte[gi + 1];
                GS_CUDA(cudaMemcpyAsync(hc->h_rgba + b0, outs[hc->first_view[gi]], b1 - b0, cudaMemcpyDeviceToHost,
                                        hc->copy));
            }
        }
        const cudaError_t se = cudaStreamSynchronize(st);
        if (se != cudaSuccess) {
            ctx->tile_count_dirty = true;
            return cuda_fail(se, "frame");
        }
        if (ctx->h_counters->err) {
            ctx->tile_count_dirty = true;
            return fail(GS_ERR_DEVICE_TIMEOUT, "frame look-back timed out");
        }
        const int64_t K = ctx->h_counters->total;
        if (K >= (1ll << 31)) {
            if (g) g->split = 1;
            return fail(kSplitViews, "more than 2^31 tile keys");
        }
        if (!ctx->h_counters->overflow) break;
        if (attempts >= 2) return fail(GS_ERR_CUDA, "tile list overflow after regrowing");
        if (g) drop_graph(*g);
        rc = ensure_key_buffers(ctx, std::min<int64_t>(K + K / 4, (1ll << 31) - 1));
        if (rc) return rc;
    }

    ctx->last_tiles = p.tiles_total;
    ctx->last_keys = ctx->h_counters->total;
    ctx->last_slots = (int64_t)ctx->h_counters->slots;
    ctx->last_fused_cap = fused_tile_capacity(cfg.tile_w, cfg.tile_h);
    if (stats) {
        stats->sh_eval_ms = 0.0;
        stats->project_ms = ms_between(ctx->ev[0], ctx->ev[1]);
        stats->build_tile_ms = ms_between(ctx->ev[2], ctx->ev[3]);
        stats->sort_ms = ms_between(ctx->ev[3], ctx->ev[4]);  // the tiles too big for the raster CTAs
        stats->raster_ms = ms_between(ctx->ev[4], ctx->ev[5]);
        stats->total_ms = ms_between(ctx->ev[0], ctx->ev[5]);
        stats->num_keys = ctx->h_counters->total;
        stats->num_tiles = p.tiles_total;
        // frame kernel, bucket emit, the two big-tile sorts; tile scan, tile order,
        // raster (sorts the other tiles; one launch per view group when the
        // images stream to host memory group by group)
        const bool grouped = p.host_copy && p.host_copy->groups > 1 && cfg.termination == GS_TERM_TMIN;
        stats->kernel_launches = (p.n > 0 ? 4 : 0) + 2 + (grouped ? p.host_copy->groups : 1);
        stats->graph_replay = replayed ? 1 : 0;
        stats->attempts = attempts;
    }
    return GS_OK;
}

int run_frame(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int num_views, const gs_render_cfg& cfg,
              uint8_t* const* outs, gs_stats* stats, cudaStream_t st);

// Views are independent, so a batch renders as frames over parts of its
// views with the same images: halves, as long as the tile lists or the
// (view, Gaussian) items would need 2^31 entries or more.
int run_frame_halves(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int num_views,
                     const gs_render_cfg& cfg, uint8_t* const* outs, gs_stats* stats, cudaStream_t st, int tried)
{
    const int h = num_views / 2;
    gs_stats a{}, b{};
    int rc = run_frame(ctx, scene, cams, h, cfg, outs, &a, st);
    if (rc) return rc;
    rc = run_frame(ctx, scene, cams + h, num_views - h, cfg, outs + h, &b, st);
    if (rc) return rc;
    if (stats) {
        stats->sh_eval_ms = a.sh_eval_ms + b.sh_eval_ms;
        stats->project_ms = a.project_ms + b.project_ms;
        stats->build_tile_ms = a.build_tile_ms + b.build_tile_ms;
        stats->sort_ms = a.sort_ms + b.sort_ms;
        stats->raster_ms = a.raster_ms + b.raster_ms;
        stats->total_ms = a.total_ms + b.total_ms;
        stats->num_keys = a.num_keys + b.num_keys;
        stats->num_tiles = a.num_tiles + b.num_tiles;
        stats->kernel_launches = a.kernel_launches + b.kernel_launches;
        stats->graph_replay = a.graph_replay && b.graph_replay;
        stats->attempts = tried + std::max(a.attempts, b.attempts);
    }
    return GS_OK;
}

int run_frame(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int num_views, const gs_render_cfg& cfg_in,
              uint8_t* const* outs, gs_stats* stats, cudaStream_t st)
{
    gs_render_cfg cfg = cfg_in;
    if (cfg.ordering == GS_ORDER_AUTO) cfg.ordering = GS_ORDER_BUCKETS;  // not tuned: the default ordering
    if (num_views > 1 && scene && scene->n * (int64_t)num_views >= (1ll << 31))
        return run_frame_halves(ctx, scene, cams, num_views, cfg, outs, stats, st, 0);
    int rc;
    if (cfg.ordering == GS_ORDER_ONESWEEP) {
        if (stats) stats->graph_replay = 0, stats->attempts = 1;
        rc = run_frame_onesweep(ctx, scene, cams, num_views, cfg, outs, stats, st);
    } else {
        rc = run_frame_bucket(ctx, scene, cams, num_views, cfg, outs, stats, st);
    }
    if (rc != kSplitViews) return rc;
    if (num_views == 1) return fail(GS_ERR_CAPACITY, "more than 2^31 tile keys in one view");
    return run_frame_halves(ctx, scene, cams, num_views, cfg, outs, stats, st, 1);
}

// floor(log2(x)) for x >= 1, -1 for x <= 0
int32_t floor_log2(int64_t x)
{
    int32_t b = -1;
    for (; x > 0; x >>= 1) ++b;
    return b;
}

int32_t views_bucket(int num_views)
{
    return num_views <= 1 ? 0 : num_views <= 4 ? 1 : num_views <= 8 ? 2 : num_views <= 16 ? 3 : num_views <= 32 ? 4 : 5;
}

TuneEntry tune_key(int64_t n, int64_t pixels, int num_views, const gs_render_cfg& cfg)
{
    TuneEntry e;
    e.n_log2 = floor_log2(n);
    e.px_log2 = floor_log2(pixels);
    e.views_bucket = views_bucket(num_views);
    e.termination = cfg.termination;
    e.ordering = cfg.ordering;
    return e;
}

bool same_bucket(const TuneEntry& a, const TuneEntry& b)
{
    return a.n_log2 == b.n_log2 && a.px_log2 == b.px_log2 && a.views_bucket == b.views_bucket &&
           a.termination == b.termination && a.ordering == b.ordering;
}

// One knob of gs_autotune's coordinate descent: its values, and how a value
// is written into a configuration.
struct TuneKnob {
    std::vector<int> values;
    void (*apply)(gs_render_cfg&, int);
};

// The knobs gs_autotune sweeps for `base` and `num_views`, in sweep order:
// tile shapes only where the images do not depend on them (per-pixel
// termination), views per block only where they change the frame kernel's
// grouping (distinct min(V, vpb)), the ordering only when base asks for
// GS_ORDER_AUTO, the onesweep tile shape for onesweep frames, the tile sort's
// radix width for bucket frames, the record raster's knobs for T_min frames.
// Knobs whose relevance depends on the ordering are listed after it and
// skipped when the ordering picked so far does not use them.
std::vector<TuneKnob> tune_knobs(const gs_render_cfg& base, int num_views)
{
    std::vector<TuneKnob> k;
    if (base.termination == GS_TERM_TMIN)
        k.push_back({{0, 1, 2}, [](gs_render_cfg& c, int v) {
                         static const int shapes[3][2] = {{16, 16}, {16, 8}, {8, 8}};
                         c.tile_w = shapes[v][0];
                         c.tile_h = shapes[v][1];
                     }});
    if (num_views > 8) {
        std::vector<int> vpbs;
        int last = 0;
        for (int v : {8, 16, 32}) {
            const int eff = std::min(num_views, v);
            if (eff != last) vpbs.push_back(v);
            last = eff;
        }
        k.push_back({vpbs, [](gs_render_cfg& c, int v) { c.views_per_block = v; }});
    }
    if (base.ordering == GS_ORDER_AUTO)
        k.push_back({{GS_ORDER_BUCKETS, GS_ORDER_ONESWEEP}, [](gs_render_cfg& c, int v) { c.ordering = v; }});
    k.push_back({{0, 1, 2, 3}, [](gs_render_cfg& c, int v) { c.sort_variant = v; }});
    k.push_back({{8, 16, 24, 32}, [](gs_render_cfg& c, int v) { c.sort_bits = v; }});
    if (base.termination == GS_TERM_TMIN) {
        k.push_back({{32, 64}, [](gs_render_cfg& c, int v) { c.raster_chunk = v; }});
        k.push_back({{0, 1}, [](gs_render_cfg& c, int v) { c.raster_persistent = v; }});
    }
    return k;
}

// Whether a knob (by its setter) matters for the configuration as tuned so far.
bool knob_applies(const TuneKnob& k, const gs_render_cfg& c)
{
    gs_render_cfg a = c, b = c;
    k.apply(a, k.values.front());
    k.apply(b, k.values.back());
    if (a.sort_variant != b.sort_variant) return c.ordering == GS_ORDER_ONESWEEP;
    if (a.sort_bits != b.sort_bits) return c.ordering != GS_ORDER_ONESWEEP;
    return true;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================

extern "C" {

int gs_version(void) { return 100; }

const char* gs_status_string(int status)
{
    switch (status) {
        case GS_OK: return "ok";
        case GS_ERR_INVALID: return "invalid argument";
        case GS_ERR_OOM: return "out of device memory";
        case GS_ERR_CAPACITY: return "buffer capacity exceeded";
        case GS_ERR_DEVICE_TIMEOUT: return "bounded device wait timed out";
        case GS_ERR_CUDA: return "CUDA error";
        case GS_ERR_NO_DEVICE: return "no usable sm_100 device";
        case GS_ERR_CANCELLED: return "request cancelled";
        default: return "unknown status";
    }
}

const char* gs_last_error_string(void) { return g_last_error.c_str(); }

void gs_default_cfg(gs_render_cfg* cfg)
{
    if (!cfg) return;
    cfg->sh_max_degree = 3;
    cfg->termination = GS_TERM_TMIN;
    cfg->t_min = 1e-4f;
    cfg->tile_w = 16;
    cfg->tile_h = 16;
    cfg->ordering = GS_ORDER_BUCKETS;
    cfg->sort_variant = 0;
    cfg->views_per_block = 0;
    cfg->graph = 1;
    cfg->raster_chunk = 0;
    cfg->raster_persistent = 0;
    cfg->sort_bits = 0;
}

void gs_camera_look_at(gs_camera* cam, const float eye[3], const float target[3], const float up[3], float fovy_rad,
                       int32_t width, int32_t height, float znear, float zfar)
{
    if (!cam) return;
    // glm::lookAtRH (ext/matrix_transform.inl:99-119)
    float f[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
    float fl = 1.0f / std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (float& x : f) x *= fl;
    float s[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
    float sl = 1.0f / std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (float& x : s) x *= sl;
    float u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
    float* m = cam->view;
    std::memset(m, 0, sizeof(cam->view));
    m[0] = s[0];  m[4] = s[1];  m[8] = s[2];
    m[1] = u[0];  m[5] = u[1];  m[9] = u[2];
    m[2] = -f[0]; m[6] = -f[1]; m[10] = -f[2];
    m[12] = -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]);
    m[13] = -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]);
    m[14] = (f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2]);
    m[15] = 1.0f;
    cam->position[0] = eye[0];
    cam->position[1] = eye[1];
    cam->position[2] = eye[2];
    cam->width = width;
    cam->height = height;
    cam->aspect = (float)width / (float)height;
    const float coty = 1.0f / std::tan(fovy_rad * 0.5f);
    cam->fov_cotangent[0] = coty / cam->aspect;
    cam->fov_cotangent[1] = coty;
    cam->depth_scale_bias[0] = -2.0f / (zfar - znear);
    cam->depth_scale_bias[1] = -(zfar + znear) / (zfar - znear);
}

int gs_ctx_create(int device, gs_ctx** out)
{
    if (!out) return fail(GS_ERR_INVALID, "out is null");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= device || device < 0) {
        cudaGetLastError();
        return fail(GS_ERR_NO_DEVICE, "no CUDA device");
    }
    cudaDeviceProp prop;
    GS_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10 || prop.minor != 0) return fail(GS_ERR_NO_DEVICE, "device is not sm_100 (B200)");
    GS_CUDA(cudaSetDevice(device));
    gs_ctx* c = new (std::nothrow) gs_ctx();
    if (!c) return fail(GS_ERR_OOM, "host allocation");
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    if (c->counters.ensure(sizeof(Counters), true) != cudaSuccess) {
        delete c;
        return fail(GS_ERR_OOM, "counters");
    }
    if (cudaMallocHost(&c->h_counters, sizeof(Counters)) != cudaSuccess ||
        cudaMallocHost(&c->h_init, sizeof(Counters)) != cudaSuccess) {
        if (c->h_counters) cudaFreeHost(c->h_counters);
        c->counters.release();
        delete c;
        return fail(GS_ERR_OOM, "pinned counters");
    }
    std::memset(c->h_init, 0, sizeof(Counters));
    std::memset(c->h_counters, 0, sizeof(Counters));
    for (auto& ev : c->ev) cudaEventCreate(&ev);
    for (auto& ev : c->ev_group) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    *out = c;
    return GS_OK;
}

int gs_ctx_destroy(gs_ctx* ctx)
{
    if (!ctx) return GS_OK;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    for (FrameGraph& g : ctx->graphs) drop_graph(g);
    ctx->graphs.clear();
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    DevBuf* bufs[] = {&ctx->views, &ctx->color, &ctx->xy, &ctx->z, &ctx->ell, &ctx->conic, &ctx->rect,
                      &ctx->offsets, &ctx->rec, &ctx->hitmask, &ctx->scan_status, &ctx->view_stats, &ctx->keys0, &ctx->vals0, &ctx->keys1, &ctx->vals1,
                      &ctx->sort_hist, &ctx->sort_status, &ctx->ranges, &ctx->tile_count, &ctx->cursor, &ctx->big_list, &ctx->tile_order,
                      &ctx->counters, &ctx->image};
    for (DevBuf* b : bufs) b->release();
    if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
    if (ctx->h_init) cudaFreeHost(ctx->h_init);
    if (ctx->h_views) cudaFreeHost(ctx->h_views);
    for (auto& ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : ctx->ev_group)
        if (ev) cudaEventDestroy(ev);
    delete ctx;
    return GS_OK;
}

int64_t gs_ctx_device_bytes(const gs_ctx* ctx)
{
    if (!ctx) return 0;
    const DevBuf* bufs[] = {&ctx->views, &ctx->color, &ctx->xy, &ctx->z, &ctx->ell, &ctx->conic, &ctx->rect,
                            &ctx->offsets, &ctx->rec, &ctx->hitmask, &ctx->scan_status, &ctx->view_stats, &ctx->keys0, &ctx->vals0, &ctx->keys1, &ctx->vals1,
                            &ctx->sort_hist, &ctx->sort_status, &ctx->ranges, &ctx->tile_count, &ctx->cursor, &ctx->big_list, &ctx->tile_order,
                      &ctx->counters, &ctx->image};
    int64_t t = 0;
    for (const DevBuf* b : bufs) t += (int64_t)b->bytes;
    return t;
}

namespace {

// Uploads the caller's arrays to temporaries, sorts the Gaussians by the
// Morton code of their centres (the onesweep sort, 4 passes over 30 bits)
// and gathers every array into the scene's buffers in that order.
int upload_spatial(gs_ctx* ctx, gs_scene* s, int64_t n, const float* h_position, const float* h_scale_rotation,
                   const float* h_color, const float* h_sh)
{
    const size_t groups = (size_t)((n + 255) / 256);
    const size_t sh_bytes = sizeof(float) * groups * 256 * s->sh_count;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            const float v = h_position[4 * i + k];
            if (std::isfinite(v)) {
                lo[k] = std::min(lo[k], v);
                hi[k] = std::max(hi[k], v);
            }
        }
    for (int k = 0; k < 3; ++k)
        if (!(lo[k] <= hi[k])) lo[k] = hi[k] = 0.0f;
    const int64_t max_tiles = (n + kSortMinTile - 1) / kSortMinTile;
    // one temporary block: source arrays, key/value ping-pong, sort scratch
    size_t off = 0;
    auto take = [&](size_t b) {
        const size_t o = off;
        off += (b + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_pos = take(16 * (size_t)n), o_sr = take(16 * (size_t)n);
    const size_t o_col = h_color ? take(16 * (size_t)n) : 0;
    const size_t o_sh = s->sh_count && h_sh && s->sh.p ? take(sh_bytes) : 0;
    const size_t o_k0 = take(8 * (size_t)n), o_k1 = take(8 * (size_t)n);
    const size_t o_v0 = take(4 * (size_t)n), o_v1 = take(4 * (size_t)n);
    const size_t o_hist = take(sizeof(uint32_t) * kMaxPasses * kRadix);
    const size_t o_status = take(sizeof(uint64_t) * kRadix * (size_t)max_tiles);
    const size_t o_cnt = take(sizeof(unsigned long long) * kMaxPasses);
    const size_t o_err = take(sizeof(int));
    char* t = nullptr;
    cudaError_t e = cudaMalloc(&t, off);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "scene reorder scratch");
    }
    auto P = [&](size_t o) { return (void*)(t + o); };
    e = cudaMemcpy(P(o_pos), h_position, 16 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(P(o_sr), h_scale_rotation, 16 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h_color) e = cudaMemcpy(P(o_col), h_color, 16 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && o_sh) e = cudaMemcpy(P(o_sh), h_sh, sh_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(P(o_status), 0, sizeof(uint64_t) * kRadix * (size_t)max_tiles);
    if (e == cudaSuccess) e = cudaMemset(P(o_err), 0, sizeof(int));
    int passes = 0;
    if (e == cudaSuccess) {
        launch_morton(n, (const float4*)P(o_pos), lo, hi, (uint64_t*)P(o_k0), (int32_t*)P(o_v0), 0);
        SortScratch sc;
        sc.hist = (uint32_t*)P(o_hist);
        sc.status = (uint64_t*)P(o_status);
        sc.counters = (unsigned long long*)P(o_cnt);
        sc.err = (int*)P(o_err);
        sc.max_tiles = max_tiles;
        passes = launch_sort((uint64_t*)P(o_k0), (int32_t*)P(o_v0), (uint64_t*)P(o_k1), (int32_t*)P(o_v1), n, nullptr,
                             30, sc, 1, ctx->num_sms, 0);
        const int32_t* perm = (const int32_t*)P(passes % 2 ? o_v1 : o_v0);
        launch_scene_gather(n, perm, (const float4*)P(o_pos), (const float4*)P(o_sr),
                            h_color ? (const float4*)P(o_col) : nullptr, o_sh ? (const float*)P(o_sh) : nullptr,
                            s->sh_count, s->pos.as<float4>(), s->sr.as<float4>(),
                            h_color ? s->color.as<float4>() : nullptr, s->sh.as<float>(), s->orig.as<int32_t>(), 0);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    int err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&err, P(o_err), sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(t);
    if (e != cudaSuccess) return cuda_fail(e, "scene reorder");
    if (err) return fail(GS_ERR_DEVICE_TIMEOUT, "scene reorder: sort look-back timed out");
    return GS_OK;
}

}  // namespace

int gs_scene_create_ex(gs_ctx* ctx, int64_t n, const float* h_position, const float* h_scale_rotation,
                       const float* h_color, const float* h_sh, int32_t sh_degree, uint32_t flags, gs_scene** out)
{
    if (!ctx || !out || n < 0 || !h_position || !h_scale_rotation) return fail(GS_ERR_INVALID, "null argument");
    if (sh_degree < 0 || sh_degree > 3) return fail(GS_ERR_INVALID, "sh_degree must be 0..3");
    if (sh_degree > 0 && !h_sh) return fail(GS_ERR_INVALID, "SH scene without coefficients");
    if (sh_degree == 0 && !h_color) return fail(GS_ERR_INVALID, "degree-0 scene without colours");
    if (n >= (1ll << 31)) return fail(GS_ERR_INVALID, "too many Gaussians");
    if (flags & ~(uint32_t)GS_SCENE_KEEP_ORDER) return fail(GS_ERR_INVALID, "unknown scene flags");
    *out = nullptr;
    GS_CUDA(cudaSetDevice(ctx->device));
    gs_scene* s = new (std::nothrow) gs_scene();
    if (!s) return fail(GS_ERR_OOM, "host allocation");
    s->uid = g_scene_uid.fetch_add(1);
    s->device = ctx->device;
    s->n = n;
    s->sh_degree = sh_degree;
    s->sh_count = 3 * (sh_degree + 1) * (sh_degree + 1);
    const bool spatial = !(flags & GS_SCENE_KEEP_ORDER) && n >= 2;
    const size_t m = (size_t)std::max<int64_t>(n, 1);
    const size_t groups = (size_t)((n + 255) / 256);
    bool ok = s->pos.ensure(16 * m) == cudaSuccess && s->sr.ensure(16 * m) == cudaSuccess;
    if (ok && h_color) ok = s->color.ensure(16 * m) == cudaSuccess;
    if (ok && sh_degree > 0) ok = s->sh.ensure(sizeof(float) * std::max<size_t>(groups, 1) * 256 * s->sh_count) == cudaSuccess;
    if (ok && spatial) ok = s->orig.ensure(4 * m) == cudaSuccess;
    if (!ok) {
        gs_scene_destroy(s);
        return fail(GS_ERR_OOM, "scene buffers");
    }
    if (spatial) {
        // padding of the last SH group stays zero, as in the caller's layout
        if (sh_degree > 0 && cudaMemset(s->sh.p, 0, s->sh.bytes) != cudaSuccess) {
            gs_scene_destroy(s);
            return cuda_fail(cudaGetLastError(), "scene clear");
        }
        const int rc = upload_spatial(ctx, s, n, h_position, h_scale_rotation, h_color, sh_degree > 0 ? h_sh : nullptr);
        if (rc) {
            gs_scene_destroy(s);
            return rc;
        }
        *out = s;
        return GS_OK;
    }
    cudaError_t e = cudaMemcpy(s->pos.p, h_position, 16 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->sr.p, h_scale_rotation, 16 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h_color) e = cudaMemcpy(s->color.p, h_color, 16 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && sh_degree > 0)
        e = cudaMemcpy(s->sh.p, h_sh, sizeof(float) * groups * 256 * s->sh_count, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        gs_scene_destroy(s);
        return cuda_fail(e, "scene upload");
    }
    *out = s;
    return GS_OK;
}

int gs_scene_create(gs_ctx* ctx, int64_t n, const float* h_position, const float* h_scale_rotation,
                    const float* h_color, const float* h_sh, int32_t sh_degree, gs_scene** out)
{
    return gs_scene_create_ex(ctx, n, h_position, h_scale_rotation, h_color, h_sh, sh_degree, 0u, out);
}

int gs_scene_destroy(gs_scene* s)
{
    if (!s) return GS_OK;
    cudaSetDevice(s->device);
    s->pos.release();
    s->sr.release();
    s->color.release();
    s->sh.release();
    s->orig.release();
    delete s;
    return GS_OK;
}

int64_t gs_scene_size(const gs_scene* s) { return s ? s->n : 0; }

int64_t gs_scene_device_bytes(const gs_scene* s)
{
    return s ? (int64_t)(s->pos.bytes + s->sr.bytes + s->color.bytes + s->sh.bytes + s->orig.bytes) : 0;
}

int gs_render(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cam, const gs_render_cfg* cfg, uint8_t* d_rgba,
              gs_stats* stats, void* stream)
{
    if (!ctx || !scene || !cam || !cfg || !d_rgba) return fail(GS_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    uint8_t* outs[1] = {d_rgba};
    return run_frame(ctx, scene, cam, 1, *cfg, outs, stats, (cudaStream_t)stream);
}

int gs_render_host(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cam, const gs_render_cfg* cfg,
                   uint8_t* h_rgba, gs_stats* stats, void* stream)
{
    if (!ctx || !scene || !cam || !cfg || !h_rgba) return fail(GS_ERR_INVALID, "null argument");
    if (!valid_cam(cam)) return fail(GS_ERR_INVALID, "invalid camera");
    std::lock_guard<std::mutex> lock(ctx->mu);
    GS_CUDA(cudaSetDevice(ctx->device));
    const size_t bytes = 4 * (size_t)cam->width * cam->height;
    if (ctx->image.ensure(bytes)) return fail(GS_ERR_OOM, "image");
    uint8_t* outs[1] = {ctx->image.as<uint8_t>()};
    cudaStream_t st = (cudaStream_t)stream;
    int rc = run_frame(ctx, scene, cam, 1, *cfg, outs, stats, st);
    if (rc) return rc;
    GS_CUDA(cudaMemcpyAsync(h_rgba, ctx->image.p, bytes, cudaMemcpyDeviceToHost, st));
    GS_CUDA(cudaStreamSynchronize(st));
    return GS_OK;
}

int gs_render_batch(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                    const gs_render_cfg* cfg, uint8_t* const* d_rgba, gs_stats* stats, void* stream)
{
    if (!ctx || !scene || !cams || !cfg || !d_rgba || num_views <= 0) return fail(GS_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    return run_frame(ctx, scene, cams, num_views, *cfg, d_rgba, stats, (cudaStream_t)stream);
}

int gs_render_batch_host(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                         const gs_render_cfg* cfg, uint8_t* h_rgba, gs_stats* stats, void* stream)
{
    if (!ctx || !scene || !cams || !cfg || !h_rgba || num_views <= 0) return fail(GS_ERR_INVALID, "null argument");
    for (int v = 0; v < num_views; ++v)
        if (!valid_cam(&cams[v])) return fail(GS_ERR_INVALID, "invalid camera");
    std::lock_guard<std::mutex> lock(ctx->mu);
    GS_CUDA(cudaSetDevice(ctx->device));
    size_t total = 0;
    std::vector<size_t> offs((size_t)num_views);
    for (int v = 0; v < num_views; ++v) {
        offs[v] = total;
        total += 4 * (size_t)cams[v].width * cams[v].height;
    }
    if (ctx->image.ensure(total)) return fail(GS_ERR_OOM, "image");
    std::vector<uint8_t*> outs((size_t)num_views);
    for (int v = 0; v < num_views; ++v) outs[v] = ctx->image.as<uint8_t>() + offs[v];
    cudaStream_t st = (cudaStream_t)stream;
    if (num_views <= kHostChunkViews) {
        int rc = run_frame(ctx, scene, cams, num_views, *cfg, outs.data(), stats, st);
        if (rc) return rc;
        GS_CUDA(cudaMemcpyAsync(h_rgba, ctx->image.p, total, cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        return GS_OK;
    }
    if (!ctx->copy_stream) GS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    if ((cfg->ordering == GS_ORDER_BUCKETS || cfg->ordering == GS_ORDER_AUTO) && cfg->termination == GS_TERM_TMIN) {
        // one frame for all views; its raster runs in view groups, each
        // group read back on the copy stream while the next one renders
        HostCopy hc;
        hc.h_rgba = h_rgba;
        hc.copy = ctx->copy_stream;
        hc.groups = std::min(kMaxRasterGroups, (num_views + kHostGroupViews - 1) / kHostGroupViews);
        // the last group's copy is the one nothing overlaps: a quarter of a
        // group's views, the others share the rest evenly
        const int last = std::max(1, (num_views + hc.groups - 1) / hc.groups / 4);
        const int per = (num_views - last + hc.groups - 2) / (hc.groups - 1);
        for (int g = 0; g < hc.groups; ++g) hc.first_view[g] = std::min(num_views - last, g * per);
        hc.first_view[hc.groups] = num_views;
        for (int g = 0; g <= hc.groups; ++g)
            hc.first_byte[g] = hc.first_view[g] < num_views ? offs[hc.first_view[g]] : total;
        const int rc = run_frame_bucket(ctx, scene, cams, num_views, *cfg, outs.data(), stats, st, &hc);
        const cudaError_t se = cudaStreamSynchronize(ctx->copy_stream);
        if (rc != kSplitViews) {
            if (rc) return rc;
            if (se != cudaSuccess) return cuda_fail(se, "image copy");
            return GS_OK;
        }
        // too many tile keys for one frame: render in chunks below
    }
    // Other frames render in chunks of kHostChunkViews views; each chunk's
    // images are copied to the host on a second stream while the next chunk
    // renders (a frame returns with its stream synchronised, so the chunk is
    // complete when its copy is queued).  The frame kernel reads the scene
    // once per 16 views anyway, so the chunks cost little batching.
    gs_stats acc{};
    acc.graph_replay = 1;
    int rc = GS_OK;
    for (int c0 = 0; c0 < num_views && rc == GS_OK; c0 += kHostChunkViews) {
        const int nv = std::min(kHostChunkViews, num_views - c0);
        gs_stats sc{};
        rc = run_frame(ctx, scene, cams + c0, nv, *cfg, outs.data() + c0, &sc, st);
        if (rc) break;
        const size_t end = c0 + nv < num_views ? offs[c0 + nv] : total;
        const cudaError_t e = cudaMemcpyAsync(h_rgba + offs[c0], outs[c0], end - offs[c0], cudaMemcpyDeviceToHost,
                                              ctx->copy_stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "image copy");
        acc.sh_eval_ms += sc.sh_eval_ms;
        acc.project_ms += sc.project_ms;
        acc.build_tile_ms += sc.build_tile_ms;
        acc.sort_ms += sc.sort_ms;
        acc.raster_ms += sc.raster_ms;
        acc.total_ms += sc.total_ms;
        acc.num_keys += sc.num_keys;
        acc.num_tiles += sc.num_tiles;
        acc.kernel_launches += sc.kernel_launches;
        acc.graph_replay = acc.graph_replay && sc.graph_replay;
        acc.attempts = std::max(acc.attempts, sc.attempts);
    }
    // the copies already queued finish before the call returns, also on an error
    const cudaError_t se = cudaStreamSynchronize(ctx->copy_stream);
    if (rc) return rc;
    if (se != cudaSuccess) return cuda_fail(se, "image copy");
    if (stats) *stats = acc;
    return GS_OK;
}

// ---- stage API ----------------------------------------------------------------

int gs_stage_sh(int64_t n, const float* d_position, const float* d_sh, int32_t sh_count, int32_t eval_degree,
                const gs_camera* cam, float* d_color, void* stream)
{
    if (n < 0 || !cam || (n > 0 && (!d_position || !d_sh || !d_color))) return fail(GS_ERR_INVALID, "null argument");
    if (eval_degree < 0 || eval_degree > 3 || sh_count < 3 * (eval_degree + 1) * (eval_degree + 1))
        return fail(GS_ERR_INVALID, "bad SH degree/count");
    gs_render_cfg cfg;
    gs_default_cfg(&cfg);
    ViewParams v;
    make_view_params(*cam, cfg, v);
    launch_sh_stage(n, (const float4*)d_position, d_sh, sh_count, eval_degree, v, (float4*)d_color,
                    (cudaStream_t)stream);
    GS_CUDA(cudaGetLastError());
    return GS_OK;
}

int gs_stage_project(int64_t n, const float* d_position, const float* d_scale_rotation, const gs_camera* cam,
                     float* d_xy, float* d_z, float* d_ellipse, float* d_conic, void* stream)
{
    if (n < 0 || !valid_cam(cam)) return fail(GS_ERR_INVALID, "bad argument");
    if (n > 0 && (!d_position || !d_scale_rotation || !d_xy || !d_z || !d_ellipse || !d_conic))
        return fail(GS_ERR_INVALID, "null argument");
    gs_render_cfg cfg;
    gs_default_cfg(&cfg);
    ViewParams v;
    make_view_params(*cam, cfg, v);
    launch_project_stage(n, (const float4*)d_position, (const float4*)d_scale_rotation, v, (float2*)d_xy, d_z,
                         (float4*)d_ellipse, (float4*)d_conic, (cudaStream_t)stream);
    GS_CUDA(cudaGetLastError());
    return GS_OK;
}

int gs_stage_build(gs_ctx* ctx, int64_t n, const float* d_xy, const float* d_z, const float* d_ellipse,
                   const gs_camera* cam, const gs_render_cfg* cfg, uint64_t* d_keys, int32_t* d_values,
                   int64_t capacity, int64_t* out_num_keys, void* stream)
{
    if (!ctx || !cfg || !valid_cam(cam) || n < 0 || !out_num_keys) return fail(GS_ERR_INVALID, "bad argument");
    if (!valid_cfg(*cfg)) return fail(GS_ERR_INVALID, "invalid render cfg");
    if (n >= (1ll << 31)) return fail(GS_ERR_INVALID, "too many Gaussians");
    std::lock_guard<std::mutex> lock(ctx->mu);
    GS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    *out_num_keys = 0;
    if (n == 0) return GS_OK;
    int rc = ensure_ctx_host(ctx, 1);
    if (rc) return rc;
    ViewParams& v = ctx->h_views[0];
    make_view_params(*cam, *cfg, v);
    const int64_t blocks = (n + 255) / 256;
    if (ctx->rect.ensure(8 * (size_t)n) || ctx->offsets.ensure(4 * (size_t)n) || ctx->hitmask.ensure(4 * (size_t)n))
        return fail(GS_ERR_OOM, "build buffers");
    ctx->per_view_capacity = 0;  // rect/offsets may have been regrown: force the frame path to re-check
    ctx->last_tiles = -1;        // the last frame's slot indices are overwritten
    if (sizeof(uint64_t) * (size_t)blocks > ctx->scan_status.bytes) {
        if (ctx->scan_status.ensure(sizeof(uint64_t) * (size_t)blocks, true)) return fail(GS_ERR_OOM, "scan status");
    }
    if (ctx->view_stats.ensure(sizeof(int64_t) * 2)) return fail(GS_ERR_OOM, "view stats");
    int64_t* view_total = ctx->view_stats.as<int64_t>();
    int64_t* view_base = view_total + 1;
    Counters* dc = ctx->counters.as<Counters>();
    GS_CUDA(cudaMemcpyAsync(ctx->views.p, &v, sizeof(ViewParams), cudaMemcpyHostToDevice, st));
    GS_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), st));
    FrameArgs fa = {};
    fa.n = n;
    fa.groups = blocks;
    fa.num_views = 1;
    fa.views_per_block = 1;
    fa.epoch = take_epochs(ctx->epoch_scan, 1, ctx->scan_status, st);
    fa.num_tiles = blocks;
    fa.views = ctx->views.as<ViewParams>();
    fa.xy = (float2*)d_xy;
    fa.ell = (float4*)d_ellipse;
    fa.rect = ctx->rect.as<int2>();
    fa.hitmask = ctx->hitmask.as<uint32_t>();
    fa.offsets = ctx->offsets.as<int32_t>();
    fa.status = ctx->scan_status.as<uint64_t>();
    fa.tile_counter = &dc->frame_tile;
    fa.view_total = view_total;
    fa.err = &dc->err;
    launch_count_stage(fa, st);
    launch_view_base(view_total, 1, view_base, &dc->total, st);
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaMemcpyAsync(ctx->h_counters, dc, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    GS_CUDA(cudaStreamSynchronize(st));
    if (ctx->h_counters->err) return fail(GS_ERR_DEVICE_TIMEOUT, "build look-back timed out");
    const int64_t K = ctx->h_counters->total;
    *out_num_keys = K;
    if (K > 0 && (!d_keys || !d_values)) return fail(GS_ERR_INVALID, "null key buffers");
    if (capacity < 0) capacity = 0;
    EmitArgs ea{};
    ea.n = n;
    ea.num_views = 1;
    ea.views = ctx->views.as<ViewParams>();
    ea.offsets = ctx->offsets.as<int32_t>();
    ea.view_total = view_total;
    ea.view_base = view_base;
    ea.rect = ctx->rect.as<int2>();
    ea.hitmask = ctx->hitmask.as<uint32_t>();
    ea.xy = (const float2*)d_xy;
    ea.ell = (const float4*)d_ellipse;
    ea.z = d_z;
    ea.keys = d_keys;
    ea.values = d_values;
    ea.capacity = capacity;
    if (K > 0 && capacity > 0) launch_emit(ea, st);
    GS_CUDA(cudaGetLastError());
    // the reference truncates a list that does not fit and reports it full
    // (gaussian_render.cu:506-509); here the first `capacity` keys in
    // Gaussian order are written and the caller learns the exact count
    if (K > capacity) return fail(GS_ERR_CAPACITY, "tile list capacity exceeded: the first `capacity` keys were written");
    return GS_OK;
}

int gs_stage_sort(gs_ctx* ctx, int64_t num_keys, int32_t key_bits, uint64_t* d_keys, int32_t* d_values,
                  uint64_t* d_keys_alt, int32_t* d_values_alt, int32_t* out_selector, void* stream)
{
    if (!ctx || !out_selector || num_keys < 0 || key_bits < 1 || key_bits > 64) return fail(GS_ERR_INVALID, "bad argument");
    if (num_keys >= (1ll << 31)) return fail(GS_ERR_INVALID, "too many keys");
    *out_selector = 0;
    if (num_keys == 0) return GS_OK;
    if (!d_keys || !d_values || !d_keys_alt || !d_values_alt) return fail(GS_ERR_INVALID, "null buffer");
    std::lock_guard<std::mutex> lock(ctx->mu);
    GS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_sort_scratch(ctx, num_keys);
    if (rc) return rc;
    Counters* dc = ctx->counters.as<Counters>();
    GS_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), st));
    SortScratch ss;
    ss.hist = ctx->sort_hist.as<uint32_t>();
    ss.status = ctx->sort_status.as<uint64_t>();
    ss.counters = dc->sort_tiles;
    ss.err = &dc->err;
    ss.max_tiles = (int64_t)(ctx->sort_status.bytes / (8 * kRadix));
    const uint32_t ep = take_epochs(ctx->epoch_sort, (uint32_t)sort_passes(key_bits), ctx->sort_status, st);
    const int passes =
        launch_sort(d_keys, d_values, d_keys_alt, d_values_alt, num_keys, nullptr, key_bits, ss, ep, ctx->num_sms, st,
                    stage_sort_variant(num_keys));
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaMemcpyAsync(&ctx->h_counters->err, &dc->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    GS_CUDA(cudaStreamSynchronize(st));
    if (ctx->h_counters->err) return fail(GS_ERR_DEVICE_TIMEOUT, "sort look-back timed out");
    *out_selector = passes % 2;
    return GS_OK;
}

int gs_probe_sort_timed(gs_ctx* ctx, int64_t num_keys, int32_t key_bits, const uint64_t* d_src_keys,
                        const int32_t* d_src_values, uint64_t* d_keys, int32_t* d_values, uint64_t* d_keys_alt,
                        int32_t* d_values_alt, int32_t iterations, int32_t* out_selector, double* out_median_ms)
{
    if (!ctx || !out_selector || !out_median_ms || num_keys <= 0 || key_bits < 1 || key_bits > 64 || iterations < 1)
        return fail(GS_ERR_INVALID, "bad argument");
    if (num_keys >= (1ll << 31)) return fail(GS_ERR_INVALID, "too many keys");
    if (!d_src_keys || !d_src_values || !d_keys || !d_values || !d_keys_alt || !d_values_alt)
        return fail(GS_ERR_INVALID, "null buffer");
    std::lock_guard<std::mutex> lock(ctx->mu);
    GS_CUDA(cudaSetDevice(ctx->device));
    const cudaStream_t st = nullptr;
    int rc = ensure_sort_scratch(ctx, num_keys);
    if (rc) return rc;
    Counters* dc = ctx->counters.as<Counters>();
    std::vector<double> ms;
    int passes = 0;
    for (int it = 0; it < iterations; ++it) {
        // restore the unsorted input and clear the error flag, outside the
        // timed region
        GS_CUDA(cudaMemcpyAsync(d_keys, d_src_keys, sizeof(uint64_t) * (size_t)num_keys, cudaMemcpyDeviceToDevice, st));
        GS_CUDA(cudaMemcpyAsync(d_values, d_src_values, sizeof(int32_t) * (size_t)num_keys, cudaMemcpyDeviceToDevice,
                                st));
        GS_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), st));
        SortScratch ss;
        ss.hist = ctx->sort_hist.as<uint32_t>();
        ss.status = ctx->sort_status.as<uint64_t>();
        ss.counters = dc->sort_tiles;
        ss.err = &dc->err;
        ss.max_tiles = (int64_t)(ctx->sort_status.bytes / (8 * kRadix));
        const uint32_t ep = take_epochs(ctx->epoch_sort, (uint32_t)sort_passes(key_bits), ctx->sort_status, st);
        GS_CUDA(cudaEventRecord(ctx->ev[6], st));
        passes = launch_sort(d_keys, d_values, d_keys_alt, d_values_alt, num_keys, nullptr, key_bits, ss, ep,
                             ctx->num_sms, st, stage_sort_variant(num_keys));
        GS_CUDA(cudaGetLastError());
        GS_CUDA(cudaEventRecord(ctx->ev[7], st));
        GS_CUDA(cudaMemcpyAsync(&ctx->h_counters->err, &dc->err, sizeof(int), cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        if (ctx->h_counters->err) return fail(GS_ERR_DEVICE_TIMEOUT, "sort look-back timed out");
        ms.push_back(ms_between(ctx->ev[6], ctx->ev[7]));
    }
    std::sort(ms.begin(), ms.end());
    *out_median_ms = ms[ms.size() / 2];
    *out_selector = passes % 2;
    return GS_OK;
}

int gs_stage_ranges(int64_t num_keys, const uint64_t* d_keys, int64_t num_tiles, int32_t* d_ranges, void* stream)
{
    if (num_keys < 0 || num_tiles <= 0 || !d_ranges || (num_keys > 0 && !d_keys)) return fail(GS_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    GS_CUDA(cudaMemsetAsync(d_ranges, 0xFF, sizeof(int32_t) * 2 * (size_t)num_tiles, st));
    if (num_keys > 0) launch_ranges(d_keys, num_keys, nullptr, d_ranges, st);
    GS_CUDA(cudaGetLastError());
    return GS_OK;
}

int gs_stage_raster(const gs_camera* cam, const gs_render_cfg* cfg, const int32_t* d_ranges, const int32_t* d_values,
                    const float* d_xy, const float* d_conic, const float* d_color, uint8_t* d_rgba, void* stream)
{
    if (!valid_cam(cam) || !cfg || !d_ranges || !d_rgba) return fail(GS_ERR_INVALID, "bad argument");
    if (!valid_cfg(*cfg)) return fail(GS_ERR_INVALID, "invalid render cfg");
    // entries are staged with 8- and 16-byte asynchronous copies
    if (((uintptr_t)d_xy & 7) || ((uintptr_t)d_conic & 15) || ((uintptr_t)d_color & 15))
        return fail(GS_ERR_INVALID, "xy must be 8-byte and conic/color 16-byte aligned");
    RasterArgs ra = {};
    make_view_params(*cam, *cfg, ra.view0);
    ra.view0.out = reinterpret_cast<uchar4*>(d_rgba);
    ra.views = nullptr;
    ra.num_views = 1;
    ra.write_empty = 0;
    ra.num_tiles_total = (int64_t)ra.view0.tiles_x * ra.view0.tiles_y;
    ra.ranges = d_ranges;
    ra.values = d_values;
    ra.xy = (const float2*)d_xy;
    ra.conic = (const float4*)d_conic;
    ra.color = (const float4*)d_color;
    ra.t_min = cfg->t_min;
    launch_raster(ra, cfg->tile_w, cfg->tile_h, cfg->termination, false, device_sm_count(), (cudaStream_t)stream);
    GS_CUDA(cudaGetLastError());
    return GS_OK;
}

int gs_autotune(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                const gs_render_cfg* base, int32_t iterations, gs_render_cfg* best, double* best_ms,
                gs_tune_result* results, int32_t results_capacity, int32_t* num_results, void* stream)
{
    if (!ctx || !scene || !cams || !base || !best || num_views <= 0) return fail(GS_ERR_INVALID, "null argument");
    if (iterations < 1 || (results_capacity > 0 && !results)) return fail(GS_ERR_INVALID, "bad tuning arguments");
    if (!valid_cfg(*base)) return fail(GS_ERR_INVALID, "invalid render cfg");
    int64_t total = 0, pixels = 0;
    std::vector<size_t> offs((size_t)num_views);
    for (int v = 0; v < num_views; ++v) {
        if (!valid_cam(&cams[v])) return fail(GS_ERR_INVALID, "invalid camera");
        offs[v] = (size_t)total;
        total += 4 * (int64_t)cams[v].width * cams[v].height;
        pixels = std::max<int64_t>(pixels, (int64_t)cams[v].width * cams[v].height);
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    GS_CUDA(cudaSetDevice(ctx->device));
    if (ctx->image.ensure((size_t)total)) return fail(GS_ERR_OOM, "image");
    std::vector<uint8_t*> outs((size_t)num_views);
    for (int v = 0; v < num_views; ++v) outs[v] = ctx->image.as<uint8_t>() + offs[v];
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GS_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(cudaGetLastError(), "tuning events");
    }

    // coordinate descent: each knob at all its values, the others at the
    // best so far; a candidate already timed is not timed again
    std::vector<gs_render_cfg> timed_cfgs;
    std::vector<double> timed_ms;
    auto time_cfg = [&](const gs_render_cfg& c, double& ms) -> int {
        for (size_t i = 0; i < timed_cfgs.size(); ++i)
            if (std::memcmp(&timed_cfgs[i], &c, sizeof(c)) == 0) {
                ms = timed_ms[i];
                return GS_OK;
            }
        int r = GS_OK;
        for (int w = 0; w < 2 && r == GS_OK; ++w) r = run_frame(ctx, scene, cams, num_views, c, outs.data(), nullptr, st);
        std::vector<float> times((size_t)iterations);
        for (int it = 0; it < iterations && r == GS_OK; ++it) {
            cudaEventRecord(e0, st);
            r = run_frame(ctx, scene, cams, num_views, c, outs.data(), nullptr, st);
            cudaEventRecord(e1, st);
            if (r == GS_OK && cudaEventSynchronize(e1) != cudaSuccess) r = cuda_fail(cudaGetLastError(), "tuning");
            times[it] = ms_between(e0, e1);
        }
        if (r != GS_OK) return r;
        std::sort(times.begin(), times.end());
        ms = times[(size_t)iterations / 2];
        timed_cfgs.push_back(c);
        timed_ms.push_back(ms);
        return GS_OK;
    };
    gs_render_cfg cur = *base;
    // defaults spelled out, so a default and its explicit value are one candidate
    if (cur.ordering == GS_ORDER_AUTO) cur.ordering = GS_ORDER_BUCKETS;
    if (cur.raster_chunk == 0) cur.raster_chunk = 32;
    if (cur.sort_bits == 0) cur.sort_bits = 16;
    int rc = GS_OK;
    bool have = false;
    double win_ms = 0.0;
    for (const TuneKnob& k : tune_knobs(*base, num_views)) {
        if (rc != GS_OK) break;
        if (!knob_applies(k, cur)) continue;
        gs_render_cfg knob_best = cur;
        for (int v : k.values) {
            gs_render_cfg c = cur;
            k.apply(c, v);
            double ms = 0.0;
            const int r = time_cfg(c, ms);
            if (r == GS_OK) {
                if (!have || ms < win_ms) {
                    win_ms = ms;
                    knob_best = c;
                    have = true;
                }
            } else if (r == GS_ERR_OOM || r == GS_ERR_CAPACITY) {
                cudaGetLastError();  // this setting does not fit: the others may
            } else {
                rc = r;
                break;
            }
        }
        cur = knob_best;
    }
    if (!have && rc == GS_OK) {
        // no knob applies (a single-view reference frame): time the base alone
        double ms = 0.0;
        rc = time_cfg(cur, ms);
        if (rc == GS_OK) {
            win_ms = ms;
            have = true;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int timed = (int)timed_cfgs.size();
    for (int i = 0; i < timed && i < results_capacity; ++i) results[i] = gs_tune_result{timed_cfgs[i], timed_ms[i]};
    if (num_results) *num_results = timed;
    if (rc) return rc;
    if (!have) return fail(GS_ERR_OOM, "no knob setting fit in device memory");

    TuneEntry e = tune_key(scene->n, pixels, num_views, *base);
    e.tile_w = cur.tile_w;
    e.tile_h = cur.tile_h;
    e.views_per_block = cur.views_per_block;
    e.sort_variant = cur.sort_variant;
    e.ordering_picked = cur.ordering;
    e.raster_chunk = cur.raster_chunk;
    e.raster_persistent = cur.raster_persistent;
    e.sort_bits = cur.sort_bits;
    e.ms = win_ms;
    e.stamp = ++ctx->tune_clock;
    auto it = std::find_if(ctx->tune.begin(), ctx->tune.end(), [&](const TuneEntry& x) { return same_bucket(x, e); });
    if (it != ctx->tune.end()) {
        *it = e;
    } else {
        if (ctx->tune.size() >= kMaxTuneEntries)
            ctx->tune.erase(std::min_element(ctx->tune.begin(), ctx->tune.end(),
                                             [](const TuneEntry& a, const TuneEntry& b) { return a.stamp < b.stamp; }));
        ctx->tune.push_back(e);
    }
    *best = cur;
    if (best_ms) *best_ms = win_ms;
    return GS_OK;
}

int gs_autotune_lookup(gs_ctx* ctx, int64_t n, int32_t width, int32_t height, int32_t num_views, gs_render_cfg* cfg,
                       int32_t* found)
{
    if (!ctx || !cfg || !found) return fail(GS_ERR_INVALID, "null argument");
    if (n < 0 || width <= 0 || height <= 0 || num_views <= 0) return fail(GS_ERR_INVALID, "bad bucket");
    std::lock_guard<std::mutex> lock(ctx->mu);
    const TuneEntry k = tune_key(n, (int64_t)width * height, num_views, *cfg);
    *found = 0;
    for (const TuneEntry& e : ctx->tune)
        if (same_bucket(e, k)) {
            cfg->tile_w = e.tile_w;
            cfg->tile_h = e.tile_h;
            cfg->views_per_block = e.views_per_block;
            cfg->sort_variant = e.sort_variant;
            cfg->ordering = e.ordering_picked;
            cfg->raster_chunk = e.raster_chunk;
            cfg->raster_persistent = e.raster_persistent;
            cfg->sort_bits = e.sort_bits;
            *found = 1;
            break;
        }
    return GS_OK;
}

int gs_autotune_bucket(int64_t n, int32_t width, int32_t height, int32_t num_views, int32_t bucket[3])
{
    if (!bucket || n < 0 || width <= 0 || height <= 0 || num_views <= 0) return fail(GS_ERR_INVALID, "bad bucket");
    bucket[0] = floor_log2(n);
    bucket[1] = floor_log2((int64_t)width * height);
    bucket[2] = views_bucket(num_views);
    return GS_OK;
}

int32_t gs_autotune_entries(gs_ctx* ctx)
{
    if (!ctx) return 0;
    std::lock_guard<std::mutex> lock(ctx->mu);
    return (int32_t)ctx->tune.size();
}

int64_t gs_num_tiles(int32_t width, int32_t height, const gs_render_cfg* cfg)
{
    if (!cfg || width <= 0 || height <= 0 || cfg->tile_w <= 0 || cfg->tile_h <= 0) return 0;
    return (int64_t)((width + cfg->tile_w - 1) / cfg->tile_w) * ((height + cfg->tile_h - 1) / cfg->tile_h);
}

int32_t gs_key_bits(int64_t num_tiles)
{
    int32_t bits = 0;
    while (bits < 31 && (1ll << bits) < num_tiles) ++bits;
    return 32 + bits;
}

// ---- failure-path test hooks ------------------------------------------------------

void gs_test_fail_allocations(int32_t skip, int32_t count)
{
    std::lock_guard<std::mutex> lk(g_alloc_hook_mu);
    g_alloc_skip = skip > 0 ? skip : 0;
    g_fail_allocs = count > 0 ? count : 0;
    g_alloc_hook = g_fail_allocs > 0;
}

int32_t gs_test_pending_allocation_failures(void)
{
    std::lock_guard<std::mutex> lk(g_alloc_hook_mu);
    return g_alloc_hook ? g_fail_allocs : 0;
}

int gs_test_bounded_wait(int32_t spin_limit, void* stream)
{
    if (spin_limit < 1 || spin_limit > kSpinLimit) return fail(GS_ERR_INVALID, "spin limit out of range");
    cudaStream_t st = (cudaStream_t)stream;
    WaitWords* w = nullptr;
    GS_CUDA(cudaMalloc(&w, sizeof(WaitWords)));
    int err = 0;
    cudaError_t e = cudaMemsetAsync(w, 0, sizeof(WaitWords), st);
    if (e == cudaSuccess) {
        wait_selftest_kernel<<<1, 32, 0, st>>>(w, spin_limit);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, &w->err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(w);
    if (e != cudaSuccess) return cuda_fail(e, "bounded wait");
    if (err == kErrTimeout) return fail(GS_ERR_DEVICE_TIMEOUT, "the bounded wait gave up, as it must");
    return fail(GS_ERR_CUDA, "the bounded wait did not report its timeout");
}

// ---- frame probe ------------------------------------------------------------------

int gs_probe_frame(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                   const gs_render_cfg* cfg, uint8_t* const* d_rgba, const gs_frame_probe* probe, gs_stats* stats,
                   void* stream)
{
    if (!ctx || !scene || !cams || !cfg || !d_rgba || !probe || num_views <= 0) return fail(GS_ERR_INVALID, "null argument");
    if (!probe->d_xy || !probe->d_z || !probe->d_ellipse || !probe->d_conic)
        return fail(GS_ERR_INVALID, "probe geometry outputs are required");
    if (cfg->ordering == GS_ORDER_ONESWEEP) return fail(GS_ERR_INVALID, "the probe covers GS_ORDER_BUCKETS frames");
    std::lock_guard<std::mutex> lock(ctx->mu);
    gs_render_cfg c = *cfg;
    c.graph = 0;  // the probe outputs are arguments of this launch only
    ctx->last_tiles = -1;
    const int rc = run_frame_bucket(ctx, scene, cams, num_views, c, d_rgba, stats, (cudaStream_t)stream, nullptr, probe);
    if (rc == kSplitViews) return fail(GS_ERR_CAPACITY, "the probe frame needs 2^31 tile keys or more");
    return rc;
}

int gs_probe_tile_lists(gs_ctx* ctx, int32_t* h_ranges, int64_t ranges_capacity, uint64_t* h_keys, int32_t* h_order,
                        int64_t keys_capacity, int32_t* h_slot_index, int64_t slots_capacity, int64_t out_sizes[3],
                        int32_t* out_fused_cap)
{
    if (!ctx || !out_sizes) return fail(GS_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (ctx->last_tiles < 0) return fail(GS_ERR_INVALID, "no tile-bucket frame since the lists last changed");
    out_sizes[0] = ctx->last_tiles;
    out_sizes[1] = ctx->last_keys;
    out_sizes[2] = ctx->last_slots;
    if (out_fused_cap) *out_fused_cap = ctx->last_fused_cap;
    GS_CUDA(cudaSetDevice(ctx->device));
    if (h_ranges) {
        if (ranges_capacity < 2 * ctx->last_tiles) return fail(GS_ERR_CAPACITY, "ranges buffer too small");
        GS_CUDA(cudaMemcpy(h_ranges, ctx->ranges.p, sizeof(int32_t) * 2 * (size_t)ctx->last_tiles,
                           cudaMemcpyDeviceToHost));
    }
    if (h_keys || h_order) {
        if (keys_capacity < ctx->last_keys) return fail(GS_ERR_CAPACITY, "key buffers too small");
        if (h_keys)
            GS_CUDA(cudaMemcpy(h_keys, ctx->keys0.p, sizeof(uint64_t) * (size_t)ctx->last_keys, cudaMemcpyDeviceToHost));
        if (h_order)
            GS_CUDA(cudaMemcpy(h_order, ctx->vals0.p, sizeof(int32_t) * (size_t)ctx->last_keys, cudaMemcpyDeviceToHost));
    }
    if (h_slot_index) {
        if (slots_capacity < ctx->last_slots) return fail(GS_ERR_CAPACITY, "slot buffer too small");
        GS_CUDA(cudaMemcpy(h_slot_index, ctx->offsets.p, sizeof(int32_t) * (size_t)ctx->last_slots,
                           cudaMemcpyDeviceToHost));
    }
    return GS_OK;
}

}  // extern "C"
