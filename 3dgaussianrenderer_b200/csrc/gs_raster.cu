// Tile rasteriser (replaces rasterizeTilesKernel, core/gaussian_render.cu:679-775).
//
// One CTA per tile, one thread per pixel; each warp owns an 8x4 block of
// the tile.  The tile's depth-sorted entries are staged in shared memory
// (centre, conic + opacity, colour) and the pixels blend them front to back
// in FP32 with the reference's arithmetic.
//
// Termination:
//  * GS_TERM_REFERENCE: every pixel evaluates every entry; after every 32nd
//    entry of the tile's list the CTA stops once no in-image pixel has
//    T > 0.02 (the reference's test at :745).  Batches of 32 entries,
//    double-buffered so the gather of the next batch overlaps the blending
//    of this one.  Bit-identical to the reference kernel.  (The GS_TERM_TMIN
//    variant of this kernel stages one entry per thread.)
//  * GS_TERM_TMIN: a pixel stops once its T < t_min; a warp whose pixels are
//    all done skips the rest (warp ballot), the CTA stops when every pixel
//    is done.  Each warp first tests 32 staged splats at a time against its
//    8x4 pixel block (one splat per lane) and blends only the survivors
//    (ballot compaction).  A splat survives when its cutoff ellipse, where
//    opacity * exp(-q/2) = kCullAlpha, touches the block; the contributions
//    skipped are each below kCullAlpha (2^-18), so a pixel needs more than a
//    thousand of them to move by 1/255.
//
// The plain path launches one CTA per tile; the batched path runs a
// persistent grid that pulls global tile ids (all views' tiles, flattened)
// from an atomic queue.
#include "gs_kernels.h"
#include "gs_tilesort.cuh"
#include "gs_f32x2.cuh"

#include <algorithm>

namespace gs {

struct RasterSmem {
    float2* xy;
    float4* con;  // (a, b, c, opacity)
    float4* col;
    float4* box;  // cutoff box (x0, x1, y0, y1), GS_TERM_TMIN only
};

__device__ __forceinline__ void blend(const float cx, const float cy, const float2 c, const float4 k, const float4 col,
                                      float& r, float& g, float& b, float& T)
{
    const float dx = cx - c.x, dy = cy - c.y;
    const float q = k.x * dx * dx + k.z * dy * dy + 2.0f * k.y * dx * dy;
    const float density = __expf(-0.5f * q);
    const float alpha = k.w * __saturatef(density);
    r += col.x * T * alpha;
    g += col.y * T * alpha;
    b += col.z * T * alpha;
    T *= (1.0f - alpha);
}

__device__ __forceinline__ void cp_async(void* dst, const void* src, const int bytes_is_16)
{
    if (bytes_is_16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copies entry `s` (centre, conic, colour) into shared-memory slot `slot`.
__device__ __forceinline__ void stage_entry(const RasterArgs& a, const int s, const struct RasterSmem& sm,
                                            const int slot)
{
    cp_async(&sm.xy[slot], &a.xy[s], 0);
    cp_async(&sm.con[slot], &a.conic[s], 1);
    cp_async(&sm.col[slot], &a.color[s], 1);
}

template <int TW, int TH, int MODE>
__device__ __forceinline__ void raster_tile(const RasterArgs& a, const ViewParams& v, const int64_t gtile,
                                            const int local_tile, const RasterSmem& sm)
{
    constexpr int NT = TW * TH;
    constexpr int WX = TW / 8;  // warps per tile row
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int first = __ldg(&a.ranges[2 * gtile]);
    const int last = __ldg(&a.ranges[2 * gtile + 1]);
    const int count = last - first;
    const int tx = local_tile % v.tiles_x, ty = local_tile / v.tiles_x;
    const int wx0 = tx * TW + (warp % WX) * 8, wy0 = ty * TH + (warp / WX) * 4;
    const int px = wx0 + (lane & 7);
    const int py = wy0 + (lane >> 3);
    const bool inimg = px < v.width && py < v.height;
    if (count <= 0) {
        // the reference clears the image and skips empty tiles (main.cpp:363);
        // writing zeros here instead saves the separate clear
        if (a.write_empty && inimg) v.out[(int64_t)py * v.width + px] = make_uchar4(0, 0, 0, 0);
        return;
    }
    // pixel corner sample, gaussian_render.cu:701-704
    const float cx = (float)px * v.texel_x - 1.0f;
    const float cy = (float)py * v.texel_y - 1.0f;
    // this warp's 8x4 block in clip space
    const float bx0 = (float)wx0 * v.texel_x - 1.0f, bx1 = (float)(wx0 + 7) * v.texel_x - 1.0f;
    const float by0 = (float)wy0 * v.texel_y - 1.0f, by1 = (float)(wy0 + 3) * v.texel_y - 1.0f;

    float r = 0.0f, g = 0.0f, b = 0.0f;
    float T = 1.0f;
    bool done = !inimg;

    for (int base = 0; MODE == 1 && base < count; base += NT) {
        const int nb = min(NT, count - base);
        __syncthreads();
        if ((int)threadIdx.x < nb) {
            const int s = __ldg(&a.values[first + base + threadIdx.x]);
            const float4 col = __ldg(&a.color[s]);
            const float4 con = __ldg(&a.conic[s]);
            const float2 c = __ldg(&a.xy[s]);
            sm.xy[threadIdx.x] = c;
            sm.con[threadIdx.x] = make_float4(con.x, con.y, con.z, col.w);
            sm.col[threadIdx.x] = col;
            {
                float4 box;
                const float det = con.x * con.z - con.y * con.y;
                if (!(col.w > kCullAlpha)) {
                    box = make_float4(1e30f, -1e30f, 1e30f, -1e30f);  // contributes nothing
                } else if (!(det > 0.0f) || !(con.x > 0.0f) || !(con.z > 0.0f)) {
                    box = make_float4(-1e30f, 1e30f, -1e30f, 1e30f);  // degenerate: never cull
                } else {
                    const float qc = 2.0f * logf(col.w / kCullAlpha);
                    const float ex = sqrtf(qc * con.z / det), ey = sqrtf(qc * con.x / det);
                    box = make_float4(c.x - ex, c.x + ex, c.y - ey, c.y + ey);
                }
                sm.box[threadIdx.x] = box;
            }
        }
        __syncthreads();
        {
            for (int c0 = 0; c0 < nb; c0 += 32) {
                if (__all_sync(kFull, done)) break;
                const int j = c0 + lane;
                bool keep = false;
                if (j < nb) {
                    const float4 bx = sm.box[j];
                    keep = bx.x <= bx1 && bx.y >= bx0 && bx.z <= by1 && bx.w >= by0;
                }
                unsigned m = __ballot_sync(kFull, keep);
                while (m) {
                    const int k = c0 + __ffs(m) - 1;
                    m &= m - 1;
                    if (!done) {
                        blend(cx, cy, sm.xy[k], sm.con[k], sm.col[k], r, g, b, T);
                        if (T < a.t_min) done = true;
                    }
                }
            }
            if (__syncthreads_count(!done) == 0) break;
        }
    }

    if (inimg) {
        uchar4 qc;
        qc.x = r * 255;
        qc.y = g * 255;
        qc.z = b * 255;
        qc.w = 255;
        v.out[(int64_t)py * v.width + px] = qc;
    }
}

__device__ __forceinline__ void store_pixel(const ViewParams& v, const int px, const int py, const float r,
                                            const float g, const float b)
{
    uchar4 qc;
    qc.x = r * 255;
    qc.y = g * 255;
    qc.z = b * 255;
    qc.w = 255;
    v.out[(int64_t)py * v.width + px] = qc;
}

// ---- per-tile sort inside the raster CTA ----------------------------------------
//
// In tile-bucket frames a tile of at most fused_cap keys arrives unsorted;
// its CTA orders it in shared memory (gs_tilesort.cuh) before blending and
// reads the slots from there.  Larger tiles were sorted ahead of the raster
// and are read from `values`.

template <int NT>
struct FusedSortSmem {
    uint64_t k[NT * kFusedIpt];
    int32_t v[NT * kFusedIpt];
    int32_t bexcl[256];
    int32_t dcount[256];
    int32_t scan[NT / 32];
    uint64_t red[2 * (NT / 32)];
};

// Returns the tile's sorted keys in shared memory, or null when the order
// is in a.values.  Every thread of the CTA must call it.
template <int NT>
__device__ __forceinline__ const uint64_t* fused_sort(const RasterArgs& a, const int first, const int count,
                                                      FusedSortSmem<NT>& fs)
{
    if (!a.keys || count > a.fused_cap) return nullptr;
    if (count == 1) {
        if (threadIdx.x == 0) fs.k[0] = a.keys[first];
        __syncthreads();
        return fs.k;
    }
    tilesort::Smem sm;
    sm.k = fs.k;
    sm.v = fs.v;
    sm.whist = reinterpret_cast<uint32_t*>(fs.k);
    sm.bexcl = fs.bexcl;
    sm.dcount = fs.dcount;
    sm.scan = fs.scan;
    sm.red = fs.red;
    sm.run = nullptr;
    const uint64_t* src = a.keys + first;
    if (count <= NT)
        tilesort::sort_tile<NT, 1>(src, count, a.slot_gi, sm, a.sort_prefix_bits);
    else if (count <= 2 * NT)
        tilesort::sort_tile<NT, 2>(src, count, a.slot_gi, sm, a.sort_prefix_bits);
    else if (count <= 4 * NT)
        tilesort::sort_tile<NT, 4>(src, count, a.slot_gi, sm, a.sort_prefix_bits);
    else
        tilesort::sort_tile<NT, 8>(src, count, a.slot_gi, sm, a.sort_prefix_bits);
    return fs.k;
}

// Slot of the idx-th entry of the tile whose list starts at `first`.
__device__ __forceinline__ int slot_at(const RasterArgs& a, const uint64_t* sk, const int first, const int idx)
{
    return sk ? (int)(uint32_t)sk[idx] : __ldg(&a.values[first + idx]);
}

// ---- GS_TERM_REFERENCE ------------------------------------------------------------
//
// The reference's blend and termination, bit for bit: every pixel evaluates
// every entry, in batches of 32, and after each batch the tile stops once no
// pixel has T > 0.02.  Each warp owns an 8x8 pixel block, two pixels per
// thread (rows y and y + 4, same column) that share dx and the column terms.
// The reference's expression (gaussian_render.cu:727-737) as nvcc contracts it:
//   q     = fma((2 b) dx, dy, fma(a dx, dx, (c dy) dy))
//   alpha = opacity * sat(__expf(-0.5 q))
//   rgb   = fma(rgb_s T, alpha, rgb);   T = T (1 - alpha)
// Every lane reads each entry from shared memory (40 bytes: centre, conic,
// colour, as staged), so the tile's reads of an entry are as small as the
// entry: the shared-memory data path, not the FP32 pipe, bounds this loop.
// The batches are double-buffered: the first warp starts asynchronous
// copies (cp.async, global -> shared, no registers held) of batch k + 1 and
// loads the indices of batch k + 2 before the tile blends batch k; the
// barrier that ends batch k publishes batch k + 1.
struct RefSmem {
    float2 xy[64];
    float4 con[64];  // (a, b, c, -)
    float4 col[64];  // (red, green, blue, opacity)
};

// One pixel of the pair: dy, the row terms, alpha, colour and T.
__device__ __forceinline__ void blend_ref_pixel(const float cy, const float y, const float dx, const float adx,
                                                const float b2dx, const float4 k, const float4 col, float& R, float& G,
                                                float& B, float& T)
{
    const float dy = __fsub_rn(cy, y);
    const float inner = fmaf(adx, dx, __fmul_rn(__fmul_rn(k.z, dy), dy));
    const float q = fmaf(b2dx, dy, inner);
    const float alpha = __fmul_rn(col.w, __saturatef(__expf(__fmul_rn(-0.5f, q))));
    R = fmaf(__fmul_rn(col.x, T), alpha, R);
    G = fmaf(__fmul_rn(col.y, T), alpha, G);
    B = fmaf(__fmul_rn(col.z, T), alpha, B);
    T = __fmul_rn(T, __fsub_rn(1.0f, alpha));
}

// 2 b is exact (a power of two scaling), so forming it here changes no rounding.
__device__ __forceinline__ void blend_ref_pair(const float cx, const float cy0, const float cy1, const RefSmem& sm,
                                               const int j, float (&R)[2], float (&G)[2], float (&B)[2], float (&T)[2])
{
    const float2 c = sm.xy[j];
    const float4 k = sm.con[j];
    const float4 col = sm.col[j];
    const float dx = __fsub_rn(cx, c.x);
    const float adx = __fmul_rn(k.x, dx);
    const float b2dx = __fmul_rn(2.0f * k.y, dx);
    blend_ref_pixel(cy0, c.y, dx, adx, b2dx, k, col, R[0], G[0], B[0], T[0]);
    blend_ref_pixel(cy1, c.y, dx, adx, b2dx, k, col, R[1], G[1], B[1], T[1]);
}

template <int TW, int TH>
__device__ __forceinline__ void raster_ref_tile(const RasterArgs& a, const ViewParams& v, const int64_t gtile,
                                                const int local_tile, RefSmem& sm, FusedSortSmem<TW * TH / 2>& fs)
{
    constexpr int WX = TW / 8;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int first = __ldg(&a.ranges[2 * gtile]);
    const int last = __ldg(&a.ranges[2 * gtile + 1]);
    const int count = last - first;
    const int tx = local_tile % v.tiles_x, ty = local_tile / v.tiles_x;
    const int wx0 = tx * TW + (warp % WX) * 8, wy0 = ty * TH + (warp / WX) * 8;
    const int px = wx0 + (lane & 7), py0 = wy0 + (lane >> 3), py1 = py0 + 4;
    const bool in0 = px < v.width && py0 < v.height;
    const bool in1 = px < v.width && py1 < v.height;
    if (count <= 0) {
        // the reference clears the image and skips empty tiles (main.cpp:363);
        // writing zeros here instead saves the separate clear
        if (a.write_empty) {
            if (in0) v.out[(int64_t)py0 * v.width + px] = make_uchar4(0, 0, 0, 0);
            if (in1) v.out[(int64_t)py1 * v.width + px] = make_uchar4(0, 0, 0, 0);
        }
        return;
    }
    const uint64_t* sk = fused_sort<TW * TH / 2>(a, first, count, fs);
    // pixel corner sample, gaussian_render.cu:701-704
    const float cx = (float)px * v.texel_x - 1.0f;
    const float cy0 = (float)py0 * v.texel_y - 1.0f;
    const float cy1 = (float)py1 * v.texel_y - 1.0f;
    float R[2] = {0.0f, 0.0f}, G[2] = {0.0f, 0.0f}, B[2] = {0.0f, 0.0f}, T[2] = {1.0f, 1.0f};
    const RasterSmem rs = {sm.xy, sm.con, sm.col, nullptr};
    const bool loader = threadIdx.x < 32;
    const int t = (int)threadIdx.x;
    if (loader && t < count) stage_entry(a, slot_at(a, sk, first, t), rs, t);
    cp_async_commit();
    int idx_next = (loader && 32 + t < count) ? slot_at(a, sk, first, 32 + t) : 0;
    cp_async_wait_all();
    __syncthreads();
    for (int base = 0; base < count; base += 32) {
        const int buf = (base >> 5) & 1;
        const int nb = min(32, count - base);
        const bool more = loader && base + 32 + t < count;
        if (more) stage_entry(a, idx_next, rs, 32 * (buf ^ 1) + t);
        cp_async_commit();
        const int n2 = base + 64 + t;
        const int idx2 = (loader && n2 < count) ? slot_at(a, sk, first, n2) : 0;
        const int j0 = 32 * buf;
        if (nb == 32) {
#pragma unroll 8
            for (int j = j0; j < j0 + 32; ++j) blend_ref_pair(cx, cy0, cy1, sm, j, R, G, B, T);
        } else {
            for (int j = j0; j < j0 + nb; ++j) blend_ref_pair(cx, cy0, cy1, sm, j, R, G, B, T);
        }
        idx_next = idx2;
        cp_async_wait_all();
        if (__syncthreads_count((in0 && T[0] > 0.02f) || (in1 && T[1] > 0.02f)) == 0) break;
    }
    if (in0) store_pixel(v, px, py0, R[0], G[0], B[0]);
    if (in1) store_pixel(v, px, py1, R[1], G[1], B[1]);
}

template <int TW, int TH>
__global__ void __launch_bounds__(TW * TH / 2, 2048 / (TW * TH)) raster_ref_kernel(RasterArgs a)
{
    __shared__ RefSmem sm;
    __shared__ FusedSortSmem<TW * TH / 2> fs;
    const int64_t gtile = a.order ? (int64_t)__ldg(&a.order[blockIdx.x]) : (int64_t)blockIdx.x + a.view0.tile_offset;
    raster_ref_tile<TW, TH>(a, a.view0, gtile, (int)(gtile - a.view0.tile_offset), sm, fs);
}

// Persistent variant over the flattened tiles of all views.
template <int TW, int TH>
__global__ void __launch_bounds__(TW * TH / 2, 2048 / (TW * TH)) raster_ref_persistent_kernel(RasterArgs a)
{
    __shared__ RefSmem sm;
    __shared__ FusedSortSmem<TW * TH / 2> fs;
    __shared__ int64_t s_tile;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const int64_t k = (int64_t)atomicAdd(a.tile_counter, 1ull);
            s_tile = k < a.num_tiles_total && a.order ? (int64_t)a.order[k] : k;
        }
        __syncthreads();
        const int64_t gtile = s_tile;
        if (gtile >= a.num_tiles_total) return;
        int lo = 0, hi = a.num_views - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.views[mid].tile_offset <= gtile)
                lo = mid;
            else
                hi = mid - 1;
        }
        const ViewParams& v = a.views[lo];
        raster_ref_tile<TW, TH>(a, v, gtile, (int)(gtile - v.tile_offset), sm, fs);
    }
}

template <int TW, int TH, int MODE>
__global__ void __launch_bounds__(TW * TH, 2048 / (TW * TH) * 5 / 8) raster_kernel(RasterArgs a)
{
    __shared__ float2 s_xy[TW * TH];
    __shared__ float4 s_con[TW * TH];
    __shared__ float4 s_col[TW * TH];
    __shared__ float4 s_box[TW * TH];
    const RasterSmem sm = {s_xy, s_con, s_col, s_box};
    raster_tile<TW, TH, MODE>(a, a.view0, (int64_t)blockIdx.x + a.view0.tile_offset, (int)blockIdx.x, sm);
}

// Persistent variant over the flattened tiles of all views.
template <int TW, int TH, int MODE>
__global__ void __launch_bounds__(TW * TH) raster_persistent_kernel(RasterArgs a)
{
    __shared__ float2 s_xy[TW * TH];
    __shared__ float4 s_con[TW * TH];
    __shared__ float4 s_col[TW * TH];
    __shared__ float4 s_box[TW * TH];
    __shared__ int64_t s_tile;
    const RasterSmem sm = {s_xy, s_con, s_col, s_box};
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(a.tile_counter, 1ull);
        __syncthreads();
        const int64_t gtile = s_tile;
        if (gtile >= a.num_tiles_total) return;
        // view owning this tile: binary search over the views' first tiles
        int lo = 0, hi = a.num_views - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.views[mid].tile_offset <= gtile)
                lo = mid;
            else
                hi = mid - 1;
        }
        const ViewParams& v = a.views[lo];
        raster_tile<TW, TH, MODE>(a, v, gtile, (int)(gtile - v.tile_offset), sm);
    }
}

// ---- GS_TERM_TMIN from raster records --------------------------------------
//
// The frame pipeline's kernel for the T_min mode.  One CTA per tile (all
// views' tiles in one grid), no CTA-wide barrier: each warp owns an 8x8
// pixel block, two pixels per lane (rows y and y + 4, same column), and
// walks the tile's sorted list on its own, 32 entries at a time -- lane l
// loads entry l's record (48 bytes, gathered through L1, shared by the
// tile's warps) and tests its cull extents against the block; the
// survivors are packed in list order into per-warp shared-memory slots
// (rank = popcount of the ballot below the lane) and every lane blends them
// into both its pixels.  Every lane reads every survivor, so the slots hold
// each value once (36 bytes: x, A, B, L, y, C and the colour): the
// shared-memory reads, not the arithmetic, bound this loop, and duplicated
// pair operands would double them.  The column terms of the exponent
// (A dx^2 + L, B dx) are formed once per lane and shared by its two pixels;
// the weights and T are updated as one packed f32x2 pair.
// Blend per pixel: alpha = 2^(A dx^2 + B dx dy + C dy^2 + L) (opacity
// folded in as L = log2(opacity); the conics are positive definite, so
// alpha <= opacity), w = T alpha, colour += rgb w, T -= w.  A warp stops
// after the chunk in which all its pixels reached T < t_min; a pixel that
// got there earlier keeps blending until then, which adds less than t_min
// to its colour (the w that follow sum to less than its T).

__device__ __forceinline__ float ex2_approx(const float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Shared memory of the record raster: per-warp survivor slots (CHUNK per
// warp) and the fused tile sort.
template <int TW, int TH, int CHUNK>
struct RecSmem {
    static constexpr int NW = TW * TH / 64;
    float4 s[NW][CHUNK];  // (x, A, B, L)
    float4 q[NW][CHUNK];  // (y, C, red, green)
    float b[NW][CHUNK];   // blue
    FusedSortSmem<TW * TH / 2> fs;
};

// The view a global tile belongs to: binary search over the views' first tiles.
__device__ __forceinline__ const ViewParams& view_of_tile(const RasterArgs& a, const int64_t gtile)
{
    if (a.num_views <= 1) return a.view0;
    int vi = 0, hi = a.num_views - 1;
    while (vi < hi) {
        const int mid = (vi + hi + 1) >> 1;
        if (a.views[mid].tile_offset <= gtile)
            vi = mid;
        else
            hi = mid - 1;
    }
    return a.views[vi];
}

// One tile of the record raster.  Every thread of the CTA must call it (the
// fused sort synchronises the CTA).  CHUNK = the entries a warp culls and
// stages in shared memory per step, the raster's batch of Gaussians (32 or
// 64: R = CHUNK / 32 records per lane).
template <int TW, int TH, int CHUNK>
__device__ __forceinline__ void raster_rec_tile(const RasterArgs& a, const int64_t gtile, RecSmem<TW, TH, CHUNK>& sm)
{
    constexpr int WX = TW / 8;
    constexpr int R = CHUNK / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const ViewParams& v = view_of_tile(a, gtile);
    const int local_tile = (int)(gtile - v.tile_offset);
    const int first = __ldg(&a.ranges[2 * gtile]);
    const int last = __ldg(&a.ranges[2 * gtile + 1]);
    const int tx = local_tile % v.tiles_x, ty = local_tile / v.tiles_x;
    const int wx0 = tx * TW + (warp % WX) * 8, wy0 = ty * TH + (warp / WX) * 8;
    const int px = wx0 + (lane & 7), py0 = wy0 + (lane >> 3), py1 = py0 + 4;
    const bool in0 = px < v.width && py0 < v.height;
    const bool in1 = px < v.width && py1 < v.height;
    if (last - first <= 0) {
        if (a.write_empty) {
            if (in0) v.out[(int64_t)py0 * v.width + px] = make_uchar4(0, 0, 0, 0);
            if (in1) v.out[(int64_t)py1 * v.width + px] = make_uchar4(0, 0, 0, 0);
        }
        return;
    }
    const uint64_t* sk = fused_sort<TW * TH / 2>(a, first, last - first, sm.fs);
    const float cx = (float)px * v.texel_x - 1.0f;
    const float cy0 = (float)py0 * v.texel_y - 1.0f;
    const float cy1 = (float)py1 * v.texel_y - 1.0f;
    const float bx0 = (float)wx0 * v.texel_x - 1.0f, bx1 = (float)(wx0 + 7) * v.texel_x - 1.0f;
    const float by0 = (float)wy0 * v.texel_y - 1.0f, by1 = (float)(wy0 + 7) * v.texel_y - 1.0f;
    // pixels outside the image start done (T = 0)
    f2 TT = f2_pack(in0 ? 1.0f : 0.0f, in1 ? 1.0f : 0.0f);
    float R0 = 0.0f, R1 = 0.0f, G0 = 0.0f, G1 = 0.0f, B0 = 0.0f, B1 = 0.0f;
    const float tmin = a.t_min;
    const unsigned lt = lanemask_lt();
    bool done = !in0 && !in1;

    // each chunk's cull records are loaded one chunk ahead, so their
    // latency overlaps the blend of the chunk before
    float4 qn[R];
    const float4* rpn[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        qn[r] = make_float4(0.f, 0.f, 0.f, 0.f);
        rpn[r] = nullptr;
        if (first + 32 * r + lane < last) {
            rpn[r] = a.rec + 3 * (int64_t)slot_at(a, sk, first, 32 * r + lane);
            qn[r] = __ldg(rpn[r]);
        }
    }
    for (int base = first; base < last; base += CHUNK) {
        if (__all_sync(kFull, done)) break;
        bool keep[R];
        unsigned bal[R];
        const float4* rp[R];
        float4 q0[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int j = base + 32 * r + lane;
            q0[r] = qn[r];  // (x, y, ext_x, ext_y)
            rp[r] = rpn[r];
            keep[r] = j < last && (q0[r].x - q0[r].z <= bx1) && (q0[r].x + q0[r].z >= bx0) &&
                      (q0[r].y - q0[r].w <= by1) && (q0[r].y + q0[r].w >= by0);
            bal[r] = __ballot_sync(kFull, keep[r]);
        }
        float4 q1[R], q2[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (keep[r]) {
                q1[r] = __ldg(rp[r] + 1);  // (A, B, C, L)
                q2[r] = __ldg(rp[r] + 2);  // (red, green, blue, 0)
            }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int j = base + CHUNK + 32 * r + lane;
            if (j < last) {
                rpn[r] = a.rec + 3 * (int64_t)slot_at(a, sk, first, j - first);
                qn[r] = __ldg(rpn[r]);
            }
        }
        int below = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (keep[r]) {
                const int k = below + __popc(bal[r] & lt);
                sm.s[warp][k] = make_float4(q0[r].x, q1[r].x, q1[r].y, q1[r].w);
                sm.q[warp][k] = make_float4(q0[r].y, q1[r].z, q2[r].x, q2[r].y);
                sm.b[warp][k] = q2[r].z;
            }
            below += __popc(bal[r]);
        }
        __syncwarp();  // slot writes visible to the whole warp
        const int cnt = below;
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            const float4 e = sm.s[warp][k];
            const float4 q = sm.q[warp][k];
            const float bl = sm.b[warp][k];
            const float dx = cx - e.x;
            const float adx2 = fmaf(e.y * dx, dx, e.w);  // A dx^2 + L
            const float bdx = __fmul_rn(e.z, dx);  // kept apart from the fma below
            const float dy0 = cy0 - q.x, dy1 = cy1 - q.x;
            const float p0 = fmaf(fmaf(q.y, dy0, bdx), dy0, adx2);
            const float p1 = fmaf(fmaf(q.y, dy1, bdx), dy1, adx2);
            const f2 w = f2_mul(TT, f2_pack(ex2_approx(p0), ex2_approx(p1)));
            float w0, w1;
            f2_unpack(w, w0, w1);
            R0 = fmaf(q.z, w0, R0);
            R1 = fmaf(q.z, w1, R1);
            G0 = fmaf(q.w, w0, G0);
            G1 = fmaf(q.w, w1, G1);
            B0 = fmaf(bl, w0, B0);
            B1 = fmaf(bl, w1, B1);
            TT = f2_sub(TT, w);
        }
        __syncwarp();  // slots are rewritten by the next chunk
        float T0, T1;
        f2_unpack(TT, T0, T1);
        done = T0 < tmin && T1 < tmin;
    }
    if (in0) store_pixel(v, px, py0, R0, G0, B0);
    if (in1) store_pixel(v, px, py1, R1, G1, B1);
}

// One CTA per tile, in the raster order (heavy tiles first) or of the view
// group [tile_base, tile_base + grid).
template <int TW, int TH, int CHUNK>
__global__ void __launch_bounds__(TW * TH / 2, 2048 / (TW * TH)) raster_rec_kernel(RasterArgs a)
{
    __shared__ RecSmem<TW, TH, CHUNK> sm;
    const int64_t gtile = a.order ? (int64_t)__ldg(&a.order[blockIdx.x]) : a.tile_base + (int64_t)blockIdx.x;
    raster_rec_tile<TW, TH, CHUNK>(a, gtile, sm);
}

// Persistent CTAs (as many as fit on the SMs at once) that pull tiles from
// an atomic queue over the raster order (heavy tiles first) until it runs
// dry.
template <int TW, int TH, int CHUNK>
__global__ void __launch_bounds__(TW * TH / 2, 2048 / (TW * TH)) raster_rec_persistent_kernel(RasterArgs a)
{
    __shared__ RecSmem<TW, TH, CHUNK> sm;
    __shared__ int64_t s_tile;
    for (;;) {
        if (threadIdx.x == 0) {
            const int64_t k = (int64_t)atomicAdd(a.tile_counter, 1ull);
            s_tile = k < a.num_tiles_total ? (a.order ? (int64_t)__ldg(&a.order[k]) : a.tile_base + k) : -1;
        }
        __syncthreads();
        const int64_t gtile = s_tile;
        if (gtile < 0) return;
        raster_rec_tile<TW, TH, CHUNK>(a, gtile, sm);
        __syncthreads();  // s_tile and the sort's shared memory are reused
    }
}

template <int TW, int TH, int CHUNK>
static void launch_rec(const RasterArgs& a, bool persistent, int num_sms, cudaStream_t st)
{
    if (a.num_tiles_total <= 0) return;
    if (!persistent) {
        raster_rec_kernel<TW, TH, CHUNK><<<(unsigned)a.num_tiles_total, TW * TH / 2, 0, st>>>(a);
        return;
    }
    static int per_sm = 0;  // same on every B200; queried once
    if (per_sm == 0) {
        int x = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&x, raster_rec_persistent_kernel<TW, TH, CHUNK>, TW * TH / 2, 0);
        per_sm = std::max(x, 1);
    }
    const int64_t grid = std::min<int64_t>((int64_t)per_sm * num_sms, a.num_tiles_total);
    raster_rec_persistent_kernel<TW, TH, CHUNK><<<(unsigned)grid, TW * TH / 2, 0, st>>>(a);
}

template <int TW, int TH>
static void launch_shape(const RasterArgs& a, int termination, bool persistent, int num_sms, cudaStream_t st)
{
    if (a.rec && termination == 1) {
        // the record raster's queue is the frame's tile counter; persistent
        // only when asked (RasterArgs::rec_persistent)
        if (a.rec_chunk == 64)
            launch_rec<TW, TH, 64>(a, a.rec_persistent != 0, num_sms, st);
        else
            launch_rec<TW, TH, 32>(a, a.rec_persistent != 0, num_sms, st);
        return;
    }
    if (termination == 0) {
        if (a.num_tiles_total <= 0) return;
        if (persistent) {
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raster_ref_persistent_kernel<TW, TH>, TW * TH / 2, 0);
            const int64_t grid = std::min<int64_t>((int64_t)std::max(per_sm, 1) * num_sms, a.num_tiles_total);
            raster_ref_persistent_kernel<TW, TH><<<(unsigned)grid, TW * TH / 2, 0, st>>>(a);
        } else {
            raster_ref_kernel<TW, TH><<<(unsigned)a.num_tiles_total, TW * TH / 2, 0, st>>>(a);
        }
        return;
    }
    if (persistent) {
        int per_sm = 0;
        if (termination == 0)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raster_persistent_kernel<TW, TH, 0>, TW * TH, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raster_persistent_kernel<TW, TH, 1>, TW * TH, 0);
        const int64_t grid = std::min<int64_t>((int64_t)std::max(per_sm, 1) * num_sms, a.num_tiles_total);
        if (grid <= 0) return;
        if (termination == 0)
            raster_persistent_kernel<TW, TH, 0><<<(unsigned)grid, TW * TH, 0, st>>>(a);
        else
            raster_persistent_kernel<TW, TH, 1><<<(unsigned)grid, TW * TH, 0, st>>>(a);
    } else {
        if (a.num_tiles_total <= 0) return;
        if (termination == 0)
            raster_kernel<TW, TH, 0><<<(unsigned)a.num_tiles_total, TW * TH, 0, st>>>(a);
        else
            raster_kernel<TW, TH, 1><<<(unsigned)a.num_tiles_total, TW * TH, 0, st>>>(a);
    }
}

void launch_raster(const RasterArgs& a, int tile_w, int tile_h, int termination, bool persistent, int num_sms,
                   cudaStream_t st)
{
    if (tile_w == 16 && tile_h == 16)
        launch_shape<16, 16>(a, termination, persistent, num_sms, st);
    else if (tile_w == 16 && tile_h == 8)
        launch_shape<16, 8>(a, termination, persistent, num_sms, st);
    else
        launch_shape<8, 8>(a, termination, persistent, num_sms, st);
}

}  // namespace gs
