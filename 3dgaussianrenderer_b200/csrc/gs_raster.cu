// Tile rasteriser (replaces rasterizeTilesKernel, core/gaussian_render.cu:679-775).
//
// One CTA per tile, one thread per pixel.  The tile's depth-sorted entries
// are consumed in batches of one entry per thread: every thread gathers one
// splat (centre, conic + opacity, colour) into shared memory, then every
// pixel blends the whole batch front to back in FP32.
//
// Termination:
//  * GS_TERM_REFERENCE: after every 32nd entry of the tile's list the CTA
//    stops once no in-image pixel has T > 0.02 (the reference's test at
//    :745, at the same 32-entry granularity whatever the batch size).
//  * GS_TERM_TMIN: a pixel stops once its T < t_min; a warp whose pixels
//    are all done skips the batch (warp ballot), the CTA stops when every
//    pixel is done.
//
// The plain path launches one CTA per tile; the batched path runs a
// persistent grid that pulls global tile ids (all views' tiles, flattened)
// from an atomic queue.
#include "gs_kernels.h"

#include <algorithm>

namespace gs {

template <int TW, int TH, int MODE>
__device__ __forceinline__ void raster_tile(const RasterArgs& a, const ViewParams& v, const int64_t gtile,
                                            const int local_tile, float2* s_xy, float4* s_con, float4* s_col)
{
    constexpr int NT = TW * TH;
    const int first = __ldg(&a.ranges[2 * gtile]);
    const int last = __ldg(&a.ranges[2 * gtile + 1]);
    const int count = last - first;
    const int tx = local_tile % v.tiles_x, ty = local_tile / v.tiles_x;
    const int px = tx * TW + (int)(threadIdx.x % TW);
    const int py = ty * TH + (int)(threadIdx.x / TW);
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

    float r = 0.0f, g = 0.0f, b = 0.0f;
    float T = 1.0f;
    bool done = !inimg;

    for (int base = 0; base < count; base += NT) {
        const int nb = min(NT, count - base);
        __syncthreads();
        if ((int)threadIdx.x < nb) {
            const int s = __ldg(&a.values[first + base + threadIdx.x]);
            const float4 col = __ldg(&a.color[s]);
            const float4 con = __ldg(&a.conic[s]);
            s_xy[threadIdx.x] = __ldg(&a.xy[s]);
            s_con[threadIdx.x] = make_float4(con.x, con.y, con.z, col.w);
            s_col[threadIdx.x] = col;
        }
        __syncthreads();
        if (MODE == 0) {
            bool stop = false;
            for (int j = 0; j < nb; ++j) {
                const float2 c = s_xy[j];
                const float4 k = s_con[j];
                const float4 col = s_col[j];
                const float dx = cx - c.x, dy = cy - c.y;
                const float q = k.x * dx * dx + k.z * dy * dy + 2.0f * k.y * dx * dy;
                const float density = __expf(-0.5f * q);
                const float alpha = k.w * __saturatef(density);
                r += col.x * T * alpha;
                g += col.y * T * alpha;
                b += col.z * T * alpha;
                T *= (1.0f - alpha);
                const int e = base + j + 1;
                if ((e & 31) == 0 || e == count) {
                    if (__syncthreads_count(inimg && T > 0.02f) == 0) {
                        stop = true;
                        break;
                    }
                }
            }
            if (stop) break;
        } else {
            if (__any_sync(kFull, !done)) {
                for (int j = 0; j < nb; ++j) {
                    if (!done) {
                        const float2 c = s_xy[j];
                        const float4 k = s_con[j];
                        const float4 col = s_col[j];
                        const float dx = cx - c.x, dy = cy - c.y;
                        const float q = k.x * dx * dx + k.z * dy * dy + 2.0f * k.y * dx * dy;
                        const float density = __expf(-0.5f * q);
                        const float alpha = k.w * __saturatef(density);
                        r += col.x * T * alpha;
                        g += col.y * T * alpha;
                        b += col.z * T * alpha;
                        T *= (1.0f - alpha);
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

template <int TW, int TH, int MODE>
__global__ void __launch_bounds__(TW * TH) raster_kernel(RasterArgs a)
{
    __shared__ float2 s_xy[TW * TH];
    __shared__ float4 s_con[TW * TH];
    __shared__ float4 s_col[TW * TH];
    raster_tile<TW, TH, MODE>(a, a.view0, (int64_t)blockIdx.x + a.view0.tile_offset, (int)blockIdx.x, s_xy, s_con,
                              s_col);
}

// Persistent variant over the flattened tiles of all views.
template <int TW, int TH, int MODE>
__global__ void __launch_bounds__(TW * TH) raster_persistent_kernel(RasterArgs a)
{
    __shared__ float2 s_xy[TW * TH];
    __shared__ float4 s_con[TW * TH];
    __shared__ float4 s_col[TW * TH];
    __shared__ int64_t s_tile;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(a.tile_counter, 1ull);
        __syncthreads();
        const int64_t gtile = s_tile;
        if (gtile >= a.num_tiles_total) return;
        // view owning this tile: views are few, a linear scan is enough
        int view = 0;
        while (view + 1 < a.num_views && a.views[view + 1].tile_offset <= gtile) ++view;
        const ViewParams& v = a.views[view];
        raster_tile<TW, TH, MODE>(a, v, gtile, (int)(gtile - v.tile_offset), s_xy, s_con, s_col);
    }
}

template <int TW, int TH>
static void launch_shape(const RasterArgs& a, int termination, bool persistent, int num_sms, cudaStream_t st)
{
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
