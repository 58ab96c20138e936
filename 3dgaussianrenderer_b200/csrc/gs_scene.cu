// Spatial storage order of a scene (scene upload, Renderer::UploadModel,
// core/renderer.cpp:36-88).
//
// A scene is stored in Morton (Z-curve) order of the Gaussian centres, so
// Gaussians that are close in space are close in memory: a warp of the
// frame kernel then tends to see Gaussians of one screen region (whole
// warps outside the view skip the SH evaluation, per-tile count atomics and
// raster records of one tile come from nearby slots), which is what the
// caller's order does not guarantee.  The order is a storage detail: every
// Gaussian keeps its caller index (`orig`), and the tile lists break equal
// depths by that index, so images are those of the caller's order.
#include "gs_kernels.h"

namespace gs {

namespace {

// 10 bits of x spread to every third bit
__device__ __forceinline__ uint32_t spread3(uint32_t x)
{
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x30000FFu;
    x = (x | (x << 8)) & 0x300F00Fu;
    x = (x | (x << 4)) & 0x30C30C3u;
    x = (x | (x << 2)) & 0x9249249u;
    return x;
}

__device__ __forceinline__ uint32_t cell(const float v, const float lo, const float scale)
{
    // NaN and out-of-box values land on the box's faces
    return (uint32_t)fminf(fmaxf((v - lo) * scale, 0.0f), 1023.0f);
}

__global__ void __launch_bounds__(256) morton_kernel(int64_t n, const float4* __restrict__ pos, float3 lo,
                                                     float3 scale, uint64_t* __restrict__ keys,
                                                     int32_t* __restrict__ vals)
{
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float4 p = __ldg(&pos[i]);
    const uint32_t code = spread3(cell(p.x, lo.x, scale.x)) | (spread3(cell(p.y, lo.y, scale.y)) << 1) |
                          (spread3(cell(p.z, lo.z, scale.z)) << 2);
    keys[i] = code;
    vals[i] = (int32_t)i;
}

// dst[j] = src[perm[j]] for the float4 arrays; orig[j] = perm[j]
__global__ void __launch_bounds__(256) gather_kernel(int64_t n, const int32_t* __restrict__ perm,
                                                     const float4* __restrict__ pos_in, const float4* __restrict__ sr_in,
                                                     const float4* __restrict__ col_in, float4* __restrict__ pos,
                                                     float4* __restrict__ sr, float4* __restrict__ col,
                                                     int32_t* __restrict__ orig)
{
    const int64_t j = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (j >= n) return;
    const int32_t o = __ldg(&perm[j]);
    if (o < 0 || o >= n) return;  // only after a failed sort (reported by its error word)
    pos[j] = __ldg(&pos_in[o]);
    sr[j] = __ldg(&sr_in[o]);
    if (col) col[j] = __ldg(&col_in[o]);
    orig[j] = o;
}

// Grouped SH layout [group][coefficient][256]: one thread per (j, c); the
// writes of a warp are one coefficient row of 32 consecutive Gaussians.
__global__ void __launch_bounds__(256) gather_sh_kernel(int64_t n, int32_t sh_count, const int32_t* __restrict__ perm,
                                                        const float* __restrict__ in, float* __restrict__ out)
{
    const int64_t j = (int64_t)blockIdx.x * 256 + threadIdx.x;  // destination Gaussian
    const int c = blockIdx.y;
    if (j >= n) return;
    const int64_t o = __ldg(&perm[j]);
    if (o < 0 || o >= n) return;
    out[(j >> 8) * 256 * sh_count + (int64_t)c * 256 + (j & 255)] =
        __ldg(&in[(o >> 8) * 256 * sh_count + (int64_t)c * 256 + (o & 255)]);
}

}  // namespace

void launch_morton(int64_t n, const float4* pos, const float lo[3], const float hi[3], uint64_t* keys, int32_t* vals,
                   cudaStream_t st)
{
    if (n <= 0) return;
    float3 l = make_float3(lo[0], lo[1], lo[2]);
    float3 s;
    s.x = hi[0] > lo[0] ? 1024.0f / (hi[0] - lo[0]) : 0.0f;
    s.y = hi[1] > lo[1] ? 1024.0f / (hi[1] - lo[1]) : 0.0f;
    s.z = hi[2] > lo[2] ? 1024.0f / (hi[2] - lo[2]) : 0.0f;
    morton_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, pos, l, s, keys, vals);
}

void launch_scene_gather(int64_t n, const int32_t* perm, const float4* pos_in, const float4* sr_in,
                         const float4* col_in, const float* sh_in, int32_t sh_count, float4* pos, float4* sr,
                         float4* col, float* sh, int32_t* orig, cudaStream_t st)
{
    if (n <= 0) return;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    gather_kernel<<<blocks, 256, 0, st>>>(n, perm, pos_in, sr_in, col_in, pos, sr, col, orig);
    if (sh_in && sh_count > 0) gather_sh_kernel<<<dim3(blocks, (unsigned)sh_count), 256, 0, st>>>(n, sh_count, perm, sh_in, sh);
}

}  // namespace gs
