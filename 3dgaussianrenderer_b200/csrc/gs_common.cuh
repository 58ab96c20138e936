// Shared device code of the gs_b200 frame pipeline (sm_100a).
//
// The projection and tile-overlap arithmetic below keeps the operation
// order of the reference kernels (RobinSongx/3DGaussianRenderer,
// core/gaussian_render.cu:45-310, which use glm 0.9.9): tile counts, keys
// and ranges derive from these floats, and they can only be bit-exact with
// the reference if every product and sum is formed in the same order and
// contracted the same way by nvcc.  The code is otherwise this project's
// own: plain scalar CUDA, no glm.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gs {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Per-view constants, filled on the host by make_view_params().
struct ViewParams {
    float view[16];  // column-major, view[c*4 + r]
    float cam[3];
    float cot[2];
    float dsb[2];
    float aspect;
    int32_t width, height;
    int32_t tile_w, tile_h;
    int32_t tiles_x, tiles_y;
    float tiles_xf, tiles_yf;  // W / tile_w, H / tile_h (64.0 at 1024/16)
    float tclip_x, tclip_y;    // (tile_w / W) * 2 (0.03125 at 1024/16)
    float texel_x, texel_y;    // 2 / W, 2 / H
    float bump_x, bump_y;      // (1/pi) * texel^2, gaussian_render.cu:184-188
    int64_t tile_offset;       // first global tile id of this view (batched frames)
    uchar4* out;               // this view's RGBA image (raster output)
};

// glm scalar min/max/clamp (glm/detail/func_common.inl:17-30, 505-509).
__device__ __forceinline__ float gmin(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return (x < y) ? y : x; }
__device__ __forceinline__ float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
__device__ __forceinline__ int imin(int x, int y) { return (y < x) ? y : x; }
__device__ __forceinline__ int imax(int x, int y) { return (x < y) ? y : x; }
__device__ __forceinline__ int iclamp(int x, int lo, int hi) { return imin(imax(x, lo), hi); }

// 3x3 matrix, column-major m[col][row], multiplied in glm's order
// (glm/detail/type_mat3x3.inl:486-520).
struct M3 {
    float m[3][3];
};

__device__ __forceinline__ M3 mul(const M3& a, const M3& b)
{
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            r.m[i][j] = a.m[0][j] * b.m[i][0] + a.m[1][j] * b.m[i][1] + a.m[2][j] * b.m[i][2];
        }
    }
    return r;
}

__device__ __forceinline__ M3 transpose(const M3& a)
{
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
    return r;
}

// Result of projecting one Gaussian (gaussian_render.cu:135-215).
struct Splat {
    float x, y, z;      // clip-space centre (-128 when culled)
    float cs, sn;       // ellipse major axis direction
    float ex, ey;       // 3-sigma extents (0 when culled)
    float ca, cb, cc;   // conic
};

// Approximate PTX arithmetic for the T_min frames' projection (FAST): the
// hardware reciprocal, square root and reciprocal square root (a few ulp),
// where the reference-compatible path keeps IEEE division and sqrtf.
__device__ __forceinline__ float rcp_approx(const float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sqrt_approx(const float x)
{
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_approx(const float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(const float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// View position and clip-space centre of one Gaussian (the first half of
// the projection, gaussian_render.cu:160-182): enough to decide the
// frustum test, so Gaussians outside the view can skip the rest.
struct ViewPos {
    float vx, vy, vz;                  // view space
    float zRcp, zRcpSqr, ftx, fty;
    float scaleX, scaleY, shearX, shearY;
    float cx, cy, cz;                  // clip space, before the cull
};

template <bool FAST = false>
__device__ __forceinline__ ViewPos view_position(const float4 p, const ViewParams& v)
{
    ViewPos w;
    // view * vec4(position, 1): (m0*x + m1*y) + (m2*z + m3*1)
    // (glm/detail/type_mat4x4.inl:536-570)
    const float* V = v.view;
    w.vx = (V[0] * p.x + V[4] * p.y) + (V[8] * p.z + V[12] * 1.0f);
    w.vy = (V[1] * p.x + V[5] * p.y) + (V[9] * p.z + V[13] * 1.0f);
    w.vz = (V[2] * p.x + V[6] * p.y) + (V[10] * p.z + V[14] * 1.0f);

    if constexpr (FAST)
        w.zRcp = rcp_approx(w.vz);
    else
        w.zRcp = 1.0f / w.vz;
    w.zRcpSqr = w.zRcp * w.zRcp;
    w.scaleX = -v.cot[0] * w.zRcp;
    w.scaleY = -v.cot[1] * w.zRcp;
    w.ftx = v.cot[0] * w.vx;
    w.fty = v.cot[1] * w.vy;
    w.shearX = w.ftx * w.zRcpSqr;
    w.shearY = w.fty * w.zRcpSqr;
    const float translationX = -w.ftx * w.zRcp;
    const float translationY = -w.fty * w.zRcp;
    // affine * vec4(viewPosition, 1) (:182)
    w.cx = (w.scaleX * w.vx + 0.0f * w.vy) + (w.shearX * w.vz + translationX * 1.0f);
    w.cy = (0.0f * w.vx + w.scaleY * w.vy) + (w.shearY * w.vz + translationY * 1.0f);
    w.cz = (0.0f * w.vx + 0.0f * w.vy) + (v.dsb[0] * w.vz + v.dsb[1] * 1.0f);
    return w;
}

// The frustum part of the reference's visibility, step(-1, clip) *
// step(clip, 1) (:205-206): false only for a centre outside [-1, 1]^3 (a
// NaN coordinate passes, as it does there).  The eigenvalue factor
// step(0, lambda1) is always 1 (lambda1 = max(0, ...)), so a Gaussian
// that fails this test is culled and overlaps no tile.
__device__ __forceinline__ bool in_frustum(const ViewPos& w)
{
    return !(w.cx < -1.0f) && !(1.0f < w.cx) && !(w.cy < -1.0f) && !(1.0f < w.cy) && !(w.cz < -1.0f) &&
           !(1.0f < w.cz);
}

// EWA projection of one Gaussian: quaternion decode, covariance
// R S S^T R^T, affine Jacobian of the perspective divide, clip-space 2x2
// covariance plus trace bump, eigen-decomposition, conic and frustum test.
// `w` is view_position(p, v).  FAST (the T_min frames, whose geometry
// need not match the reference bit for bit): hardware reciprocal and square
// roots, and the ellipse axis taken from the normalised eigenvector itself
// instead of cos/sin of its atan2 angle, which is the same vector.
template <bool FAST = false>
__device__ __forceinline__ Splat project_gaussian(const ViewPos& w, const float4 sr, const ViewParams& v)
{
    const uint32_t bits = __float_as_uint(sr.w);
    // decodeVec4 (gaussian_render.cu:45-48), then *2 - 1 (:150)
    const float rx = (float)((bits >> 24u) & 0xFFu) / 255.0f * 2.0f - 1.0f;
    const float ry = (float)((bits >> 16u) & 0xFFu) / 255.0f * 2.0f - 1.0f;
    const float rz = (float)((bits >> 8u) & 0xFFu) / 255.0f * 2.0f - 1.0f;
    const float rw = (float)(bits & 0xFFu) / 255.0f * 2.0f - 1.0f;

    // quaternion -> rotation (glm/gtc/quaternion.inl:41-66), q = (w, x, y, z)
    const float qxx = rx * rx, qyy = ry * ry, qzz = rz * rz;
    const float qxz = rx * rz, qxy = rx * ry, qyz = ry * rz;
    const float qwx = rw * rx, qwy = rw * ry, qwz = rw * rz;
    M3 R;
    R.m[0][0] = 1.0f - 2.0f * (qyy + qzz);
    R.m[0][1] = 2.0f * (qxy + qwz);
    R.m[0][2] = 2.0f * (qxz - qwy);
    R.m[1][0] = 2.0f * (qxy - qwz);
    R.m[1][1] = 1.0f - 2.0f * (qxx + qzz);
    R.m[1][2] = 2.0f * (qyz + qwx);
    R.m[2][0] = 2.0f * (qxz + qwy);
    R.m[2][1] = 2.0f * (qyz - qwx);
    R.m[2][2] = 1.0f - 2.0f * (qxx + qyy);

    M3 S;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S.m[i][j] = 0.0f;
    S.m[0][0] = sr.x;
    S.m[1][1] = sr.y;
    S.m[2][2] = sr.z;

    const M3 RS = mul(R, S);
    const M3 cov = mul(RS, transpose(RS));

    const float* V = v.view;
    const float scaleX = w.scaleX, scaleY = w.scaleY, shearX = w.shearX, shearY = w.shearY;

    // mat3(affine) * mat3(view) (:180), affine columns
    // (scaleX,0,0) (0,scaleY,0) (shearX,shearY,dsb.x)
    M3 A;
    A.m[0][0] = scaleX; A.m[0][1] = 0.0f;   A.m[0][2] = 0.0f;
    A.m[1][0] = 0.0f;   A.m[1][1] = scaleY; A.m[1][2] = 0.0f;
    A.m[2][0] = shearX; A.m[2][1] = shearY; A.m[2][2] = v.dsb[0];
    M3 B;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) B.m[c][r] = V[c * 4 + r];
    const M3 VP = mul(A, B);
    const M3 cc = mul(mul(VP, transpose(cov)), transpose(VP));

    float cx = w.cx, cy = w.cy, cz = w.cz;

    const float c00 = cc.m[0][0] + v.bump_x;
    const float c11 = cc.m[1][1] + v.bump_y;
    const float c10 = cc.m[1][0];

    const float det = c00 * c11 - c10 * c10;
    const float mid = 0.5f * (c00 + c11);
    constexpr float eps = 1e-12f;
    const float r2 = gmax(eps, mid * mid - det);
    const float radius = FAST ? sqrt_approx(r2) : sqrtf(r2);
    const float lambda0 = mid + radius;
    const float lambda1 = gmax(0.0f, mid - radius);

    // normalize(vec2(c10, lambda0 - c00)) = v * (1 / sqrt(dot(v, v)))
    float e0x = c10, e0y = lambda0 - c00;
    const float dd = e0x * e0x + e0y * e0y;
    const float inv = FAST ? rsqrt_approx(dd) : 1.0f / sqrtf(dd);
    e0x = e0x * inv;
    e0y = e0y * inv;
    float ex = (FAST ? sqrt_approx(lambda0) : sqrtf(lambda0)) * 3.0f;
    float ey = (FAST ? sqrt_approx(lambda1) : sqrtf(lambda1)) * 3.0f;
    const float invDet = FAST ? rcp_approx(gmax(eps, det)) : 1.0f / gmax(eps, det);

    // step(-1, clip) * step(clip, 1) * step(0, lambda1)   (:205-206)
    const float edgex = (cx < -1.0f ? 0.0f : 1.0f) * (1.0f < cx ? 0.0f : 1.0f);
    const float edgey = (cy < -1.0f ? 0.0f : 1.0f) * (1.0f < cy ? 0.0f : 1.0f);
    const float edgez = (cz < -1.0f ? 0.0f : 1.0f) * (1.0f < cz ? 0.0f : 1.0f);
    const float vis = edgex * edgey * edgez * (lambda1 < 0.0f ? 0.0f : 1.0f);
    // mix(vec3(-128), clip, vis) = -128*(1-vis) + clip*vis   (:207)
    const float om = 1.0f - vis;
    cx = -128.0f * om + cx * vis;
    cy = -128.0f * om + cy * vis;
    cz = -128.0f * om + cz * vis;
    ex *= vis;
    ey *= vis;

    Splat s;
    s.x = cx;
    s.y = cy;
    s.z = cz;
    if constexpr (FAST) {
        s.cs = e0x;
        s.sn = e0y;
    } else {
        const float angle = atan2f(e0y, e0x);
        s.cs = cosf(angle);
        s.sn = sinf(angle);
    }
    s.ex = ex;
    s.ey = ey;
    s.ca = c11 * invDet;
    s.cb = -c10 * invDet;
    s.cc = c00 * invDet;
    return s;
}

__device__ __forceinline__ Splat project_gaussian(const float4 p, const float4 sr, const ViewParams& v)
{
    return project_gaussian(view_position(p, v), sr, v);
}

// ---- SH colour (gaussian_render.cu:50-94; degree 3: cuda_renderer.cu:119-156)
// sh points at coefficient 0 of this Gaussian, consecutive coefficients
// `stride` floats apart.
// G: coefficients in global memory (read-only path) or in shared memory.
template <bool G>
__device__ __forceinline__ float ldsh(const float* p)
{
    if (G) return __ldg(p);
    return *p;
}

template <int DEG, bool G = true>
__device__ __forceinline__ float3 sh_color(const float x, const float y, const float z, const float* __restrict__ sh,
                                           const int stride)
{
    float r[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c] = 0.0f + 0.282094792F * ldsh<G>(&sh[c * stride]);
    if (DEG > 0) {
        const float b1 = 0.488602512F * y, b2 = 0.488602512F * z, b3 = 0.488602512F * x;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            r[c] = r[c] + (b1 * ldsh<G>(&sh[(3 + c) * stride]) + b2 * ldsh<G>(&sh[(6 + c) * stride]) +
                           b3 * ldsh<G>(&sh[(9 + c) * stride]));
    }
    if (DEG > 1) {
        const float xx = x * x, yy = y * y;
        const float b4 = 1.09254843F * x * y;
        const float b5 = 1.09254843F * y * z;
        const float b6 = -0.946174696F * xx - 0.946174696F * yy + 0.630783131F;
        const float b7 = 1.09254843F * x * z;
        const float b8 = 0.546274215F * (x - y) * (x + y);
#pragma unroll
        for (int c = 0; c < 3; ++c)
            r[c] = r[c] + (b4 * ldsh<G>(&sh[(12 + c) * stride]) + b5 * ldsh<G>(&sh[(15 + c) * stride]) +
                           b6 * ldsh<G>(&sh[(18 + c) * stride]) + b7 * ldsh<G>(&sh[(21 + c) * stride]) +
                           b8 * ldsh<G>(&sh[(24 + c) * stride]));
    }
    if (DEG > 2) {
        const float xx = x * x, yy = y * y;
        const float b9 = 0.295021795F * y * (6.0F * xx - 2.0F * yy);
        const float b10 = 2.89061144F * x * y * z;
        const float b11 = 3.6563664F * y * (-0.625F * xx - 0.625F * yy + 0.5F);
        const float b12 = 0.373176333F * z * (-5.0F * xx - 5.0F * yy + 2.0F);
        const float b13 = 0.457045799F * x * (-5.0F * xx - 5.0F * yy + 4.0F);
        const float b14 = 1.44530572F * z * (x - y) * (x + y);
        const float b15 = 0.59004359F * x * (xx - 3.0F * yy);
#pragma unroll
        for (int c = 0; c < 3; ++c)
            r[c] = r[c] + (b9 * ldsh<G>(&sh[(27 + c) * stride]) + b10 * ldsh<G>(&sh[(30 + c) * stride]) +
                           b11 * ldsh<G>(&sh[(33 + c) * stride]) + b12 * ldsh<G>(&sh[(36 + c) * stride]) +
                           b13 * ldsh<G>(&sh[(39 + c) * stride]) + b14 * ldsh<G>(&sh[(42 + c) * stride]) +
                           b15 * ldsh<G>(&sh[(45 + c) * stride]));
    }
    return make_float3(gclamp(r[0] + 0.5f, 0.0f, 1.0f), gclamp(r[1] + 0.5f, 0.0f, 1.0f),
                       gclamp(r[2] + 0.5f, 0.0f, 1.0f));
}

// Unit view direction from a Gaussian to the camera, glm::normalize order.
__device__ __forceinline__ float3 view_dir(const ViewParams& v, const float4 p)
{
    const float dx = v.cam[0] - p.x, dy = v.cam[1] - p.y, dz = v.cam[2] - p.z;
    const float d2 = dx * dx + dy * dy + dz * dz;
    const float inv = 1.0f / sqrtf(d2);
    return make_float3(dx * inv, dy * inv, dz * inv);
}

// ---- ellipse / rectangle tests (gaussian_render.cu:234-310) -------------

struct Ell {
    float cx, cy, cs, sn, ex, ey;
};

// A point in the ellipse's frame, in units of its extents
// (convertToEllipseCoordinates, gaussian_render.cu:234-240).
__device__ __forceinline__ void to_ellipse(const Ell& e, const float px, const float py, float& ox, float& oy)
{
    const float dx = px - e.cx, dy = py - e.cy;
    ox = (dx * e.cs + dy * e.sn) / e.ex;
    oy = (dy * e.cs - dx * e.sn) / e.ey;
}

__device__ __forceinline__ float len2(const float x, const float y) { return x * x + y * y; }

__device__ __forceinline__ bool hits_unit_circle(const float v0x, const float v0y, const float v1x, const float v1y)
{
    const float dx = v1x - v0x, dy = v1y - v0y;
    const float l2 = dx * dx + dy * dy;
    const float num = (-v0x) * dx + (-v0y) * dy;
    const float t = __saturatef(num / l2);
    const float prx = v0x + t * (v1x - v0x);
    const float pry = v0y + t * (v1y - v0y);
    return len2(prx, pry) < 1.0f;
}

// The reference's tests evaluated with the hardware reciprocal, each result
// kept as the value compared with 1 (the rectangle centre and the nearer
// edge of each parallel pair; see below).  Returns 1 (overlap) or 0 (none) when every
// value lies clearly on one side of 1, -1 otherwise.  "Clearly" is a margin
// from an error bound.  Both evaluations start from the same corners, centre,
// axis and extents.  Let R be D / min(ex, ey), where D bounds the image-space
// offsets |dx| + |dy| of the corners from the centre.  Every ellipse
// coordinate either side computes is then within about 25 u R of the exact
// one (u = 2^-24): the offset, product, sum and division roundings, and the
// reciprocal's ulp.  A distance to a segment moves by at most its endpoints'
// displacement, and its own evaluation adds a few u R more, so each compared
// value differs between the two evaluations by under about 100 u R plus a
// few u.  An emulation of both in single precision (2M candidates up to
// R = 1500, contracted and uncontracted products, reciprocals 1 ulp off either
// way) found at most 2.1 u R + 340 u.  The margin is 256 u R + 2^-15, so where
// this says clear, the reference's IEEE evaluation decides the same.
__device__ __forceinline__ int ellipse_rect_overlap_clear(const Ell& e, const float x0, const float y0,
                                                          const float x1, const float y1);

// The reference's four tests after its centre-in-rectangle test, in IEEE
// arithmetic (gaussian_render.cu:250-272).  Not inlined: it runs only for
// the rare values the cheap evaluation cannot decide, and keeping its
// divisions out of the callers' loops keeps their registers from spilling.
static __device__ __noinline__ bool ellipse_rect_overlap_ieee(const Ell e, const float x0, const float y0, const float x1,
                                                       const float y1)
{
    // Rect::getCenter = min + (max - min) * 0.5
    const float rcx = x0 + (x1 - x0) * 0.5f;
    const float rcy = y0 + (y1 - y0) * 0.5f;
    float ux, uy;
    to_ellipse(e, rcx, rcy, ux, uy);
    bool ov = len2(ux, uy) < 1.0f;
    float p0x, p0y, p1x, p1y, p2x, p2y, p3x, p3y;
    to_ellipse(e, x0, y0, p0x, p0y);
    to_ellipse(e, x1, y0, p1x, p1y);
    to_ellipse(e, x1, y1, p2x, p2y);
    to_ellipse(e, x0, y1, p3x, p3y);
    ov |= hits_unit_circle(p0x, p0y, p1x, p1y);
    ov |= hits_unit_circle(p1x, p1y, p2x, p2y);
    ov |= hits_unit_circle(p2x, p2y, p3x, p3y);
    ov |= hits_unit_circle(p3x, p3y, p0x, p0y);
    return ov;
}

// ellipseRectOverlap (gaussian_render.cu:250-272): the centre-in-rectangle
// test, then the other four of the reference's five tests, decided by a
// cheap evaluation wherever it is clear of the threshold and in IEEE
// arithmetic otherwise.  Bit-exact with the reference on every input.
__device__ __forceinline__ bool ellipse_rect_overlap(const Ell& e, const float x0, const float y0, const float x1,
                                                     const float y1)
{
    // The reference ORs all five tests, so a centre strictly inside the tile
    // decides the result; skipping the rest changes nothing.
    if (e.cx > x0 && e.cx < x1 && e.cy > y0 && e.cy < y1) return true;
    const int clear = ellipse_rect_overlap_clear(e, x0, y0, x1, y1);
    if (clear >= 0) return clear != 0;
    return ellipse_rect_overlap_ieee(e, x0, y0, x1, y1);
}

__device__ __forceinline__ int ellipse_rect_overlap_clear(const Ell& e, const float x0, const float y0,
                                                          const float x1, const float y1)
{
    // The tile's image in ellipse coordinates is a parallelogram: corner
    // (x0, y0) maps to a, the x edge to u, the y edge to v, so the other
    // corners are a + u, a + u + v, a + v and each edge's squared length is
    // |u|^2 or |v|^2 -- the same five values as the reference's tests,
    // rounded differently.
    // A zero extent -- every splat whose covariance sits at the trace bump
    // (mid^2 - det under the eps floor makes lambda1 = 0): the reference's
    // divisions give +-inf or NaN in that axis, no value compares below 1,
    // and only the centre-in-rectangle test (the caller's) can pass.
    if (e.ex == 0.0f || e.ey == 0.0f) return 0;
    const float iex = rcp_approx(e.ex), iey = rcp_approx(e.ey);
    const float dx0 = x0 - e.cx, dy0 = y0 - e.cy;
    const float ax = (dx0 * e.cs + dy0 * e.sn) * iex, ay = (dy0 * e.cs - dx0 * e.sn) * iey;
    const float w = x1 - x0, h = y1 - y0;
    const float ux = (w * e.cs) * iex, uy = -(w * e.sn) * iey;
    const float vx = (h * e.sn) * iex, vy = (h * e.cs) * iey;
    // margin from R (above); a NaN or infinite input or a corner thousands
    // of radii away lands here too: let IEEE decide
    const float R = (fabsf(dx0) + fabsf(dy0) + w + h) * fmaxf(fabsf(iex), fabsf(iey));
    const float margin = fmaf(R, 256.0f / 16777216.0f, 1.0f / 32768.0f);
    if (!(margin <= 0.125f)) return -1;
    bool unclear = false;
    auto test = [&](const float val) {  // val < 1 with its margin
        if (val < 1.0f - margin) return true;
        if (!(val > 1.0f + margin)) unclear = true;
        return false;
    };
    // rect centre in the ellipse
    if (test(len2(ax + 0.5f * (ux + vx), ay + 0.5f * (uy + vy)))) return 1;
    // the edges: the point of segment p + t d (t in [0, 1]) nearest the
    // origin.  Of two parallel edges only the nearer line's is needed: both
    // span the same range along their direction, so the farther one's
    // squared length is the nearer one's plus the difference of the squared
    // line distances.  Where the nearer edge's value lies clearly above 1,
    // the farther edge's does too; where the two are nearly equally far,
    // either gives nearly the same value.
    const float iu = rcp_approx(len2(ux, uy)), iv = rcp_approx(len2(vx, vy));
    auto edge = [](const float px, const float py, const float dx, const float dy, const float inv) {
        const float t = __saturatef(-(px * dx + py * dy) * inv);
        return len2(px + t * dx, py + t * dy);
    };
    // u edges through a (x0, y0) and a + v (x0, y1); v edges through a and
    // a + u (x1, y0): compare the lines' distances by cross products
    const float su = ax * uy - ay * ux, kuv = vx * uy - vy * ux, sv = ax * vy - ay * vx;
    const bool u_at_a = fabsf(su) <= fabsf(su + kuv);
    const bool v_at_a = fabsf(sv) <= fabsf(sv - kuv);
    if (test(edge(u_at_a ? ax : ax + vx, u_at_a ? ay : ay + vy, ux, uy, iu))) return 1;
    if (test(edge(v_at_a ? ax : ax + ux, v_at_a ? ay : ay + uy, vx, vy, iv))) return 1;
    return unclear ? -1 : 0;
}

struct RectF {
    float x0, y0, x1, y1;
};

__device__ __forceinline__ RectF aabb_rect(const Ell& e)
{
    const float rxx = e.cs * e.ex, rxy = e.sn * e.ex;   // principal axis
    const float uxx = e.sn * e.ey, uxy = -e.cs * e.ey;  // minor axis
    RectF r;
    r.x0 = 1e12f;
    r.y0 = 1e12f;
    r.x1 = -1e12f;
    r.y1 = -1e12f;
#pragma unroll
    for (int j = 0; j != 4; ++j) {
        const int bottomBit = j & 1;
        const int topBit = j >> 1;
        const float sr = (bottomBit ^ topBit) * 2.0f - 1.0f;
        const float su = (topBit) * 2.0f - 1.0f;
        const float vx = rxx * sr + uxx * su;
        const float vy = rxy * sr + uxy * su;
        r.x0 = gmin(r.x0, vx);
        r.y0 = gmin(r.y0, vy);
        r.x1 = gmax(r.x1, vx);
        r.y1 = gmax(r.y1, vy);
    }
    r.x0 += e.cx;
    r.y0 += e.cy;
    r.x1 += e.cx;
    r.y1 += e.cy;
    return r;
}

// Tile rectangle (x0, y0, w, h) of an ellipse (gaussian_render.cu:377-389).
__device__ __forceinline__ int4 tile_rect(const Ell& e, const ViewParams& v)
{
    const RectF a = aabb_rect(e);
    const float fx0 = (a.x0 + 1.0f) * 0.5f * v.tiles_xf;
    const float fy0 = (a.y0 + 1.0f) * 0.5f * v.tiles_yf;
    const float fx1 = (a.x1 + 1.0f) * 0.5f * v.tiles_xf;
    const float fy1 = (a.y1 + 1.0f) * 0.5f * v.tiles_yf;
    const int x0 = iclamp((int32_t)floorf(fx0), 0, v.tiles_x);
    const int y0 = iclamp((int32_t)floorf(fy0), 0, v.tiles_y);
    const int x1 = iclamp((int32_t)ceilf(fx1), 0, v.tiles_x);
    const int y1 = iclamp((int32_t)ceilf(fy1), 0, v.tiles_y);
    return make_int4(x0, y0, x1 - x0, y1 - y0);
}

__device__ __forceinline__ int rect_candidates(const int4 r) { return imax(0, r.z * r.w); }

// C's quotient and remainder of c / d for c >= 0.  For d >= 1 and
// c < 2^20 a float estimate (the hardware reciprocal is within a few ulp, so
// the estimate is within 1 of the quotient) and one correction step either
// way: exact, and shorter than the integer division sequence.  Larger c,
// and d <= 0 (the inverted rectangles of NaN axes), take the integer
// division.
__device__ __forceinline__ void divmod_small(const int c, const int d, int& q, int& r)
{
    if (d <= 0 || c >= (1 << 20)) {
        q = c / d;
        r = c % d;
        return;
    }
    int qq = (int)(__int2float_rn(c) * rcp_approx(__int2float_rn(d)));
    int rr = c - qq * d;
    if (rr < 0) {
        --qq;
        rr += d;
    } else if (rr >= d) {
        ++qq;
        rr -= d;
    }
    q = qq;
    r = rr;
}

// Clip-space rectangle of tile (gx, gy) (gaussian_render.cu:471-473).
__device__ __forceinline__ void tile_clip_rect(const ViewParams& v, const int gx, const int gy, float& x0, float& y0,
                                               float& x1, float& y1)
{
    x0 = (float)gx * v.tclip_x - 1.0f;
    y0 = (float)gy * v.tclip_y - 1.0f;
    x1 = x0 + v.tclip_x;
    y1 = y0 + v.tclip_y;
}

// Candidate c of a tile rectangle, row-major (gaussian_render.cu:466-483),
// tested without the IEEE evaluation: 1 = overlap, 0 = none, -1 = too close
// to call (candidate_hit_ieee decides).  Sets the view-local tile index
// whenever the candidate lies on screen.  Off-screen candidates only arise
// from the inverted rectangles of NaN axes; their centre test cannot pass
// for a visible splat, so they never overlap.
__device__ __forceinline__ int candidate_state(const Ell& e, const int4 r, const int c, const ViewParams& v, int& tile)
{
    int lx, ly;
    divmod_small(c, r.z, ly, lx);
    const int gx = r.x + lx, gy = r.y + ly;
    if (gx < 0 || gx >= v.tiles_x || gy < 0 || gy >= v.tiles_y) return 0;
    tile = gy * v.tiles_x + gx;
    float x0, y0, x1, y1;
    tile_clip_rect(v, gx, gy, x0, y0, x1, y1);
    if (e.cx > x0 && e.cx < x1 && e.cy > y0 && e.cy < y1) return 1;  // centre in the tile decides
    return ellipse_rect_overlap_clear(e, x0, y0, x1, y1);
}

// The IEEE decision of a candidate that candidate_state could not call.
__device__ __forceinline__ bool candidate_hit_ieee(const Ell& e, const int tile, const ViewParams& v)
{
    float x0, y0, x1, y1;
    tile_clip_rect(v, tile % v.tiles_x, tile / v.tiles_x, x0, y0, x1, y1);
    return ellipse_rect_overlap_ieee(e, x0, y0, x1, y1);
}

// Candidate c of a tile rectangle: true on overlap (exactly the reference's
// test), with the view-local tile index.
__device__ __forceinline__ bool candidate_hit(const Ell& e, const int4 r, const int c, const ViewParams& v, int& tile)
{
    const int st = candidate_state(e, r, c, v, tile);
    if (st >= 0) return st != 0;
    return candidate_hit_ieee(e, tile, v);
}

// getKey (gaussian_render.cu:306-310): tile << 32 | quantised depth.
__device__ __forceinline__ uint64_t make_key(const uint64_t tile, const float depth)
{
    const uint32_t q = (uint32_t)(gclamp((depth + 1.0f) * 0.5f, 0.0f, 1.0f) * 0xffffffffu);
    return (tile << 32) | q;
}

// Packs a tile rectangle into 8 bytes (x0, y0 unsigned; w, h signed 16-bit).
__device__ __forceinline__ int2 pack_rect(const int4 r)
{
    return make_int2((r.x & 0xFFFF) | (r.y << 16), (r.z & 0xFFFF) | (r.w << 16));
}
__device__ __forceinline__ int4 unpack_rect(const int2 p)
{
    return make_int4(p.x & 0xFFFF, (int)((unsigned)p.x >> 16), (int)(short)(p.y & 0xFFFF), p.y >> 16);
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- TMA bulk copy global -> shared (cp.async.bulk, no tensor map) ---------

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arms the barrier for `bytes` and starts one bulk copy completing on it.
// dst, src and bytes must be multiples of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// ---- bounded decoupled look-back ------------------------------------------
// Status word: bit 63 = inclusive prefix available, bit 62 = block
// aggregate available, bits 46..61 = epoch, bits 0..45 = value.  Every
// launch uses a fresh epoch, so words left by earlier launches read as
// "not yet published" and the status arrays never need clearing (the host
// clears them once when the 16-bit epoch wraps).
constexpr uint64_t kFlagP = 1ull << 63;
constexpr uint64_t kFlagA = 1ull << 62;
constexpr int kEpochShift = 46;
constexpr uint64_t kEpochMask = 0xFFFFull << kEpochShift;
constexpr uint64_t kValueMask = (1ull << kEpochShift) - 1;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ uint64_t status_word(const uint64_t flag, const uint32_t epoch, const uint64_t value)
{
    return flag | ((uint64_t)(epoch & 0xFFFFu) << kEpochShift) | (value & kValueMask);
}

__device__ __forceinline__ void store_status(uint64_t* p, const uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t load_status(const uint64_t* p)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int load_flag(const int* p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Exclusive prefix of `tile`'s aggregate over all earlier tiles, walking
// back through status[tile-1], status[tile-2], ... (`stride` words apart).
// Gives up after kSpinLimit polls, or as soon as another block has
// reported an error, setting *err; the result is then meaningless and the
// host discards the frame.
__device__ __forceinline__ uint64_t look_back(const uint64_t* status, const int64_t tile, const int64_t stride,
                                              const uint32_t epoch, int* err, const int err_code,
                                              const int spin_limit = kSpinLimit)
{
    const uint64_t want = (uint64_t)(epoch & 0xFFFFu) << kEpochShift;
    uint64_t excl = 0;
    int64_t j = tile - 1;
    int spins = 0;
    while (j >= 0) {
        const uint64_t s = load_status(status + j * stride);
        if ((s & (kFlagP | kFlagA)) == 0 || (s & kEpochMask) != want) {
            if (++spins > spin_limit || load_flag(err) != 0) {
                atomicCAS(err, 0, err_code);
                return excl;
            }
            if (spins > 64) __nanosleep(32);
            continue;
        }
        excl += s & kValueMask;
        if (s & kFlagP) break;
        --j;
    }
    return excl;
}

}  // namespace gs
