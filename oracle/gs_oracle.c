/*
 * CPU ORACLE (test infrastructure only; see gs_oracle.h).
 *
 * Plain-C restatement of RobinSongx/3DGaussianRenderer's frame pipeline,
 * core/gaussian_render.cu.  Each function cites the reference lines it
 * follows.  Compiled with -ffp-contract=off so that every fused
 * multiply-add below is an explicit fmaf() chosen by the fma mode.
 */
#include "gs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_fma = 1;

void gso_set_fma_mode(int mode) { g_fma = mode; }
int gso_get_fma_mode(void) { return g_fma; }

void gso_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int gso_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- contraction model ------------------------------------------------ */

/* a*b + c */
static inline float mad(float a, float b, float c) { return g_fma ? fmaf(a, b, c) : a * b + c; }
/* a*b + c*d */
static inline float mad2(float a, float b, float c, float d)
{
    if (g_fma == 1) return fmaf(a, b, c * d);
    if (g_fma == 2) return fmaf(c, d, a * b);
    return a * b + c * d;
}
/* a*b - c*d */
static inline float msub2(float a, float b, float c, float d)
{
    if (g_fma == 1) return fmaf(a, b, -(c * d));
    if (g_fma == 2) return fmaf(-c, d, a * b);
    return a * b - c * d;
}
/* (a*b + c*d) + e*f */
static inline float mad3(float a, float b, float c, float d, float e, float f)
{
    if (g_fma) return fmaf(e, f, mad2(a, b, c, d));
    return (a * b + c * d) + e * f;
}

/* glm 0.9.9 scalar semantics (detail/func_common.inl:17-30) */
static inline float gmin(float x, float y) { return (y < x) ? y : x; }
static inline float gmax(float x, float y) { return (x < y) ? y : x; }
static inline float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
static inline int imin(int x, int y) { return (y < x) ? y : x; }
static inline int imax(int x, int y) { return (x < y) ? y : x; }
static inline int iclamp(int x, int lo, int hi) { return imin(imax(x, lo), hi); }

/* Device float->int32 conversion (cvt.rzi.s32.f32): truncate, saturate, NaN -> 0. */
static inline int32_t cvt_s32(float x)
{
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)x;
}
/* Device float->uint32 conversion: truncate, saturate, NaN -> 0. */
static inline uint32_t cvt_u32(float x)
{
    if (x != x || x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
/* float -> unsigned char as the reference's uchar4 store (gaussian_render.cu:752-754).
 * Mode 0: truncate and saturate to [0,255]; 1: truncate to int32 (saturating), keep
 * the low byte; 2: truncate to uint32 (negatives -> 0, saturating), keep the low byte.
 * The reference's kernels do 2 (pinned by the out-of-range-colour golden frame):
 * a colour of 256/255 stores 0, not 255. */
static int g_u8 = 2;
void gso_set_u8_mode(int mode) { g_u8 = mode; }
static inline uint8_t cvt_u8(float x)
{
    if (g_u8 == 1) return (uint8_t)((uint32_t)cvt_s32(x) & 0xFFu);
    if (g_u8 == 2) return (uint8_t)(cvt_u32(x) & 0xFFu);
    if (x != x || x <= 0.0f) return 0;
    if (x >= 255.0f) return 255;
    return (uint8_t)x;
}
/* __saturatef: clamp to [0,1], NaN -> 0 */
static inline float saturate(float x)
{
    if (x != x) return 0.0f;
    return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
}

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

/* ---- SH (core/gaussian_render.cu:50-116; deg 3: core/cuda_renderer.cu:119-156) */

static void sh_color(int degree, float x, float y, float z, const float* sh, int stride, float out[3])
{
    float r[3];
    for (int c = 0; c < 3; ++c) r[c] = 0.282094792f * sh[c * stride];
    if (degree > 0) {
        for (int c = 0; c < 3; ++c) {
            float s1 = sh[(3 + c) * stride], s2 = sh[(6 + c) * stride], s3 = sh[(9 + c) * stride];
            r[c] = r[c] + (((0.488602512f * y) * s1 + (0.488602512f * z) * s2) + (0.488602512f * x) * s3);
        }
        if (degree > 1) {
            float xx = x * x, yy = y * y;
            float b4 = 1.09254843f * x * y;
            float b5 = 1.09254843f * y * z;
            float b6 = -0.946174696f * xx - 0.946174696f * yy + 0.630783131f;
            float b7 = 1.09254843f * x * z;
            float b8 = 0.546274215f * (x - y) * (x + y);
            for (int c = 0; c < 3; ++c) {
                r[c] = r[c] + ((((b4 * sh[(12 + c) * stride] + b5 * sh[(15 + c) * stride]) + b6 * sh[(18 + c) * stride]) +
                                b7 * sh[(21 + c) * stride]) +
                               b8 * sh[(24 + c) * stride]);
            }
            if (degree > 2) {
                float b9 = 0.295021795f * y * (6.0f * xx - 2.0f * yy);
                float b10 = 2.89061144f * x * y * z;
                float b11 = 3.6563664f * y * (-0.625f * xx - 0.625f * yy + 0.5f);
                float b12 = 0.373176333f * z * (-5.0f * xx - 5.0f * yy + 2.0f);
                float b13 = 0.457045799f * x * (-5.0f * xx - 5.0f * yy + 4.0f);
                float b14 = 1.44530572f * z * (x - y) * (x + y);
                float b15 = 0.59004359f * x * (xx - 3.0f * yy);
                for (int c = 0; c < 3; ++c) {
                    r[c] = r[c] + ((((((b9 * sh[(27 + c) * stride] + b10 * sh[(30 + c) * stride]) +
                                       b11 * sh[(33 + c) * stride]) +
                                      b12 * sh[(36 + c) * stride]) +
                                     b13 * sh[(39 + c) * stride]) +
                                    b14 * sh[(42 + c) * stride]) +
                                   b15 * sh[(45 + c) * stride]);
                }
            }
        }
    }
    for (int c = 0; c < 3; ++c) out[c] = gclamp(r[c] + 0.5f, 0.0f, 1.0f);
}

void gso_sh(int64_t n, const float* pos4, const float* sh, int32_t sh_count, int32_t eval_degree,
            const float cam_pos[3], float* color4)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        float px = pos4[4 * i], py = pos4[4 * i + 1], pz = pos4[4 * i + 2];
        float dx = cam_pos[0] - px, dy = cam_pos[1] - py, dz = cam_pos[2] - pz;
        /* glm::normalize: v * (1 / sqrt(dot(v, v))) */
        float d2 = (dx * dx + dy * dy) + dz * dz;
        float inv = 1.0f / sqrtf(d2);
        float x = dx * inv, y = dy * inv, z = dz * inv;
        int64_t g = i / 256, t = i % 256;
        const float* base = sh + (g * 256 * (int64_t)sh_count) + t;
        float rgb[3];
        sh_color(eval_degree, x, y, z, base, 256, rgb);
        color4[4 * i] = rgb[0];
        color4[4 * i + 1] = rgb[1];
        color4[4 * i + 2] = rgb[2];
        color4[4 * i + 3] = pos4[4 * i + 3];
    }
}

/* ---- projection (core/gaussian_render.cu:135-215) ---------------------- */

/* glm mat3 * mat3 (detail/type_mat3x3.inl:486-520): R[i][j] = A0j*Bi0 + A1j*Bi1 + A2j*Bi2 */
static void mat3_mul(const float A[3][3], const float B[3][3], float R[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = mad3(A[0][j], B[i][0], A[1][j], B[i][1], A[2][j], B[i][2]);
}

static void mat3_transpose(const float A[3][3], float R[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = A[j][i];
}

/* glm mat4 * vec4(v, 1) (detail/type_mat4x4.inl:536-570):
 * (m0*x + m1*y) + (m2*z + m3)   [the multiply by the constant 1 folds away] */
static float mat4_row_xyz1(const float m0, const float m1, const float m2, const float m3, float x, float y,
                           float z)
{
    float a0 = mad2(m0, x, m1, y);
    float a1 = mad(m2, z, m3);
    return a0 + a1;
}

static void project_one(const float* p4, const float* sr4, const gso_camera* cam, float k_bump_x, float k_bump_y,
                        float* xy, float* zout, float* ell, float* con)
{
    float px = p4[0], py = p4[1], pz = p4[2];
    float sx = sr4[0], sy = sr4[1], sz = sr4[2];
    uint32_t bits;
    memcpy(&bits, &sr4[3], 4);
    /* decodeVec4 (:45-48) then *2-1 (:150) */
    float q[4];
    for (int c = 0; c < 4; ++c) {
        float b = (float)((bits >> (24 - 8 * c)) & 0xFFu) / 255.0f;
        q[c] = mad(b, 2.0f, -1.0f);
    }
    float qx = q[0], qy = q[1], qz = q[2], qw = q[3]; /* glm::quat(w=rv.w, x, y, z) */

    /* glm::mat3_cast (gtc/quaternion.inl:41-66) */
    float qxx = qx * qx, qyy = qy * qy, qzz = qz * qz;
    float qxz = qx * qz, qxy = qx * qy, qyz = qy * qz;
    float qwx = qw * qx, qwy = qw * qy, qwz = qw * qz;
    (void)qxx;
    float R[3][3];
    R[0][0] = 1.0f - 2.0f * (qy * qy + qz * qz);
    R[0][1] = 2.0f * (qx * qy + qw * qz);
    R[0][2] = 2.0f * (qx * qz - qw * qy);
    R[1][0] = 2.0f * (qx * qy - qw * qz);
    R[1][1] = 1.0f - 2.0f * (qx * qx + qz * qz);
    R[1][2] = 2.0f * (qy * qz + qw * qx);
    R[2][0] = 2.0f * (qx * qz + qw * qy);
    R[2][1] = 2.0f * (qy * qz - qw * qx);
    R[2][2] = 1.0f - 2.0f * (qx * qx + qy * qy);
    if (g_fma) {
        R[0][0] = 1.0f - 2.0f * mad2(qy, qy, qz, qz);
        R[0][1] = 2.0f * mad2(qx, qy, qw, qz);
        R[0][2] = 2.0f * msub2(qx, qz, qw, qy);
        R[1][0] = 2.0f * msub2(qx, qy, qw, qz);
        R[1][1] = 1.0f - 2.0f * mad2(qx, qx, qz, qz);
        R[1][2] = 2.0f * mad2(qy, qz, qw, qx);
        R[2][0] = 2.0f * mad2(qx, qz, qw, qy);
        R[2][1] = 2.0f * msub2(qy, qz, qw, qx);
        R[2][2] = 1.0f - 2.0f * mad2(qx, qx, qy, qy);
    } else {
        R[0][0] = 1.0f - 2.0f * (qyy + qzz);
        R[0][1] = 2.0f * (qxy + qwz);
        R[0][2] = 2.0f * (qxz - qwy);
        R[1][0] = 2.0f * (qxy - qwz);
        R[1][1] = 1.0f - 2.0f * (qx * qx + qzz);
        R[1][2] = 2.0f * (qyz + qwx);
        R[2][0] = 2.0f * (qxz + qwy);
        R[2][1] = 2.0f * (qyz - qwx);
        R[2][2] = 1.0f - 2.0f * (qx * qx + qyy);
    }

    /* RS = R * diag(s): column i scaled by s_i (the zero products add exact zeros) */
    float S[3] = {sx, sy, sz};
    float RS[3][3], RSt[3][3], Cov[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) RS[i][j] = R[i][j] * S[i];
    mat3_transpose(RS, RSt);
    mat3_mul(RS, RSt, Cov);

    const float* V = cam->view; /* column-major: V[c*4 + r] */
    float vx = mat4_row_xyz1(V[0], V[4], V[8], V[12], px, py, pz);
    float vy = mat4_row_xyz1(V[1], V[5], V[9], V[13], px, py, pz);
    float vz = mat4_row_xyz1(V[2], V[6], V[10], V[14], px, py, pz);

    float cotx = cam->fov_cotangent[0], coty = cam->fov_cotangent[1];
    float dsbx = cam->depth_scale_bias[0], dsby = cam->depth_scale_bias[1];
    float zRcp = 1.0f / vz;
    float zRcpSqr = zRcp * zRcp;
    float scaleX = -cotx * zRcp;
    float scaleY = -coty * zRcp;
    float fx = cotx * vx, fy = coty * vy;
    float shearX = fx * zRcpSqr;
    float shearY = fy * zRcpSqr;
    float trX = -fx * zRcp;
    float trY = -fy * zRcp;

    /* mat3(affine) * mat3(view) (:180) with A = [[sX,0,0],[0,sY,0],[shX,shY,dsbx]] (columns) */
    float A[3][3] = {{scaleX, 0.0f, 0.0f}, {0.0f, scaleY, 0.0f}, {shearX, shearY, dsbx}};
    float B[3][3];
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) B[c][r] = V[c * 4 + r];
    float VP[3][3], VPt[3][3], CovT[3][3], T1[3][3], CC[3][3];
    mat3_mul(A, B, VP);
    mat3_transpose(Cov, CovT);
    mat3_transpose(VP, VPt);
    mat3_mul(VP, CovT, T1);
    mat3_mul(T1, VPt, CC);

    /* clip position: affine * vec4(viewPosition, 1) */
    float cx = mat4_row_xyz1(scaleX, 0.0f, shearX, trX, vx, vy, vz);
    float cy = mat4_row_xyz1(0.0f, scaleY, shearY, trY, vx, vy, vz);
    float cz = mat4_row_xyz1(0.0f, 0.0f, dsbx, dsby, vx, vy, vz);

    float c00 = CC[0][0] + k_bump_x;
    float c11 = CC[1][1] + k_bump_y;
    float c10 = CC[1][0];

    float det = msub2(c00, c11, c10, c10);
    float mid = 0.5f * (c00 + c11);
    const float eps = 1e-12f;
    float radius = sqrtf(gmax(eps, g_fma ? fmaf(mid, mid, -det) : mid * mid - det));
    float lambda0 = mid + radius;
    float lambda1 = gmax(0.0f, mid - radius);

    float e0x = c10, e0y = lambda0 - c00;
    float dd = mad2(e0x, e0x, e0y, e0y);
    float inv = 1.0f / sqrtf(dd);
    e0x = e0x * inv;
    e0y = e0y * inv;
    float angle = atan2f(e0y, e0x);
    float ex = sqrtf(lambda0) * 3.0f;
    float ey = sqrtf(lambda1) * 3.0f;
    float invDet = 1.0f / gmax(eps, det);
    float ka = c11 * invDet, kb = -c10 * invDet, kc = c00 * invDet;

    /* visibility (:205-208): step(-1, clip) * step(clip, 1) * step(0, lambda1) */
    float ex_ = (cx < -1.0f ? 0.0f : 1.0f) * (1.0f < cx ? 0.0f : 1.0f);
    float ey_ = (cy < -1.0f ? 0.0f : 1.0f) * (1.0f < cy ? 0.0f : 1.0f);
    float ez_ = (cz < -1.0f ? 0.0f : 1.0f) * (1.0f < cz ? 0.0f : 1.0f);
    float vis = ((ex_ * ey_) * ez_) * (lambda1 < 0.0f ? 0.0f : 1.0f);
    /* mix(vec3(-128), clip, vis) = -128*(1-vis) + clip*vis */
    float om = 1.0f - vis;
    cx = mad2(-128.0f, om, cx, vis);
    cy = mad2(-128.0f, om, cy, vis);
    cz = mad2(-128.0f, om, cz, vis);
    ex *= vis;
    ey *= vis;

    xy[0] = cx;
    xy[1] = cy;
    *zout = cz;
    ell[0] = cosf(angle);
    ell[1] = sinf(angle);
    ell[2] = ex;
    ell[3] = ey;
    con[0] = ka;
    con[1] = kb;
    con[2] = kc;
    con[3] = 0.0f;
}

/* The trace bump (:184-188) uses the fixed 1024-pixel screen; a W x H
 * frame uses the texel size of each axis (identical at 1024x1024). */
static void trace_bump(const gso_camera* cam, float* bx, float* by)
{
    const float k_Pi = 3.14159265359f;
    float tx = 2.0f / (float)cam->width;
    float ty = 2.0f / (float)cam->height;
    *bx = ((1.0f / k_Pi) * tx) * tx;
    *by = ((1.0f / k_Pi) * ty) * ty;
}

void gso_project(int64_t n, const float* pos4, const float* scale_rot4, const gso_camera* cam, float* xy,
                 float* z, float* ellipse4, float* conic4)
{
    float bx, by;
    trace_bump(cam, &bx, &by);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        project_one(pos4 + 4 * i, scale_rot4 + 4 * i, cam, bx, by, xy + 2 * i, z + i, ellipse4 + 4 * i,
                    conic4 + 4 * i);
}

/* ---- ellipse / rect helpers (core/gaussian_render.cu:234-310) ---------- */

typedef struct { float cx, cy, cs, sn, ex, ey; } ellipse_t;
typedef struct { float x0, y0, x1, y1; } rect_t;

static inline void to_ellipse(const ellipse_t* e, float px, float py, float* ox, float* oy)
{
    float dx = px - e->cx, dy = py - e->cy;
    *ox = mad2(dx, e->cs, dy, e->sn) / e->ex;
    *oy = msub2(dy, e->cs, dx, e->sn) / e->ey;
}

static inline float len2(float x, float y) { return mad2(x, x, y, y); }

static inline int hits_unit_circle(float v0x, float v0y, float v1x, float v1y)
{
    float dx = v1x - v0x, dy = v1y - v0y;
    float l2 = len2(dx, dy);
    float t = saturate(mad2(-v0x, dx, -v0y, dy) / l2);
    float prx = mad(t, dx, v0x);
    float pry = mad(t, dy, v0y);
    return len2(prx, pry) < 1.0f;
}

static int ellipse_rect_overlap(const ellipse_t* e, const rect_t* r)
{
    int ov = e->cx > r->x0 && e->cx < r->x1 && e->cy > r->y0 && e->cy < r->y1;
    /* Rect::getCenter: min + (max - min) * 0.5 */
    float rcx = mad(r->x1 - r->x0, 0.5f, r->x0);
    float rcy = mad(r->y1 - r->y0, 0.5f, r->y0);
    float ux, uy;
    to_ellipse(e, rcx, rcy, &ux, &uy);
    ov |= len2(ux, uy) < 1.0f;
    float p[4][2];
    to_ellipse(e, r->x0, r->y0, &p[0][0], &p[0][1]);
    to_ellipse(e, r->x1, r->y0, &p[1][0], &p[1][1]);
    to_ellipse(e, r->x1, r->y1, &p[2][0], &p[2][1]);
    to_ellipse(e, r->x0, r->y1, &p[3][0], &p[3][1]);
    ov |= hits_unit_circle(p[0][0], p[0][1], p[1][0], p[1][1]);
    ov |= hits_unit_circle(p[1][0], p[1][1], p[2][0], p[2][1]);
    ov |= hits_unit_circle(p[2][0], p[2][1], p[3][0], p[3][1]);
    ov |= hits_unit_circle(p[3][0], p[3][1], p[0][0], p[0][1]);
    return ov;
}

static rect_t aabb_rect(const ellipse_t* e)
{
    float rx = e->cs * e->ex, ry = e->sn * e->ex;    /* principal axis */
    float ux = e->sn * e->ey, uy = -e->cs * e->ey;   /* minor axis */
    rect_t r = {1e12f, 1e12f, -1e12f, -1e12f};
    for (int j = 0; j < 4; ++j) {
        int bb = j & 1, tb = j >> 1;
        float sr = (float)(bb ^ tb) * 2.0f - 1.0f;
        float su = (float)tb * 2.0f - 1.0f;
        /* right*r + up*u: nvcc keeps the principal-axis product unrounded,
         * fma(cos*r, extent.x, round(sin*extent.y)*u) (pinned by the probes) */
        float vx = g_fma ? fmaf(e->cs * sr, e->ex, ux * su) : rx * sr + ux * su;
        float vy = g_fma ? fmaf(e->sn * sr, e->ex, uy * su) : ry * sr + uy * su;
        r.x0 = gmin(r.x0, vx);
        r.y0 = gmin(r.y0, vy);
        r.x1 = gmax(r.x1, vx);
        r.y1 = gmax(r.y1, vy);
    }
    r.x0 += e->cx;
    r.y0 += e->cy;
    r.x1 += e->cx;
    r.y1 += e->cy;
    return r;
}

static inline uint64_t make_key(int32_t tile, float depth)
{
    float q = gclamp((depth + 1.0f) * 0.5f, 0.0f, 1.0f) * 4294967296.0f;
    return ((uint64_t)(uint32_t)tile << 32) | (uint64_t)cvt_u32(q);
}

void gso_aabb(int64_t n, const float* ell6, float* rect4)
{
    for (int64_t i = 0; i < n; ++i) {
        ellipse_t e = {ell6[6 * i], ell6[6 * i + 1], ell6[6 * i + 2], ell6[6 * i + 3], ell6[6 * i + 4], ell6[6 * i + 5]};
        rect_t r = aabb_rect(&e);
        rect4[4 * i] = r.x0;
        rect4[4 * i + 1] = r.y0;
        rect4[4 * i + 2] = r.x1;
        rect4[4 * i + 3] = r.y1;
    }
}

void gso_overlap(int64_t n, const float* ell6, const float* rect4, int32_t* out)
{
    for (int64_t i = 0; i < n; ++i) {
        ellipse_t e = {ell6[6 * i], ell6[6 * i + 1], ell6[6 * i + 2], ell6[6 * i + 3], ell6[6 * i + 4], ell6[6 * i + 5]};
        rect_t r = {rect4[4 * i], rect4[4 * i + 1], rect4[4 * i + 2], rect4[4 * i + 3]};
        out[i] = ellipse_rect_overlap(&e, &r);
    }
}

void gso_key(int64_t n, const int32_t* tile, const float* depth, uint64_t* out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = make_key(tile[i], depth[i]);
}

/* ---- tile geometry ------------------------------------------------------ */

typedef struct {
    int tiles_x, tiles_y;
    float tiles_xf, tiles_yf;     /* W / tile_w, H / tile_h as float (64 at 1024/16) */
    float tclip_x, tclip_y;       /* (tile_w / W) * 2 (0.03125 at 1024/16) */
} tilegeo_t;

static tilegeo_t tile_geo(const gso_camera* cam, const gso_cfg* cfg)
{
    tilegeo_t g;
    g.tiles_x = (cam->width + cfg->tile_w - 1) / cfg->tile_w;
    g.tiles_y = (cam->height + cfg->tile_h - 1) / cfg->tile_h;
    g.tiles_xf = (float)cam->width / (float)cfg->tile_w;
    g.tiles_yf = (float)cam->height / (float)cfg->tile_h;
    g.tclip_x = ((float)cfg->tile_w / (float)cam->width) * 2.0f;
    g.tclip_y = ((float)cfg->tile_h / (float)cam->height) * 2.0f;
    return g;
}

/* :377-389 */
static void tile_rect(const ellipse_t* e, const tilegeo_t* g, int32_t r[4])
{
    rect_t a = aabb_rect(e);
    float fx0 = ((a.x0 + 1.0f) * 0.5f) * g->tiles_xf;
    float fy0 = ((a.y0 + 1.0f) * 0.5f) * g->tiles_yf;
    float fx1 = ((a.x1 + 1.0f) * 0.5f) * g->tiles_xf;
    float fy1 = ((a.y1 + 1.0f) * 0.5f) * g->tiles_yf;
    int x0 = iclamp(cvt_s32(floorf(fx0)), 0, g->tiles_x);
    int y0 = iclamp(cvt_s32(floorf(fy0)), 0, g->tiles_y);
    int x1 = iclamp(cvt_s32(ceilf(fx1)), 0, g->tiles_x);
    int y1 = iclamp(cvt_s32(ceilf(fy1)), 0, g->tiles_y);
    r[0] = x0;
    r[1] = y0;
    r[2] = x1 - x0;
    r[3] = y1 - y0;
}

/* Candidate c of a rectangle (:466-476): row-major, C integer division
 * semantics (the width can be negative for the inverted rectangles that a
 * NaN ellipse axis produces). Returns 1 and the tile on a hit. */
static inline int candidate_hit(const ellipse_t* e, const int32_t r[4], int c, const tilegeo_t* g, int32_t* tile)
{
    int lx = c % r[2], ly = c / r[2];
    int gx = r[0] + lx, gy = r[1] + ly;
    rect_t tr;
    tr.x0 = mad((float)gx, g->tclip_x, -1.0f);
    tr.y0 = mad((float)gy, g->tclip_y, -1.0f);
    tr.x1 = tr.x0 + g->tclip_x;
    tr.y1 = tr.y0 + g->tclip_y;
    if (!ellipse_rect_overlap(e, &tr)) return 0;
    if (gx < 0 || gx >= g->tiles_x || gy < 0 || gy >= g->tiles_y) return 0; /* never reached by visible splats */
    *tile = gy * g->tiles_x + gx;
    return 1;
}

static inline void load_ellipse(ellipse_t* e, const float* xy, const float* ell4, int64_t i)
{
    e->cx = xy[2 * i];
    e->cy = xy[2 * i + 1];
    e->cs = ell4[4 * i];
    e->sn = ell4[4 * i + 1];
    e->ex = ell4[4 * i + 2];
    e->ey = ell4[4 * i + 3];
}

void gso_tile_counts(int64_t n, const float* xy, const float* ellipse4, const gso_camera* cam,
                     const gso_cfg* cfg, int32_t* rect4, int32_t* cand, int32_t* hits)
{
    tilegeo_t g = tile_geo(cam, cfg);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; ++i) {
        ellipse_t e;
        load_ellipse(&e, xy, ellipse4, i);
        int32_t r[4];
        tile_rect(&e, &g, r);
        int count = imax(0, r[2] * r[3]);
        if (rect4) memcpy(rect4 + 4 * i, r, sizeof(r));
        if (cand) cand[i] = count;
        if (hits) {
            int h = 0;
            int32_t t;
            for (int c = 0; c < count; ++c) h += candidate_hit(&e, r, c, &g, &t);
            hits[i] = h;
        }
    }
}

int64_t gso_build(int64_t n, const float* xy, const float* ellipse4, const float* z, const gso_camera* cam,
                  const gso_cfg* cfg, uint64_t* keys, int32_t* values, int64_t capacity)
{
    tilegeo_t g = tile_geo(cam, cfg);
    int32_t* hits = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    gso_tile_counts(n, xy, ellipse4, cam, cfg, NULL, NULL, hits);
    int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    off[0] = 0;
    for (int64_t i = 0; i < n; ++i) off[i + 1] = off[i] + hits[i];
    int64_t K = off[n];
    if (keys && values) {
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; ++i) {
            if (hits[i] == 0) continue;
            ellipse_t e;
            load_ellipse(&e, xy, ellipse4, i);
            int32_t r[4];
            tile_rect(&e, &g, r);
            int count = imax(0, r[2] * r[3]);
            int64_t o = off[i];
            for (int c = 0; c < count; ++c) {
                int32_t t;
                if (candidate_hit(&e, r, c, &g, &t)) {
                    if (o < capacity) {
                        keys[o] = make_key(t, z[i]);
                        values[o] = (int32_t)i;
                    }
                    ++o;
                }
            }
        }
    }
    free(off);
    free(hits);
    return K;
}

/* ---- sort: stable LSD radix, 8-bit digits -------------------------------- */

void gso_sort(int64_t k, uint64_t* keys, int32_t* values, int32_t key_bits)
{
    if (k <= 1) return;
    uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)k);
    int32_t* v2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)k);
    int nthreads = gso_max_threads();
    int64_t* hist = (int64_t*)malloc(sizeof(int64_t) * 256 * (size_t)nthreads);
    uint64_t *src = keys, *dst = k2;
    int32_t *vsrc = values, *vdst = v2;
    for (int shift = 0; shift < key_bits; shift += 8) {
        memset(hist, 0, sizeof(int64_t) * 256 * (size_t)nthreads);
#pragma omp parallel num_threads(nthreads)
        {
#ifdef _OPENMP
            int t = omp_get_thread_num();
            int nt = omp_get_num_threads();
#else
            int t = 0, nt = 1;
#endif
            int64_t lo = k * t / nt, hi = k * (t + 1) / nt;
            int64_t* h = hist + 256 * t;
            for (int64_t i = lo; i < hi; ++i) h[(src[i] >> shift) & 0xFF]++;
#pragma omp barrier
#pragma omp single
            {
                int64_t run = 0;
                for (int d = 0; d < 256; ++d)
                    for (int tt = 0; tt < nt; ++tt) {
                        int64_t c = hist[256 * tt + d];
                        hist[256 * tt + d] = run;
                        run += c;
                    }
            }
            for (int64_t i = lo; i < hi; ++i) {
                int64_t p = h[(src[i] >> shift) & 0xFF]++;
                dst[p] = src[i];
                vdst[p] = vsrc[i];
            }
        }
        uint64_t* tk = src; src = dst; dst = tk;
        int32_t* tv = vsrc; vsrc = vdst; vdst = tv;
    }
    if (src != keys) {
        memcpy(keys, src, sizeof(uint64_t) * (size_t)k);
        memcpy(values, vsrc, sizeof(int32_t) * (size_t)k);
    }
    free(hist);
    free(k2);
    free(v2);
}

/* ---- ranges (core/gaussian_render.cu:634-660) ---------------------------- */

void gso_ranges(int64_t k, const uint64_t* keys, int32_t num_tiles, int32_t* ranges)
{
    if (k <= 0) return;
    (void)num_tiles;
    ranges[(keys[0] >> 32) * 2] = 0;
    ranges[(keys[k - 1] >> 32) * 2 + 1] = (int32_t)k;
    for (int64_t i = 1; i < k; ++i) {
        uint64_t pt = keys[i - 1] >> 32, t = keys[i] >> 32;
        if (t != pt) {
            ranges[pt * 2 + 1] = (int32_t)i;
            ranges[t * 2] = (int32_t)i;
        }
    }
}

/* ---- camera ---------------------------------------------------------------- */

/* Look-at camera: glm::lookAtRH (external/glm/glm/ext/matrix_transform.inl:
 * 99-119) for the view matrix, core/camera.cpp:30-55 for the pose, and the
 * built frame loop's projection terms (app/main.cpp:352-358):
 * cot_y = 1/tan(fovy/2), cot_x = cot_y/aspect, depth (-2/(f-n), -(f+n)/(f-n)). */
void gso_look_at(gso_camera* cam, const float eye[3], const float target[3], const float up[3], float fovy_rad,
                 int32_t width, int32_t height, float znear, float zfar)
{
    float f[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
    const float fl = 1.0f / sqrtf(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (int k = 0; k < 3; ++k) f[k] *= fl;
    float s[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
    const float sl = 1.0f / sqrtf(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (int k = 0; k < 3; ++k) s[k] *= sl;
    const float u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
    float* m = cam->view;
    memset(m, 0, sizeof(cam->view));
    /* column-major: m[col * 4 + row] */
    m[0] = s[0]; m[4] = s[1]; m[8] = s[2];
    m[1] = u[0]; m[5] = u[1]; m[9] = u[2];
    m[2] = -f[0]; m[6] = -f[1]; m[10] = -f[2];
    m[12] = -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]);
    m[13] = -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]);
    m[14] = (f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2]);
    m[15] = 1.0f;
    for (int k = 0; k < 3; ++k) cam->position[k] = eye[k];
    cam->width = width;
    cam->height = height;
    cam->aspect = (float)width / (float)height;
    const float coty = 1.0f / tanf(fovy_rad * 0.5f);
    cam->fov_cotangent[0] = coty / cam->aspect;
    cam->fov_cotangent[1] = coty;
    cam->depth_scale_bias[0] = -2.0f / (zfar - znear);
    cam->depth_scale_bias[1] = -(zfar + znear) / (zfar - znear);
}

/* ---- raster (core/gaussian_render.cu:679-759) ----------------------------- */

/* Work count of the GPU's T_min raster, which has no counterpart in the
 * reference: each warp there owns an 8x8 pixel block, walks the tile's list
 * 32 entries at a time, keeps the entries whose cutoff box (where
 * opacity * density = 2^-18) touches the block, blends every kept entry into
 * all 64 pixels, and stops after a chunk once every pixel of the block has
 * T < t_min.  gso_raster adds the (pixel, entry) evaluations that this walk
 * executes to a counter when counting is on (the raster roofline's work);
 * the image and the `evals` output of gso_raster are unchanged. */
static int g_count_blocks = 0;
static int64_t g_block_evals = 0;
void gso_set_count_block_evals(int on)
{
    g_count_blocks = on;
    g_block_evals = 0;
}
int64_t gso_block_evals(void) { return g_block_evals; }

static const float kGsoCullAlpha = 3.814697265625e-06f; /* 2^-18 */

static int64_t block_walk_evals(int tile_px0, int tile_py0, int tw, int th, int W, int H, float texx, float texy,
                                const int32_t* list, int count, const float* xy, const float* conic4,
                                const float* color4, float t_min)
{
    int64_t e = 0;
    for (int by = 0; by < th; by += 8)
        for (int bx = 0; bx < tw; bx += 8) {
            const int wx0 = tile_px0 + bx, wy0 = tile_py0 + by;
            const float bx0 = (float)wx0 * texx - 1.0f, bx1 = (float)(wx0 + 7) * texx - 1.0f;
            const float by0 = (float)wy0 * texy - 1.0f, by1 = (float)(wy0 + 7) * texy - 1.0f;
            float T[64];
            int live = 0;
            for (int p = 0; p < 64; ++p) {
                const int px = wx0 + (p & 7), py = wy0 + (p >> 3);
                T[p] = (px < W && py < H) ? 1.0f : 0.0f;
                live += T[p] >= t_min;
            }
            for (int c0 = 0; c0 < count && live; c0 += 32) {
                const int nb = count - c0 < 32 ? count - c0 : 32;
                for (int j = 0; j < nb; ++j) {
                    const int32_t s = list[c0 + j];
                    const float x = xy[2 * s], y = xy[2 * s + 1];
                    const float ca = conic4[4 * s], cb = conic4[4 * s + 1], cc = conic4[4 * s + 2];
                    const float o = color4[4 * s + 3];
                    const float det = ca * cc - cb * cb;
                    /* below the cutoff, or a conic that is not positive definite: no record */
                    if (!(o > kGsoCullAlpha) || !(det > 0.0f) || !(ca > 0.0f) || !(cc > 0.0f)) continue;
                    const float qc = 2.0f * logf(o / kGsoCullAlpha);
                    const float ex = sqrtf(qc * cc / det), ey = sqrtf(qc * ca / det);
                    if (!(x - ex <= bx1 && x + ex >= bx0 && y - ey <= by1 && y + ey >= by0)) continue;
                    e += 64;
                    for (int p = 0; p < 64; ++p) {
                        if (T[p] < t_min) continue;
                        const float dx = ((float)(wx0 + (p & 7)) * texx - 1.0f) - x;
                        const float dy = ((float)(wy0 + (p >> 3)) * texy - 1.0f) - y;
                        const float q = ca * dx * dx + cc * dy * dy + 2.0f * cb * dx * dy;
                        float a = o * expf(-0.5f * q);
                        a = a > 1.0f ? 1.0f : (a < 0.0f ? 0.0f : a);
                        T[p] -= T[p] * a;
                    }
                }
                live = 0;
                for (int p = 0; p < 64; ++p) live += T[p] >= t_min;
            }
        }
    return e;
}

void gso_raster(const gso_camera* cam, const gso_cfg* cfg, const int32_t* ranges, const int32_t* values,
                const float* xy, const float* conic4, const float* color4, uint8_t* rgba, int64_t* evals)
{
    tilegeo_t g = tile_geo(cam, cfg);
    const int W = cam->width, H = cam->height;
    const int tw = cfg->tile_w, th = cfg->tile_h, np = tw * th;
    const float texx = 2.0f / (float)W, texy = 2.0f / (float)H;
    const int ntiles = g.tiles_x * g.tiles_y;
    int64_t total_evals = 0, block_evals = 0;
    const int count_blocks = g_count_blocks && cfg->termination == 1 && tw % 8 == 0 && th % 8 == 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total_evals, block_evals)
    for (int tile = 0; tile < ntiles; ++tile) {
        int32_t first = ranges[2 * tile], last = ranges[2 * tile + 1];
        int count = last - first;
        if (count == 0) continue;
        int tx = tile % g.tiles_x, ty = tile / g.tiles_x;
        if (count_blocks)
            block_evals += block_walk_evals(tx * tw, ty * th, tw, th, W, H, texx, texy, values + first, count, xy,
                                            conic4, color4, cfg->t_min);
        float T[1024], C[1024][3], pcx[1024], pcy[1024];
        int inimg[1024], done[1024];
        for (int p = 0; p < np; ++p) {
            int px = tx * tw + p % tw, py = ty * th + p / tw;
            inimg[p] = px < W && py < H;
            pcx[p] = mad((float)px, texx, -1.0f);
            pcy[p] = mad((float)py, texy, -1.0f);
            T[p] = 1.0f;
            C[p][0] = C[p][1] = C[p][2] = 0.0f;
            done[p] = !inimg[p];
        }
        if (cfg->termination == 0) {
            /* reference: batches of 32 entries, stop once no in-image pixel has T > 0.02 */
            for (int base = 0; base < count; base += 32) {
                int nb = count - base < 32 ? count - base : 32;
                for (int j = 0; j < nb; ++j) {
                    int32_t s = values[first + base + j];
                    float sx = xy[2 * s], sy = xy[2 * s + 1];
                    float ca = conic4[4 * s], cb = conic4[4 * s + 1], cc = conic4[4 * s + 2];
                    const float* col = color4 + 4 * s;
                    for (int p = 0; p < np; ++p) {
                        float dx = pcx[p] - sx, dy = pcy[p] - sy;
                        float q = ca * dx * dx + cc * dy * dy + 2.0f * cb * dx * dy;
                        float alpha = col[3] * saturate(expf(-0.5f * q));
                        float ta = T[p] * alpha;
                        C[p][0] += col[0] * ta;
                        C[p][1] += col[1] * ta;
                        C[p][2] += col[2] * ta;
                        T[p] *= (1.0f - alpha);
                    }
                }
                total_evals += (int64_t)nb * np;
                int any = 0;
                for (int p = 0; p < np; ++p) any |= inimg[p] && T[p] > 0.02f;
                if (!any) break;
            }
        } else {
            for (int j = 0; j < count; ++j) {
                int32_t s = values[first + j];
                float sx = xy[2 * s], sy = xy[2 * s + 1];
                float ca = conic4[4 * s], cb = conic4[4 * s + 1], cc = conic4[4 * s + 2];
                const float* col = color4 + 4 * s;
                int active = 0;
                for (int p = 0; p < np; ++p) {
                    if (done[p]) continue;
                    ++active;
                    float dx = pcx[p] - sx, dy = pcy[p] - sy;
                    float q = ca * dx * dx + cc * dy * dy + 2.0f * cb * dx * dy;
                    float alpha = col[3] * saturate(expf(-0.5f * q));
                    float ta = T[p] * alpha;
                    C[p][0] += col[0] * ta;
                    C[p][1] += col[1] * ta;
                    C[p][2] += col[2] * ta;
                    T[p] *= (1.0f - alpha);
                    if (T[p] < cfg->t_min) done[p] = 1;
                }
                total_evals += active;
                if (active == 0) break;
            }
        }
        for (int p = 0; p < np; ++p) {
            if (!inimg[p]) continue;
            int px = tx * tw + p % tw, py = ty * th + p / tw;
            uint8_t* o = rgba + 4 * ((int64_t)py * W + px);
            o[0] = cvt_u8(C[p][0] * 255.0f);
            o[1] = cvt_u8(C[p][1] * 255.0f);
            o[2] = cvt_u8(C[p][2] * 255.0f);
            o[3] = 255;
        }
    }
    if (evals) *evals = total_evals;
    if (count_blocks) g_block_evals += block_evals;
}

/* ---- whole frame --------------------------------------------------------- */

int64_t gso_render(int64_t n, const float* pos4, const float* scale_rot4, const float* color4_in,
                   const float* sh, int32_t sh_degree, int32_t sh_count, const gso_camera* cam, const gso_cfg* cfg,
                   uint8_t* rgba, int64_t key_capacity, int64_t* evals, double* stage_ms)
{
    double t0 = now_ms();
    float* color = (float*)malloc(sizeof(float) * 4 * (size_t)(n > 0 ? n : 1));
    if (sh_degree > 0) {
        int deg = sh_degree < cfg->sh_max_degree ? sh_degree : cfg->sh_max_degree;
        gso_sh(n, pos4, sh, sh_count, deg, cam->position, color);
    } else {
        memcpy(color, color4_in, sizeof(float) * 4 * (size_t)n);
    }
    double t1 = now_ms();
    float* xy = (float*)malloc(sizeof(float) * 2 * (size_t)(n > 0 ? n : 1));
    float* z = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* ell = (float*)malloc(sizeof(float) * 4 * (size_t)(n > 0 ? n : 1));
    float* con = (float*)malloc(sizeof(float) * 4 * (size_t)(n > 0 ? n : 1));
    gso_project(n, pos4, scale_rot4, cam, xy, z, ell, con);
    double t2 = now_ms();
    int64_t K = gso_build(n, xy, ell, z, cam, cfg, NULL, NULL, 0);
    int64_t result = K;
    if (K > key_capacity) {
        result = -1;
    } else {
        uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(K > 0 ? K : 1));
        int32_t* vals = (int32_t*)malloc(sizeof(int32_t) * (size_t)(K > 0 ? K : 1));
        gso_build(n, xy, ell, z, cam, cfg, keys, vals, K);
        double t3 = now_ms();
        tilegeo_t g = tile_geo(cam, cfg);
        int ntiles = g.tiles_x * g.tiles_y;
        int bits = 32;
        while ((1ll << (bits - 32)) < ntiles) ++bits;
        gso_sort(K, keys, vals, bits);
        double t4 = now_ms();
        int32_t* ranges = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)ntiles);
        memset(ranges, 0xFF, sizeof(int32_t) * 2 * (size_t)ntiles);
        gso_ranges(K, keys, ntiles, ranges);
        double t5 = now_ms();
        gso_raster(cam, cfg, ranges, vals, xy, con, color, rgba, evals);
        double t6 = now_ms();
        if (stage_ms) {
            stage_ms[0] = t1 - t0;
            stage_ms[1] = t2 - t1;
            stage_ms[2] = t3 - t2;
            stage_ms[3] = t4 - t3;
            stage_ms[4] = t5 - t4;
            stage_ms[5] = t6 - t5;
        }
        free(ranges);
        free(keys);
        free(vals);
    }
    free(color);
    free(xy);
    free(z);
    free(ell);
    free(con);
    return result;
}
