/*
 * CPU ORACLE for the 3D Gaussian splatting frame pipeline.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  This is a plain-C restatement of
 * the reference renderer's five stages (RobinSongx/3DGaussianRenderer,
 * core/gaussian_render.cu) used only by tests/, the smoke check and the
 * CPU-baseline leg of bench.py, as the checker of the CUDA path.  The
 * product library never links or calls it.
 *
 * Parity is pinned against the reference itself: oracle/ref/build_ref.sh
 * compiles the reference's own kernels into oracle/_ref/libgsref.so, and
 * tests/golden/ holds outputs of those kernels run on a B200 (with the
 * script that produced them).  The tests check this oracle against them.
 *
 * Floating-point model.  Every expression follows the reference's
 * operation order (glm 0.9.9 semantics: min(x,y) = y<x ? y : x,
 * max(x,y) = x<y ? y : x, normalize(v) = v * (1/sqrt(dot(v,v))),
 * step(e,x) = x<e ? 0 : 1, mix(x,y,a) = x*(1-a) + y*a).  nvcc contracts
 * a*b+c into fused multiply-adds; which product of a sum it fuses is
 * selected by gso_set_fma_mode() and pinned by the tests against the
 * reference kernels' outputs.  Device float->int conversions saturate
 * (NaN -> 0); the oracle emulates that explicitly.
 */
#ifndef GS_ORACLE_H
#define GS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-view camera, same layout as gs_camera in include/gs_b200.h. */
typedef struct gso_camera {
    float view[16];            /* world -> view, column-major (glm) */
    float position[3];         /* camera centre, world space */
    float fov_cotangent[2];    /* (cot(fovy/2)/aspect, cot(fovy/2)) */
    float depth_scale_bias[2]; /* (-2/(f-n), -(f+n)/(f-n)) */
    float aspect;
    int32_t width, height;
} gso_camera;

/* Tile / termination parameters, same meaning as gs_render_cfg. */
typedef struct gso_cfg {
    int32_t sh_max_degree; /* evaluate SH up to min(scene degree, this); reference evaluates <= 2 */
    int32_t termination;   /* 0: reference tile-wide T<=0.02 test after every 32 entries; 1: per-pixel T<t_min */
    float t_min;
    int32_t tile_w, tile_h;
} gso_cfg;

/* Look-at camera (glm::lookAtRH view, core/camera.cpp:30-55 pose, the built
 * frame loop's projection terms app/main.cpp:352-358); fovy in radians. */
void gso_look_at(gso_camera* cam, const float eye[3], const float target[3], const float up[3], float fovy_rad,
                 int32_t width, int32_t height, float znear, float zfar);

/* 0: no contraction; 1: fuse the first product of a sum; 2: fuse the last. */
void gso_set_fma_mode(int mode);
/* float -> uint8 conversion of the final colour: 0 saturate, 1 int32 low byte,
 * 2 uint32 low byte (see gs_oracle.c). */
void gso_set_u8_mode(int mode);
int gso_get_fma_mode(void);
void gso_set_threads(int n);
int gso_max_threads(void);

/* ---- stage functions (reference buffer layouts) ---------------------- */

/* SH colour, core/gaussian_render.cu:50-116 (+ degree-3 terms of
 * core/cuda_renderer.cu:119-156 when eval_degree == 3).  sh uses the
 * reference's grouped layout [ceil(n/256)][sh_count][256]. */
void gso_sh(int64_t n, const float* pos4, const float* sh, int32_t sh_count, int32_t eval_degree,
            const float cam_pos[3], float* color4);

/* EWA projection, core/gaussian_render.cu:135-215.  Outputs: xy[2n], z[n],
 * ellipse[4n] = (cos, sin, extent.x, extent.y), conic[4n] = (a, b, c, 0). */
void gso_project(int64_t n, const float* pos4, const float* scale_rot4, const gso_camera* cam, float* xy,
                 float* z, float* ellipse4, float* conic4);

/* getAABBRect, core/gaussian_render.cu:274-298.  ell6 = (cx, cy, cos, sin, ex, ey). */
void gso_aabb(int64_t n, const float* ell6, float* rect4);
/* ellipseRectOverlap, core/gaussian_render.cu:250-272. */
void gso_overlap(int64_t n, const float* ell6, const float* rect4, int32_t* out);
/* getKey, core/gaussian_render.cu:306-310. */
void gso_key(int64_t n, const int32_t* tile, const float* depth, uint64_t* out);

/* Tile rectangle (x0, y0, w, h) and candidate count max(0, w*h) per
 * Gaussian (core/gaussian_render.cu:377-389), plus the exact number of
 * overlapping tiles.  Either output pointer may be NULL. */
void gso_tile_counts(int64_t n, const float* xy, const float* ellipse4, const gso_camera* cam,
                     const gso_cfg* cfg, int32_t* rect4, int32_t* cand, int32_t* hits);

/* Tile-list build (core/gaussian_render.cu:312-564) emitted in Gaussian
 * order, candidates row-major inside each rectangle.  Returns K.  keys /
 * values may be NULL to count only; at most `capacity` entries are written. */
int64_t gso_build(int64_t n, const float* xy, const float* ellipse4, const float* z, const gso_camera* cam,
                  const gso_cfg* cfg, uint64_t* keys, int32_t* values, int64_t capacity);

/* Stable sort of (key, value) pairs on key bits [0, key_bits)
 * (core/gaussian_render.cu:591-632 uses bits [0,44)). */
void gso_sort(int64_t k, uint64_t* keys, int32_t* values, int32_t key_bits);

/* Tile ranges (core/gaussian_render.cu:634-660).  ranges[2*num_tiles] must
 * be pre-filled with -1 by the caller, as the reference frame does. */
void gso_ranges(int64_t k, const uint64_t* keys, int32_t num_tiles, int32_t* ranges);

/* Tile rasteriser (core/gaussian_render.cu:679-759).  rgba[4*W*H] must be
 * pre-cleared by the caller.  If evals != NULL it receives the number of
 * (pixel, splat) blend evaluations executed. */
/* When on (reset to 0 by the call), gso_raster in T_min mode also adds to a
 * counter the (pixel, entry) evaluations that the GPU's warp-culled raster
 * executes (8x8 blocks, 32-entry chunks, cutoff alpha 2^-18); read it with
 * gso_block_evals. */
void gso_set_count_block_evals(int on);
int64_t gso_block_evals(void);
void gso_raster(const gso_camera* cam, const gso_cfg* cfg, const int32_t* ranges, const int32_t* values,
                const float* xy, const float* conic4, const float* color4, uint8_t* rgba, int64_t* evals);

/* Whole frame: SH (if sh_degree > 0; otherwise color4_in is used as the
 * colour buffer), project, build, sort, ranges, raster.  Returns K, or -1
 * when K exceeds key_capacity (nothing is rendered then). */
int64_t gso_render(int64_t n, const float* pos4, const float* scale_rot4, const float* color4_in,
                   const float* sh, int32_t sh_degree, int32_t sh_count, const gso_camera* cam, const gso_cfg* cfg,
                   uint8_t* rgba, int64_t key_capacity, int64_t* evals, double* stage_ms);

#ifdef __cplusplus
}
#endif
#endif
