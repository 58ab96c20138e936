/*
 * gs_b200 — B200-native 3D Gaussian splatting frame pipeline, C ABI.
 *
 * Drop-in for the stage API of RobinSongx/3DGaussianRenderer
 * (core/gaussian_render.cuh:113-126, implemented in core/gaussian_render.cu)
 * and the engine behind its Renderer API (core/renderer.h:13-50).  All
 * entry points are extern "C", take plain pointers and sizes, return an
 * int status (GS_OK = 0) and never exit the process.  Device pointers are
 * marked d_; host pointers h_.  `stream` is a cudaStream_t passed as void*
 * (NULL = legacy default stream).
 *
 * Buffer layouts are the reference's:
 *   position          float4[n]  (x, y, z, opacity)                 main.cpp:295
 *   scale_rotation    float4[n]  (sx, sy, sz, quat8 bit-cast)        ply_parser.cpp:385-388
 *                     quat8: x<<24 | y<<16 | z<<8 | w, byte = (q+1)/2*255
 *   sh                float[ceil(n/256)*256*sh_count] grouped as
 *                     [group][coefficient][256], RGB interleaved per
 *                     coefficient                                 main.cpp:147-177
 *   color             float4[n]  (r, g, b, opacity)
 *   xy / z            float2[n] / float[n]  clip-space centre / depth
 *   ellipse           float4[n]  (cos, sin, extent.x, extent.y)
 *   conic             float4[n]  (a, b, c, 0)
 *   keys / values     uint64[K] (tile << 32 | quantised depth) / int32[K]
 *   ranges            int32[2 * tiles]  [first, one-past-last)
 *   rgba              uint8[4 * W * H], row 0 = bottom
 */
#ifndef GS_B200_H
#define GS_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GS_API __attribute__((visibility("default")))
#else
#define GS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    GS_OK = 0,
    GS_ERR_INVALID = 1,        /* bad argument */
    GS_ERR_OOM = 2,            /* device allocation failed */
    GS_ERR_CAPACITY = 3,       /* a caller-sized buffer is too small */
    GS_ERR_DEVICE_TIMEOUT = 4, /* a bounded device wait gave up */
    GS_ERR_CUDA = 5,           /* other CUDA error (see gs_last_error_string) */
    GS_ERR_NO_DEVICE = 6,      /* no usable sm_100 device */
    GS_ERR_CANCELLED = 7       /* a server request cancelled before it was rendered */
};

enum { GS_TERM_REFERENCE = 0, GS_TERM_TMIN = 1 };

/* Per-view camera.  Same fields as the reference's CameraData
 * (gaussian_render.cuh:16-25) minus the unused projection matrices, plus
 * the image size. */
typedef struct gs_camera {
    float view[16];            /* world -> view, column-major */
    float position[3];         /* camera centre, world space */
    float fov_cotangent[2];    /* (cot(fovy/2)/aspect, cot(fovy/2))   main.cpp:352-354 */
    float depth_scale_bias[2]; /* (-2/(f-n), -(f+n)/(f-n))            main.cpp:355-358 */
    float aspect;
    int32_t width, height;
} gs_camera;

/* Pipeline options. */
typedef struct gs_render_cfg {
    int32_t sh_max_degree; /* SH degrees evaluated: 2 = reference (gaussian_render.cu:62-91), 3 = full */
    int32_t termination;   /* GS_TERM_REFERENCE (T<=0.02 tile-wide every 32 entries) or GS_TERM_TMIN */
    float t_min;           /* per-pixel transmittance floor for GS_TERM_TMIN (1e-4) */
    int32_t tile_w, tile_h;/* 16x16 (reference), 16x8 or 8x8 */
    int32_t ordering;      /* GS_ORDER_BUCKETS (default) or GS_ORDER_ONESWEEP: how the tile list is ordered */
    int32_t sort_variant;  /* GS_ORDER_ONESWEEP tile shape: 0 = 512x8 keys, 1 = 256x8, 2 = 256x16, 3 = 512x16 */
    int32_t views_per_block; /* views the fused projection handles per block (0 = 16) */
    int32_t graph;         /* 1 (default): a frame whose scene, options and views' sizes and outputs repeat
                              is captured once into a CUDA graph and replayed; 0: plain stream launches */
    int32_t raster_chunk;  /* GS_TERM_TMIN raster: Gaussians each warp culls and stages in shared memory per
                              step, 32 or 64 (0 = 32) */
    int32_t raster_persistent; /* GS_TERM_TMIN raster: 1 = persistent CTAs pulling tiles (heavy first) from an
                              atomic queue; 0 (default) = one CTA per tile */
    int32_t sort_bits;     /* per-tile depth sort of GS_ORDER_BUCKETS frames inside the raster CTA: the top
                              varying depth bits sorted by radix passes, 8..32 (0 = 16); the rest is ordered by
                              insertion within runs.  The larger tiles, sorted ahead of the raster, use one
                              counting pass over 13 or 15 bits and fall back on this form for long runs */
} gs_render_cfg;

/* Tile-list ordering of the whole-frame entry points.  Both give the order of
 * the reference's stable (tile | depth) sort of keys emitted in Gaussian
 * order.  BUCKETS: per-tile counts, keys written straight into their tile's
 * range, one shared-memory depth sort per tile.  ONESWEEP: keys in Gaussian
 * order, onesweep radix sort on the significant tile and depth bits, then
 * per-tile ranges (the reference's structure, core/gaussian_render.cu:312-677). */
#define GS_ORDER_BUCKETS 0
#define GS_ORDER_ONESWEEP 1
/* Either ordering, as gs_autotune picked it for the batch's bucket (a frame
 * rendered with it untuned uses GS_ORDER_BUCKETS). */
#define GS_ORDER_AUTO 2

/* Per-stage device times of one frame, same fields as the reference's
 * RenderStats (core/types.h:26-33), plus the tile-list size. */
typedef struct gs_stats {
    double sh_eval_ms, project_ms, build_tile_ms, sort_ms, raster_ms, total_ms;
    int64_t num_keys;
    int64_t num_tiles;
    int64_t kernel_launches; /* gs_b200 kernels launched for the frame */
    int32_t graph_replay;    /* 1: the frame ran as a replay of a captured CUDA graph */
    int32_t attempts;        /* launches of the frame: 2 when the tile list outgrew its buffers and was redone;
                                a batch whose tile lists need 2^31 entries or more (or whose views x Gaussians
                                reach 2^31) renders as frames over halves of its views, with the same images:
                                the halves' stats add up and attempts counts the frame that found it too big */
} gs_stats;

typedef struct gs_ctx gs_ctx;
typedef struct gs_scene gs_scene;

/* ---- library / context ------------------------------------------------ */

GS_API int gs_version(void);
GS_API const char* gs_status_string(int status);
GS_API const char* gs_last_error_string(void);
GS_API void gs_default_cfg(gs_render_cfg* cfg);
/* Fills a gs_camera from a look-at pose, following camera.cpp:30-55 with the
 * built frame loop's depth convention (main.cpp:352-358). */
GS_API void gs_camera_look_at(gs_camera* cam, const float eye[3], const float target[3], const float up[3],
                       float fovy_rad, int32_t width, int32_t height, float znear, float zfar);

GS_API int gs_ctx_create(int device, gs_ctx** out);
GS_API int gs_ctx_destroy(gs_ctx* ctx);
/* Device bytes currently held by the context's frame buffers. */
GS_API int64_t gs_ctx_device_bytes(const gs_ctx* ctx);

/* ---- scenes (Renderer::UploadModel, core/renderer.cpp:36-88) ---------- */

/* Uploads host arrays (reference layouts above) into a device-resident,
 * immutable scene.  h_color may be NULL when sh_degree > 0; h_sh may be NULL
 * when sh_degree == 0.  sh_count = 3 * (sh_degree + 1)^2.
 *
 * The scene is stored in Morton order of the Gaussian centres (sorted on the
 * device during the upload); each Gaussian keeps its caller index, which
 * orders equal depths in the tile lists of GS_ORDER_BUCKETS frames, so the
 * images are those of the caller's order.  GS_ORDER_ONESWEEP frames order
 * equal depths by storage order: scenes that need that ordering to break
 * ties by caller index are created with GS_SCENE_KEEP_ORDER.  The upload
 * needs temporary device memory of about twice the scene's size. */
GS_API int gs_scene_create(gs_ctx* ctx, int64_t n, const float* h_position, const float* h_scale_rotation,
                    const float* h_color, const float* h_sh, int32_t sh_degree, gs_scene** out);
/* gs_scene_create with flags: GS_SCENE_KEEP_ORDER stores the Gaussians in the
 * caller's order (plain copies, no temporaries). */
#define GS_SCENE_KEEP_ORDER 1u
GS_API int gs_scene_create_ex(gs_ctx* ctx, int64_t n, const float* h_position, const float* h_scale_rotation,
                       const float* h_color, const float* h_sh, int32_t sh_degree, uint32_t flags, gs_scene** out);
GS_API int gs_scene_destroy(gs_scene* scene);
GS_API int64_t gs_scene_size(const gs_scene* scene);
GS_API int64_t gs_scene_device_bytes(const gs_scene* scene);

/* ---- whole frame (Renderer::Render, core/renderer.cpp:94-139) ---------- */

/* Renders one view into d_rgba (device, 4*W*H bytes, cleared by the call).
 * Stats may be NULL.  The call returns after the frame completed. */
GS_API int gs_render(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cam, const gs_render_cfg* cfg, uint8_t* d_rgba,
              gs_stats* stats, void* stream);

/* Same, with the image returned into host memory h_rgba (pinned or not). */
GS_API int gs_render_host(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cam, const gs_render_cfg* cfg,
                   uint8_t* h_rgba, gs_stats* stats, void* stream);

/* Renders V views (any mix of sizes) of one scene in one batched frame:
 * one flattened tile space with the view in the key's high bits, one
 * persistent rasteriser, replayed as a CUDA graph when the same view set
 * shape is rendered again.  d_rgba[v] (device) receive 4*W_v*H_v bytes. */
GS_API int gs_render_batch(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                    const gs_render_cfg* cfg, uint8_t* const* d_rgba, gs_stats* stats, void* stream);
/* Same, images copied into one host buffer: view v at byte offset
 * sum_{u<v} 4*W_u*H_u.  Batches of more than 16 views are read back in
 * groups of views while the next group renders: T_min bucket frames render
 * all views in one frame whose raster runs group by group; other frames
 * render 16 views at a time (the stats then add up the frames).  Returns
 * when every image is in h_rgba. */
GS_API int gs_render_batch_host(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                         const gs_render_cfg* cfg, uint8_t* h_rgba, gs_stats* stats, void* stream);

/* ---- autotuner (batching knobs per (N, resolution) bucket) ------------- */

/* One timed candidate of gs_autotune. */
typedef struct gs_tune_result {
    gs_render_cfg cfg;
    double ms;      /* median device time of one gs_render_batch call */
} gs_tune_result;

/* Times gs_render_batch of `cams` while sweeping the batching knobs, and
 * stores the fastest in the context's table under the bucket of (N = the
 * scene's size, the largest view's pixel count, num_views, base's
 * termination and ordering); gs_autotune_lookup reads it back.  The sweep is
 * a coordinate descent: each knob in turn is timed at all its values with
 * the others at the best found so far, in this order:
 *   tile shape 16x16 / 16x8 / 8x8   GS_TERM_TMIN only (the reference mode's
 *                                   tile-wide termination is defined on the
 *                                   16x16 tiles it was given; under
 *                                   per-pixel termination the colours of
 *                                   every shape agree to a few 8-bit steps
 *                                   at most, from splats whose faint tails
 *                                   reach past their tiles, while alpha,
 *                                   255 in tiles that hold any entry and 0
 *                                   elsewhere as in the reference, follows
 *                                   the grid);
 *   views_per_block 8 / 16 / 32     batches of more than 8 views;
 *   ordering buckets / onesweep     base ordering GS_ORDER_AUTO only;
 *   sort_variant 0..3               onesweep ordering;
 *   sort_bits 8 / 16 / 24 / 32      bucket ordering (the per-tile sort's
 *                                   radix width);
 *   raster_chunk 32 / 64            GS_TERM_TMIN (Gaussians per
 *                                   shared-memory batch of the raster);
 *   raster_persistent 0 / 1         GS_TERM_TMIN.
 * The sorts are exact, so sort knobs never change an image; raster_chunk
 * moves where a warp notices that its pixels are done, which changes colours
 * by less than t_min.  Each candidate renders 2 untimed frames (the second
 * captures its graph when base->graph is set) and then `iterations` timed
 * ones (>= 1) into context-owned images.  `best` receives base with the
 * winning knobs, `best_ms` its time; `results` (may be NULL) receives up to
 * `results_capacity` candidates in the order they were timed and
 * `num_results` (may be NULL) their count.  Synchronous. */
GS_API int gs_autotune(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                       const gs_render_cfg* base, int32_t iterations, gs_render_cfg* best, double* best_ms,
                       gs_tune_result* results, int32_t results_capacity, int32_t* num_results, void* stream);
/* Applies the knobs gs_autotune stored for the bucket of (n, width*height,
 * num_views, cfg->termination, cfg->ordering) to *cfg (GS_ORDER_AUTO becomes
 * the tuned ordering) and sets *found = 1;
 * leaves *cfg as it is and sets *found = 0 when that bucket was not tuned.
 * Buckets: N and the pixel count by their power of two (floor log2), the
 * view count by 1, 2-4, 5-8, 9-16, 17-32, 33+. */
GS_API int gs_autotune_lookup(gs_ctx* ctx, int64_t n, int32_t width, int32_t height, int32_t num_views,
                              gs_render_cfg* cfg, int32_t* found);
/* Entries in the context's tuning table. */
GS_API int32_t gs_autotune_entries(gs_ctx* ctx);
/* The bucket gs_autotune and gs_autotune_lookup file a batch under:
 * bucket[0] = floor(log2 n) (-1 for n = 0), bucket[1] = floor(log2(width *
 * height)), bucket[2] = view-count class 0..5 (1, 2-4, 5-8, 9-16, 17-32,
 * 33+).  No device work. */
GS_API int gs_autotune_bucket(int64_t n, int32_t width, int32_t height, int32_t num_views, int32_t bucket[3]);

/* ---- performance overlay (app/perf_overlay.cpp:115-161) ---------------- */

/* DrawPerformanceOverlay: draws the reference's eight statistics lines
 * (FPS, Gaussians, Total, SH, Project, Build, Sort, Raster; same formats)
 * as white 5x7-pixel text into the device RGBA8 image d_rgba (W x H, row 0
 * at the bottom), upright and 5 pixels from the displayed image's top-left
 * corner.  Asynchronous on `stream`; only the text pixels are written. */
GS_API int gs_draw_stats(uint8_t* d_rgba, int32_t width, int32_t height, int64_t num_gaussians,
                         const gs_stats* stats, double fps, void* stream);
/* The eight lines gs_draw_stats draws, each ending in '\n', into `out`
 * (NUL-terminated); GS_ERR_CAPACITY when `capacity` is too small. */
GS_API int gs_format_stats(int64_t num_gaussians, const gs_stats* stats, double fps, char* out, int32_t capacity);
/* The overlay font: 7 rows of glyph `c` (bit 4 = leftmost of 5 columns;
 * all zero outside ASCII 32..126). */
GS_API int gs_font_glyph(int32_t c, uint8_t rows[7]);

/* ---- headless image output (replaces the PBO display path,
 *      core/utilities.h:110-153, app/opengl_display.cpp) --------------- */

/* Write a host RGBA8 frame (W x H, row 0 at the bottom, as rendered) to a
 * file with the top row first: binary PPM (P6, RGB; alpha dropped) or PNG
 * (8-bit RGBA, uncompressed deflate blocks).  GS_ERR_INVALID on a bad
 * argument or a failed write. */
GS_API int gs_write_ppm(const char* path, const uint8_t* h_rgba, int32_t width, int32_t height);
GS_API int gs_write_png(const char* path, const uint8_t* h_rgba, int32_t width, int32_t height);

/* ---- stage API (core/gaussian_render.cuh:113-126) ---------------------- */
/* Explicit-argument replacements of the reference's constant-memory stage
 * functions.  All pointers are device pointers; every call is asynchronous
 * on `stream` unless stated otherwise. */

/* evaluateSphericalHarmonics (gaussian_render.cu:96-133) */
GS_API int gs_stage_sh(int64_t n, const float* d_position, const float* d_sh, int32_t sh_count, int32_t eval_degree,
                const gs_camera* cam, float* d_color, void* stream);

/* evaluateSplatClipData (gaussian_render.cu:135-232) */
GS_API int gs_stage_project(int64_t n, const float* d_position, const float* d_scale_rotation, const gs_camera* cam,
                     float* d_xy, float* d_z, float* d_ellipse, float* d_conic, void* stream);

/* buildTileList (gaussian_render.cu:312-589).  Exact: counts every
 * Gaussian's overlapping tiles, scans, and emits keys in Gaussian order.
 * Synchronises once to read K into *out_num_keys.  When K > capacity it
 * writes the first `capacity` keys (in Gaussian order; the reference
 * truncates in atomic order) and returns GS_ERR_CAPACITY with the exact K,
 * so the caller can grow the lists. */
GS_API int gs_stage_build(gs_ctx* ctx, int64_t n, const float* d_xy, const float* d_z, const float* d_ellipse,
                   const gs_camera* cam, const gs_render_cfg* cfg, uint64_t* d_keys, int32_t* d_values,
                   int64_t capacity, int64_t* out_num_keys, void* stream);

/* sortTileList (gaussian_render.cu:591-632): stable LSD radix sort of K
 * pairs on key bits [0, key_bits), onesweep with decoupled look-back.  The
 * result ends in (d_keys, d_values) when *out_selector == 0 and in
 * (d_keys_alt, d_values_alt) when 1.  Scratch comes from the context. */
GS_API int gs_stage_sort(gs_ctx* ctx, int64_t num_keys, int32_t key_bits, uint64_t* d_keys, int32_t* d_values,
                  uint64_t* d_keys_alt, int32_t* d_values_alt, int32_t* out_selector, void* stream);

/* No counterpart in the reference.  The same sort as gs_stage_sort, for
 * callers that must not allocate device memory (an application that hands
 * out all device memory from its own pool, or a frame loop that cannot afford
 * the device-wide synchronisation of cudaMalloc/cudaFree): its scratch is a
 * fixed array inside the library (about 2 MiB on every GPU that loads it) and
 * the call allocates nothing.  At most gs_stage_sort_noalloc_max_keys()
 * (4,194,304) keys; more returns GS_ERR_CAPACITY.  All calls share the array:
 * calls that overlap on the GPU race, so serialise them.  The first call on
 * a device loads the array's module and resolves its address; make it
 * before any stream capture.  Every call re-reads the address, so the call
 * keeps working after a cudaDeviceReset.  Synchronises `stream` before
 * returning. */
GS_API int gs_stage_sort_noalloc(int64_t num_keys, int32_t key_bits, uint64_t* d_keys, int32_t* d_values,
                                 uint64_t* d_keys_alt, int32_t* d_values_alt, int32_t* out_selector, void* stream);
GS_API int64_t gs_stage_sort_noalloc_max_keys(void);
GS_API const char* gs_stage_sort_noalloc_error(void);

/* evaluateTileRange (gaussian_render.cu:634-677).  Fills all 2*num_tiles
 * entries: tiles without keys get (-1, -1) as after the reference's
 * 0xFF clear (main.cpp:365). */
GS_API int gs_stage_ranges(int64_t num_keys, const uint64_t* d_keys, int64_t num_tiles, int32_t* d_ranges, void* stream);

/* rasterizeTile (gaussian_render.cu:679-775).  d_rgba must be cleared by
 * the caller (tiles without splats are not written, main.cpp:363). */
GS_API int gs_stage_raster(const gs_camera* cam, const gs_render_cfg* cfg, const int32_t* d_ranges, const int32_t* d_values,
                    const float* d_xy, const float* d_conic, const float* d_color, uint8_t* d_rgba, void* stream);

/* ---- serving: resident scenes, continuous batching ---------------------- */
/* No counterpart in the reference (a single-scene desktop viewer); this is
 * the serving loop built on the batched frame.  Scenes stay resident; view
 * requests from any thread are grouped per scene into batched frames as
 * workers free up (each worker: its own context and stream, so batches
 * overlap on the device), admitted against a device-memory budget. */
typedef struct gs_server gs_server;
typedef struct gs_server_cfg {
    int64_t budget_bytes;     /* scenes + frame buffers must fit (150 GiB default) */
    int32_t max_batch_views;  /* views per batched frame */
    int32_t num_workers;      /* batches in flight */
    gs_render_cfg render;     /* frame options (default: gs_default_cfg with graph = 0, the batches
                                 rarely repeat) */
    double batch_target_ms;   /* a batch stops growing once its estimated time exceeds this (8 ms; 0 = off) */
} gs_server_cfg;
typedef struct gs_server_stats {
    int64_t views_done, batches_done, max_batch;
    double p50_ms, p99_ms, mean_ms; /* submit -> image in the host buffer */
    double views_per_s;             /* views done / (last completion - first submit) */
    int64_t resident_bytes, frame_bytes, pending;
} gs_server_stats;

GS_API void gs_server_default_cfg(gs_server_cfg* cfg);
GS_API int gs_server_create(int device, const gs_server_cfg* cfg, gs_server** out);
GS_API int gs_server_destroy(gs_server* server);
/* GS_ERR_CAPACITY when the scene does not fit the budget. */
GS_API int gs_server_add_scene(gs_server* server, int64_t n, const float* h_position, const float* h_scale_rotation,
                               const float* h_color, const float* h_sh, int32_t sh_degree, int32_t* out_scene_id);
/* Non-blocking; h_rgba (4*W*H bytes, host) is written before the request completes. */
GS_API int gs_server_submit(gs_server* server, int32_t scene_id, const gs_camera* cam, uint8_t* h_rgba,
                            int64_t* out_request_id);
/* Waits up to timeout_ms; returns the request's status (GS_ERR_DEVICE_TIMEOUT if not done,
 * GS_ERR_CANCELLED if it was cancelled). */
GS_API int gs_server_wait(gs_server* server, int64_t request_id, double timeout_ms, double* out_latency_ms);
/* Cancels a request that is still queued: it completes at once with status
 * GS_ERR_CANCELLED and its host buffer is never written.  GS_ERR_INVALID when
 * the request is unknown, finished, or already part of a batch on the device
 * (which is never interrupted). */
GS_API int gs_server_cancel(gs_server* server, int64_t request_id);
/* paused = 1: submitted requests queue and no new batch is dispatched
 * (batches already on the device finish); 0: dispatching resumes. */
GS_API int gs_server_pause(gs_server* server, int32_t paused);
GS_API int gs_server_get_stats(gs_server* server, gs_server_stats* out);
GS_API int gs_server_reset_stats(gs_server* server);

/* ---- model ingest (parsePly / savePly, core/ply_parser.cpp:15-393) ------ */
/* Binary little-endian PLY with float properties named as the INRIA 3DGS
 * exporter writes them (x y z rot_0..3 scale_0..2 f_dc_0..2 f_rest_* opacity).
 * Errors are GS_ERR_INVALID with the reason in gs_ply_last_error(). */
GS_API int gs_ply_info(const char* path, int64_t* out_n, int32_t* out_sh_degree);
GS_API const char* gs_ply_last_error(void);
/* Applies the reference's load transforms (normalised quaternion -> 8-bit
 * encoding, exp(scale), sigmoid(opacity), DC*C0+0.5) and writes the host
 * buffers in the layouts above; h_sh_grouped (SH scenes) takes
 * ceil(n/256)*256*sh_count floats.  Any output may be NULL; bounds[6] =
 * (min xyz, max xyz) as the reference computes them. */
GS_API int gs_ply_read(const char* path, float* h_position, float* h_scale_rotation, float* h_color,
                       float* h_sh_grouped, float* bounds);
/* Writes a scene as a PLY that gs_ply_read (and the reference's parsePly)
 * reads back; SH scenes get f_rest_* (channel-major). */
GS_API int gs_ply_write(const char* path, int64_t n, const float* h_position, const float* h_scale_rotation,
                        const float* h_color, const float* h_sh_grouped, int32_t sh_degree);

/* ---- frame probe (diagnostics and tests) ------------------------------- */
/* No counterpart in the reference, whose stages leave every intermediate
 * buffer with the caller; the fused frame keeps them internal, and the probe
 * exposes what the parity tests compare with the reference's stages.
 * Device outputs per (view, Gaussian), num_views * n entries each, at
 * view * n + the caller's index of the Gaussian: */
typedef struct gs_frame_probe {
    float* d_xy;      /* float2 clip-space centre; frustum-culled: (-128, -128) */
    float* d_z;       /* clip-space depth; culled: -128 */
    float* d_ellipse; /* float4 (cos, sin, extent.x, extent.y) as the tile lists use it; culled: 0 */
    float* d_conic;   /* float4 (a, b, c, 0); culled: 0 */
    float* d_color;   /* float4 (r, g, b, opacity) of the Gaussians that reach a tile (others untouched); may be NULL */
} gs_frame_probe;

/* Renders like gs_render_batch with GS_ORDER_BUCKETS (never from a captured
 * graph) and writes the probe outputs.  The projection and tile lists are
 * those of an ordinary frame with the same options. */
GS_API int gs_probe_frame(gs_ctx* ctx, const gs_scene* scene, const gs_camera* cams, int32_t num_views,
                          const gs_render_cfg* cfg, uint8_t* const* d_rgba, const gs_frame_probe* probe,
                          gs_stats* stats, void* stream);
/* Copies the tile lists of the context's last GS_ORDER_BUCKETS frame to host
 * memory (GS_ERR_INVALID when a stage call or a onesweep frame has reused
 * the buffers since).  out_sizes = (tiles T, keys K, slots S);
 * *out_fused_cap = the largest tile the raster CTA sorts itself.
 *   h_ranges[2T]    first and one-past-last key of every tile (all views'
 *                   tiles, view after view);
 *   h_keys[K]       the tiles' keys as emitted, (depth bits << 32 | slot),
 *                   in any order inside a tile: the raster CTA of a tile of
 *                   at most fused_cap keys orders them by (depth, index);
 *   h_order[K]      for the larger tiles, the slots in blend order (sorted
 *                   ahead of the raster); meaningless for the others;
 *   h_slot_index[S] view * n + caller index of each slot.
 * Any output may be NULL.  Synchronous. */
GS_API int gs_probe_tile_lists(gs_ctx* ctx, int32_t* h_ranges, int64_t ranges_capacity, uint64_t* h_keys,
                               int32_t* h_order, int64_t keys_capacity, int32_t* h_slot_index, int64_t slots_capacity,
                               int64_t out_sizes[3], int32_t* out_fused_cap);

/* No counterpart in the reference.  Times gs_stage_sort's onesweep sort
 * alone, for a like-for-like comparison with a library sort timed around
 * its own call: `iterations` times, the unsorted (d_src_keys, d_src_values)
 * are copied into (d_keys, d_values) and the sort runs between two CUDA
 * events on the legacy default stream, with nothing else in the timed
 * region.  *out_median_ms = the median, *out_selector as gs_stage_sort's.
 * Synchronous. */
GS_API int gs_probe_sort_timed(gs_ctx* ctx, int64_t num_keys, int32_t key_bits, const uint64_t* d_src_keys,
                               const int32_t* d_src_values, uint64_t* d_keys, int32_t* d_values, uint64_t* d_keys_alt,
                               int32_t* d_values_alt, int32_t iterations, int32_t* out_selector,
                               double* out_median_ms);

/* ---- failure-path test hooks -------------------------------------------- */
/* No counterpart in the reference, which exits the process on any CUDA
 * error (core/cuda_error_check.h:2-11).  These let tests exercise the error
 * paths that replace it without faulting a GPU. */
/* After `skip` more device buffer allocations of contexts and scenes
 * succeed, the next `count` fail as if the device were out of memory
 * (process-wide; count = 0 clears the hook).  The failing call returns
 * GS_ERR_OOM and the context stays usable. */
GS_API void gs_test_fail_allocations(int32_t skip, int32_t count);
/* Injected failures not yet consumed. */
GS_API int32_t gs_test_pending_allocation_failures(void);
/* Runs one bounded device wait on a word nobody publishes (the decoupled
 * look-back every scan and sort pass uses) with a limit of `spin_limit`
 * polls (1 .. 4194304).  Returns GS_ERR_DEVICE_TIMEOUT when the wait gave up
 * and reported it, as it must; the context stays usable. */
GS_API int gs_test_bounded_wait(int32_t spin_limit, void* stream);

/* Number of tiles of a W x H image with the cfg's tile shape. */
GS_API int64_t gs_num_tiles(int32_t width, int32_t height, const gs_render_cfg* cfg);
/* Significant key bits for `num_tiles` tiles: 32 + ceil(log2(num_tiles)). */
GS_API int32_t gs_key_bits(int64_t num_tiles);

#ifdef __cplusplus
}
#endif
#endif
