/*
 * gs_stage_compat.hpp -- the reference's stage API on gs_b200.
 *
 * RobinSongx/3DGaussianRenderer drives its frame through eight free
 * functions declared in core/gaussian_render.cuh:113-126 and implemented in
 * core/gaussian_render.cu, which read their arguments from __constant__
 * symbols.  This header implements the same eight functions, with the same
 * signatures and the same meaning, on the C ABI of include/gs_b200.h, so a
 * program written against the reference (app/main.cpp:360-432) renders
 * with gs_b200 without a change to its call sites:
 *
 *     // one translation unit of the program, in place of gaussian_render.cu
 *     #include "gaussian_render.cuh"   // the reference's structs and CudaTimer
 *     #include "gs_stage_compat.hpp"   // this file: the eight functions
 *
 * and link with -lgs_b200 -lcudart instead of compiling gaussian_render.cu.
 * The header defines (not just declares) the functions, so it belongs in
 * exactly one translation unit.  It needs, from the reference's headers,
 * CameraData, GlobalArgs, TileListArgs, DoubleBuffer, CudaTimer
 * (start/stop), k_ScreenSize and k_TotalTiles.
 *
 * Behaviour, stage by stage, against the reference:
 *   setGlobalArgs / setTileListArgs   copy the structs on the host (no
 *                                     constant-memory upload, no sync)
 *   evaluateSphericalHarmonics        gs_stage_sh, degree min(scene, 2)
 *                                     (the reference evaluates <= 2,
 *                                     gaussian_render.cu:62-91)
 *   evaluateSplatClipData             gs_stage_project: every float bit-exact
 *   buildTileList                     gs_stage_build: K exact; a list that
 *                                     does not fit is truncated and reported
 *                                     full (returns the capacity), as the
 *                                     reference does (gaussian_render.cu:
 *                                     506-509); keys in Gaussian order
 *   sortTileList                      gs_stage_sort on bits [0, 44): stable,
 *                                     so equal keys leave in index order
 *                                     (the reference's atomic emission
 *                                     leaves that order arbitrary); no
 *                                     temporary storage is allocated, the
 *                                     scratch lives in a gs_ctx
 *   evaluateTileRange                 gs_stage_ranges (tiles without keys
 *                                     get -1, as after the frame loop's
 *                                     0xFF clear)
 *   rasterizeTile                     gs_stage_raster in the reference's
 *                                     termination mode: the reference's image
 *
 * All stages run on the legacy default stream and are timed by the caller's
 * CudaTimer exactly where the reference times them.  Errors: the reference
 * exits on CUDA errors; these functions never exit -- they print the status
 * to stderr and keep it for gs_stage_compat_status().  The gs_ctx (sort and
 * build scratch) is created on the current device at the first call that
 * needs it and kept until gs_stage_compat_release().  Not thread-safe, like
 * the reference's constant-memory globals.
 */
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include <cuda_runtime_api.h>

#include "gs_b200.h"

namespace gs_stage_compat {

inline GlobalArgs& args()
{
    static GlobalArgs a{};
    return a;
}
inline TileListArgs& tiles()
{
    static TileListArgs t{};
    return t;
}
inline int& last_status()
{
    static int s = GS_OK;
    return s;
}
inline gs_ctx*& context()
{
    static gs_ctx* c = nullptr;
    return c;
}

inline int report(int status, const char* stage)
{
    if (status != GS_OK) {
        last_status() = status;
        std::fprintf(stderr, "gs_stage_compat: %s: %s (%s)\n", stage, gs_status_string(status),
                     gs_last_error_string());
    }
    return status;
}

inline gs_ctx* ctx()
{
    if (!context()) {
        int dev = 0;
        cudaGetDevice(&dev);
        report(gs_ctx_create(dev, &context()), "gs_ctx_create");
    }
    return context();
}

// CameraData (gaussian_render.cuh:16-25) -> gs_camera at the reference's
// fixed k_ScreenSize x k_ScreenSize resolution (core/consts.h:4)
inline gs_camera camera()
{
    const CameraData& d = args().cameraData;
    gs_camera c;
    std::memset(&c, 0, sizeof(c));
    std::memcpy(c.view, &d.view[0][0], sizeof(c.view));
    c.position[0] = d.position.x;
    c.position[1] = d.position.y;
    c.position[2] = d.position.z;
    c.fov_cotangent[0] = d.fovCotangent.x;
    c.fov_cotangent[1] = d.fovCotangent.y;
    c.depth_scale_bias[0] = d.depthScaleBias.x;
    c.depth_scale_bias[1] = d.depthScaleBias.y;
    c.aspect = d.aspect;
    c.width = k_ScreenSize;
    c.height = k_ScreenSize;
    return c;
}

// the reference's behaviour: SH to degree 2, 16x16 tiles, T <= 0.02
// tile-wide termination after every 32 entries
inline gs_render_cfg reference_cfg()
{
    gs_render_cfg cfg;
    gs_default_cfg(&cfg);
    cfg.sh_max_degree = 2;
    cfg.termination = GS_TERM_REFERENCE;
    cfg.tile_w = 16;
    cfg.tile_h = 16;
    return cfg;
}

}  // namespace gs_stage_compat

/* Status of the last stage call that failed (GS_OK when none did). */
inline int gs_stage_compat_status() { return gs_stage_compat::last_status(); }

/* Destroys the context the stages created (the next call makes a new one). */
inline void gs_stage_compat_release()
{
    if (gs_stage_compat::context()) gs_ctx_destroy(gs_stage_compat::context());
    gs_stage_compat::context() = nullptr;
}

void setGlobalArgs(GlobalArgs* globalArgs) { gs_stage_compat::args() = *globalArgs; }

void setTileListArgs(TileListArgs* tileListArgs) { gs_stage_compat::tiles() = *tileListArgs; }

void evaluateSphericalHarmonics(CudaTimer& timer, int32_t count)
{
    using namespace gs_stage_compat;
    const gs_camera c = camera();
    const GlobalArgs& a = args();
    timer.start();
    report(gs_stage_sh(count, reinterpret_cast<const float*>(a.position), a.sphericalHarmonics,
                       a.sphericalHarmonicsCount, std::min(a.sphericalHarmonicsDegree, 2), &c,
                       reinterpret_cast<float*>(a.color), nullptr),
           "evaluateSphericalHarmonics");
    timer.stop();
}

void evaluateSplatClipData(CudaTimer& timer, int32_t count)
{
    using namespace gs_stage_compat;
    const gs_camera c = camera();
    const GlobalArgs& a = args();
    timer.start();
    report(gs_stage_project(count, reinterpret_cast<const float*>(a.position),
                            reinterpret_cast<const float*>(a.scaleAndRotation), &c,
                            reinterpret_cast<float*>(a.positionClipSpaceXY), a.positionClipSpaceZ,
                            reinterpret_cast<float*>(a.screenEllipse), reinterpret_cast<float*>(a.conic), nullptr),
           "evaluateSplatClipData");
    timer.stop();
}

int32_t buildTileList(CudaTimer& timer, int32_t /*numBlocks: the build sizes its own grids*/, int32_t tileListCapacity)
{
    using namespace gs_stage_compat;
    const gs_camera c = camera();
    const gs_render_cfg cfg = reference_cfg();
    const GlobalArgs& a = args();
    int64_t k = 0;
    timer.start();
    const int rc = gs_stage_build(ctx(), a.splatCount, reinterpret_cast<const float*>(a.positionClipSpaceXY),
                                  a.positionClipSpaceZ, reinterpret_cast<const float*>(a.screenEllipse), &c, &cfg,
                                  tiles().keys, tiles().values, tileListCapacity, &k, nullptr);
    timer.stop();
    if (rc == GS_ERR_CAPACITY) return tileListCapacity;  // truncated: the frame loop grows the lists
    report(rc, "buildTileList");
    return rc == GS_OK ? (int32_t)k : 0;
}

void sortTileList(CudaTimer& timer, int32_t tileListSize, void*& /*deviceTempStorage*/,
                  size_t& /*tempStorageSizeInBytes*/, DoubleBuffer<uint64_t>& keys, DoubleBuffer<int32_t>& values)
{
    using namespace gs_stage_compat;
    int32_t selector = 0;
    timer.start();
    // bits [0, 44): 12 tile bits + 32 depth bits (gaussian_render.cu:601)
    const int rc = report(gs_stage_sort(ctx(), tileListSize, 44, keys.current(), values.current(), keys.alternate(),
                                        values.alternate(), &selector, nullptr),
                          "sortTileList");
    timer.stop();
    if (rc == GS_OK && selector) {
        // the result is in the alternate buffers: make them current, as
        // CUB's DoubleBuffer does after an odd number of passes
        keys = DoubleBuffer<uint64_t>(keys.alternate(), keys.current());
        values = DoubleBuffer<int32_t>(values.alternate(), values.current());
    }
}

void evaluateTileRange(CudaTimer& timer, int32_t tileListSize)
{
    using namespace gs_stage_compat;
    timer.start();
    report(gs_stage_ranges(tileListSize, tiles().keys, k_TotalTiles, args().tileRange, nullptr), "evaluateTileRange");
    timer.stop();
}

void rasterizeTile(CudaTimer& timer)
{
    using namespace gs_stage_compat;
    const gs_camera c = camera();
    const gs_render_cfg cfg = reference_cfg();
    const GlobalArgs& a = args();
    timer.start();
    report(gs_stage_raster(&c, &cfg, a.tileRange, tiles().values, reinterpret_cast<const float*>(a.positionClipSpaceXY),
                           reinterpret_cast<const float*>(a.conic), reinterpret_cast<const float*>(a.color),
                           reinterpret_cast<uint8_t*>(a.backBuffer), nullptr),
           "rasterizeTile");
    timer.stop();
}
