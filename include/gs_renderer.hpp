// gs_renderer.hpp — the reference's C++ renderer API over the gs_b200 C ABI.
//
// Mirrors RobinSongx/3DGaussianRenderer's public classes so a caller of
// core/renderer.h can switch by changing the include and linking
// libgs_b200.so:
//   gauss_render::RenderStats   core/types.h:26-33
//   gauss_render::Gaussian,
//   gauss_render::GaussianModel core/gaussian_model.h:11-41
//   gauss_render::LoadPly       core/ply_loader.h:13
//   gauss_render::Camera        core/camera.h:11-59 (+ GetFovY/GetZNear/GetZFar
//                               that core/renderer.cpp:18,28 calls)
//   gauss_render::Renderer      core/renderer.h:13-50
//   gauss_render::DrawPerformanceOverlay  app/perf_overlay.h:9-15
//   gauss_render::SaveImage     (headless: the frame to a PNG/PPM file in place
//                               of the OpenGL display, app/opengl_display.cpp)
// Vector arguments accept any type with x/y/z members (glm::vec3 included).
// Renderer::Render writes RGBA8 into a device buffer, like the reference's
// mapped PBO (row 0 = bottom).  Errors are reported through the int
// status of the C ABI: the methods return it instead of exiting.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gs_b200.h"

namespace gauss_render {

constexpr int kTileSize = 16;
constexpr int kScreenSize = 1024;
constexpr int kDefaultScreenWidth = 1024;
constexpr int kDefaultScreenHeight = 1024;
constexpr int kDefaultShBlockSize = 256;
constexpr int kTilesPerScreen = kScreenSize / kTileSize;
constexpr int kTotalTiles = kTilesPerScreen * kTilesPerScreen;

struct Vec2 {
    float x = 0, y = 0;
};
struct Vec3 {
    float x = 0, y = 0, z = 0;
};
struct Mat4 {
    float m[16] = {};  // column-major, m[col * 4 + row]
};

struct RenderStats {
    double sh_eval_ms = 0.0;
    double project_ms = 0.0;
    double build_tile_ms = 0.0;
    double sort_ms = 0.0;
    double raster_ms = 0.0;
    double total_ms = 0.0;
};

struct Gaussian {
    float position[3];
    float opacity;      // activated (sigmoid applied)
    float scale[3];     // activated (exp applied)
    float rotation[4];  // (w, x, y, z), normalised
    float color[3];     // DC colour
};

class GaussianModel {
  public:
    std::vector<Gaussian> gaussians;
    // Per Gaussian: 3*(sh_degree+1)^2 floats, RGB interleaved per coefficient.
    std::vector<float> sh_coefficients;
    int sh_degree = 0;
    int num_gaussians = 0;
    Vec3 bounds_min;
    Vec3 bounds_max;

    // Regroups sh_coefficients into [ceil(n/256)][coefficient][256] (the
    // coalesced layout of app/main.cpp:147-177; a TODO in the reference).
    void PreprocessSh()
    {
        const int sc = 3 * (sh_degree + 1) * (sh_degree + 1);
        const int64_t n = num_gaussians, groups = (n + 255) / 256;
        aligned_sh_.assign((size_t)groups * 256 * sc, 0.0f);
        if (sh_degree == 0 || sh_coefficients.size() < (size_t)n * sc) return;
        for (int64_t i = 0; i < n; ++i)
            for (int k = 0; k < sc; ++k)
                aligned_sh_[(size_t)(i / 256) * 256 * sc + (size_t)k * 256 + i % 256] = sh_coefficients[i * sc + k];
    }
    const std::vector<float>& GetAlignedSh() const { return aligned_sh_; }
    Vec3 GetBoundsMin() const { return bounds_min; }
    Vec3 GetBoundsMax() const { return bounds_max; }

    // Device layouts exactly as gs_ply_read produced them (empty for models
    // built by hand; UploadModel then encodes `gaussians`).
    std::vector<float> position4, scale_rotation4, color4;

  private:
    std::vector<float> aligned_sh_;
};

// Loads a 3DGS PLY (core/ply_loader.cpp:105-278).  Returns the number of
// Gaussians, 0 on failure (with a message on stdout, like the reference).
inline int LoadPly(const std::string& path, GaussianModel& model)
{
    int64_t n = 0;
    int32_t deg = 0;
    if (gs_ply_info(path.c_str(), &n, &deg) != GS_OK) {
        std::printf("Failed to parse PLY: %s\n", gs_ply_last_error());
        return 0;
    }
    const int sc = 3 * (deg + 1) * (deg + 1);
    const int64_t groups = (n + 255) / 256;
    model.position4.assign((size_t)n * 4, 0.0f);
    model.scale_rotation4.assign((size_t)n * 4, 0.0f);
    model.color4.assign((size_t)n * 4, 0.0f);
    std::vector<float> grouped(deg > 0 ? (size_t)groups * 256 * sc : 0);
    float bounds[6];
    if (gs_ply_read(path.c_str(), model.position4.data(), model.scale_rotation4.data(), model.color4.data(),
                    deg > 0 ? grouped.data() : nullptr, bounds) != GS_OK) {
        std::printf("Failed to parse PLY: %s\n", gs_ply_last_error());
        return 0;
    }
    model.num_gaussians = (int)n;
    model.sh_degree = deg;
    model.bounds_min = {bounds[0], bounds[1], bounds[2]};
    model.bounds_max = {bounds[3], bounds[4], bounds[5]};
    model.gaussians.resize((size_t)n);
    model.sh_coefficients.assign((size_t)n * sc, 0.0f);
    for (int64_t i = 0; i < n; ++i) {
        Gaussian& g = model.gaussians[(size_t)i];
        const float* p = &model.position4[(size_t)i * 4];
        const float* s = &model.scale_rotation4[(size_t)i * 4];
        const float* c = &model.color4[(size_t)i * 4];
        uint32_t bits;
        std::memcpy(&bits, &s[3], 4);
        for (int k = 0; k < 3; ++k) {
            g.position[k] = p[k];
            g.scale[k] = s[k];
            g.color[k] = c[k];
        }
        g.opacity = p[3];
        const float q[4] = {(float)((bits >> 24) & 0xFF), (float)((bits >> 16) & 0xFF), (float)((bits >> 8) & 0xFF),
                            (float)(bits & 0xFF)};
        g.rotation[0] = q[3] / 255.0f * 2.0f - 1.0f;  // w
        g.rotation[1] = q[0] / 255.0f * 2.0f - 1.0f;  // x
        g.rotation[2] = q[1] / 255.0f * 2.0f - 1.0f;  // y
        g.rotation[3] = q[2] / 255.0f * 2.0f - 1.0f;  // z
        if (deg > 0)
            for (int k = 0; k < sc; ++k)
                model.sh_coefficients[(size_t)i * sc + k] = grouped[(size_t)(i / 256) * 256 * sc + (size_t)k * 256 + i % 256];
    }
    model.PreprocessSh();
    std::printf("Loaded %d gaussians from %s\n", (int)n, path.c_str());
    return (int)n;
}

class Camera {
  public:
    Camera() { Update(); }

    void SetFovY(float fov_y_rad) { fov_y_ = fov_y_rad; Update(); }
    void SetResolution(int width, int height) { width_ = width; height_ = height; Update(); }
    void SetNearFar(float near_plane, float far_plane) { near_ = near_plane; far_ = far_plane; Update(); }
    template <class V>
    void SetPose(const V& position, const V& look_at)
    {
        eye_ = {position.x, position.y, position.z};
        target_ = {look_at.x, look_at.y, look_at.z};
        Update();
    }

    Mat4 GetView() const { Mat4 r; std::memcpy(r.m, c_.view, sizeof(r.m)); return r; }
    Mat4 GetProjection() const { return projection_; }
    Mat4 GetViewProjection() const
    {
        Mat4 r;
        for (int col = 0; col < 4; ++col)
            for (int row = 0; row < 4; ++row) {
                float s = 0;
                for (int k = 0; k < 4; ++k) s += projection_.m[k * 4 + row] * c_.view[col * 4 + k];
                r.m[col * 4 + row] = s;
            }
        return r;
    }
    Vec3 GetPosition() const { return eye_; }
    float GetAspect() const { return c_.aspect; }
    Vec2 GetFovCotangent() const { return {c_.fov_cotangent[0], c_.fov_cotangent[1]}; }
    Vec2 GetDepthScaleBias() const { return {c_.depth_scale_bias[0], c_.depth_scale_bias[1]}; }
    int GetWidth() const { return width_; }
    int GetHeight() const { return height_; }
    float GetFovY() const { return fov_y_; }
    float GetZNear() const { return near_; }
    float GetZFar() const { return far_; }
    const gs_camera& Native() const { return c_; }

  private:
    void Update()
    {
        const float e[3] = {eye_.x, eye_.y, eye_.z}, t[3] = {target_.x, target_.y, target_.z}, up[3] = {0, 1, 0};
        gs_camera_look_at(&c_, e, t, up, fov_y_, width_, height_, near_, far_);
        // glm::perspective (right-handed, clip z in [-1, 1])
        const float f = 1.0f / std::tan(fov_y_ * 0.5f);
        projection_ = Mat4{};
        projection_.m[0] = f / c_.aspect;
        projection_.m[5] = f;
        projection_.m[10] = -(far_ + near_) / (far_ - near_);
        projection_.m[11] = -1.0f;
        projection_.m[14] = -(2.0f * far_ * near_) / (far_ - near_);
    }

    gs_camera c_{};
    Mat4 projection_;
    Vec3 eye_{0.0f, 0.0f, 3.0f};
    Vec3 target_{0.0f, 0.0f, 0.0f};
    float fov_y_ = 50.0f * 3.14159265358979f / 180.0f;
    float near_ = 0.01f;
    float far_ = 100.0f;
    int width_ = kDefaultScreenWidth;
    int height_ = kDefaultScreenHeight;
};

class Renderer {
  public:
    Renderer() { gs_default_cfg(&cfg_); }
    ~Renderer()
    {
        if (scene_) gs_scene_destroy(scene_);
        if (ctx_) gs_ctx_destroy(ctx_);
    }
    Renderer(const Renderer&) = delete;
    Renderer& operator=(const Renderer&) = delete;

    // Options: gs_default_cfg() (full SH, T < 1e-4) unless changed; the
    // reference's own behaviour is {sh_max_degree 2, GS_TERM_REFERENCE}.
    void SetConfig(const gs_render_cfg& cfg) { cfg_ = cfg; }
    const gs_render_cfg& Config() const { return cfg_; }

    int UploadModel(const GaussianModel& model)
    {
        int rc = EnsureCtx();
        if (rc) return rc;
        if (scene_) gs_scene_destroy(scene_);
        scene_ = nullptr;
        const int64_t n = model.num_gaussians;
        std::vector<float> pos, sr, col;
        const float* P = model.position4.data();
        const float* S = model.scale_rotation4.data();
        const float* C = model.color4.data();
        if (model.position4.size() != (size_t)n * 4) {
            Encode(model, pos, sr, col);
            P = pos.data();
            S = sr.data();
            C = col.data();
        }
        std::vector<float> aligned;
        const float* sh = nullptr;
        if (model.sh_degree > 0) {
            if (!model.GetAlignedSh().empty()) {
                sh = model.GetAlignedSh().data();
            } else {
                GaussianModel tmp = model;
                tmp.PreprocessSh();
                aligned = tmp.GetAlignedSh();
                sh = aligned.data();
            }
        }
        return gs_scene_create(ctx_, n, P, S, C, sh, model.sh_degree, &scene_);
    }

    int Render(const Camera& camera, uint8_t* output_buffer, RenderStats& stats)
    {
        if (!ctx_ || !scene_) return GS_ERR_INVALID;
        gs_stats st{};
        const int rc = gs_render(ctx_, scene_, &camera.Native(), &cfg_, output_buffer, &st, nullptr);
        if (rc) return rc;
        stats.sh_eval_ms = st.sh_eval_ms;
        stats.project_ms = st.project_ms;
        stats.build_tile_ms = st.build_tile_ms;
        stats.sort_ms = st.sort_ms;
        stats.raster_ms = st.raster_ms;
        stats.total_ms = st.total_ms;
        return GS_OK;
    }

    // gs_autotune on this camera's view: the options' batching knobs become
    // the fastest timed ones (tile shape under per-pixel termination), and
    // the context remembers them for the view's (N, resolution) bucket.
    int Autotune(const Camera& camera, int iterations = 3)
    {
        if (!ctx_ || !scene_) return GS_ERR_INVALID;
        gs_render_cfg best{};
        const int rc = gs_autotune(ctx_, scene_, &camera.Native(), 1, &cfg_, iterations, &best, nullptr, nullptr, 0,
                                   nullptr, nullptr);
        if (rc == GS_OK) cfg_ = best;
        return rc;
    }

  private:
    int EnsureCtx() { return ctx_ ? GS_OK : gs_ctx_create(0, &ctx_); }

    // parsePly's per-vertex packing (ply_parser.cpp:375-389) for hand-built models
    static void Encode(const GaussianModel& m, std::vector<float>& pos, std::vector<float>& sr, std::vector<float>& col)
    {
        const size_t n = (size_t)m.num_gaussians;
        pos.resize(4 * n);
        sr.resize(4 * n);
        col.resize(4 * n);
        auto enc = [](float v) {
            v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
            return (uint32_t)(v * 255.0f);
        };
        for (size_t i = 0; i < n; ++i) {
            const Gaussian& g = m.gaussians[i];
            pos[4 * i + 0] = g.position[0];
            pos[4 * i + 1] = g.position[1];
            pos[4 * i + 2] = g.position[2];
            pos[4 * i + 3] = g.opacity;
            sr[4 * i + 0] = g.scale[0];
            sr[4 * i + 1] = g.scale[1];
            sr[4 * i + 2] = g.scale[2];
            const uint32_t bits = (enc((g.rotation[1] + 1.0f) * 0.5f) << 24) | (enc((g.rotation[2] + 1.0f) * 0.5f) << 16) |
                                  (enc((g.rotation[3] + 1.0f) * 0.5f) << 8) | enc((g.rotation[0] + 1.0f) * 0.5f);
            std::memcpy(&sr[4 * i + 3], &bits, 4);
            col[4 * i + 0] = g.color[0];
            col[4 * i + 1] = g.color[1];
            col[4 * i + 2] = g.color[2];
            col[4 * i + 3] = g.opacity;
        }
    }

    gs_ctx* ctx_ = nullptr;
    gs_scene* scene_ = nullptr;
    gs_render_cfg cfg_{};
};

// app/perf_overlay.h:9-15: the statistics text drawn into the image.  The
// buffer is the device RGBA8 image Renderer::Render wrote (the reference's
// is the mapped host PBO); asynchronous on `stream`.
inline int DrawPerformanceOverlay(uint8_t* buffer, int width, int height, int num_gaussians, const RenderStats& stats,
                                  double fps, void* stream = nullptr)
{
    gs_stats s{};
    s.sh_eval_ms = stats.sh_eval_ms;
    s.project_ms = stats.project_ms;
    s.build_tile_ms = stats.build_tile_ms;
    s.sort_ms = stats.sort_ms;
    s.raster_ms = stats.raster_ms;
    s.total_ms = stats.total_ms;
    return gs_draw_stats(buffer, width, height, num_gaussians, &s, fps, stream);
}

// Headless stand-in for the reference's on-screen display: writes a host
// RGBA8 frame (row 0 = bottom, as Render leaves it) to `path`, top row
// first, as PNG when the name ends in ".png", else as binary PPM.
inline int SaveImage(const std::string& path, const uint8_t* host_rgba, int width, int height)
{
    const bool png = path.size() >= 4 && (path.compare(path.size() - 4, 4, ".png") == 0 ||
                                          path.compare(path.size() - 4, 4, ".PNG") == 0);
    return png ? gs_write_png(path.c_str(), host_rgba, width, height)
               : gs_write_ppm(path.c_str(), host_rgba, width, height);
}

}  // namespace gauss_render
