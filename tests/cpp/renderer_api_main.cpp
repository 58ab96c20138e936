// Drives the C++ renderer API (include/gs_renderer.hpp) the way a caller of
// the reference's core/renderer.h would: LoadPly -> UploadModel -> Render
// into a device RGBA buffer, then writes the image bytes to a file.
//   renderer_api_main <ply> <out.raw> <width> <height> <reference-mode 0|1> [autotune 0|1]
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gs_renderer.hpp"

struct V3 {
    float x, y, z;
};

int main(int argc, char** argv)
{
    if (argc < 6) return 2;
    gauss_render::GaussianModel model;
    if (gauss_render::LoadPly(argv[1], model) <= 0) return 3;
    const int w = std::atoi(argv[3]), h = std::atoi(argv[4]);
    gauss_render::Camera cam;
    cam.SetResolution(w, h);
    cam.SetFovY((float)(60.0 * 3.14159265358979323846 / 180.0));
    cam.SetNearFar(0.1f, 100.0f);
    cam.SetPose(V3{0.3f, 0.2f, 3.0f}, V3{0.0f, 0.0f, 0.0f});
    gauss_render::Renderer renderer;
    if (std::atoi(argv[5])) {
        gs_render_cfg cfg;
        gs_default_cfg(&cfg);
        cfg.sh_max_degree = 2;
        cfg.termination = GS_TERM_REFERENCE;
        renderer.SetConfig(cfg);
    }
    if (renderer.UploadModel(model) != GS_OK) return 4;
    if (argc > 6 && std::atoi(argv[6])) {
        if (renderer.Autotune(cam) != GS_OK) return 8;
        std::printf("tuned tile %dx%d\n", renderer.Config().tile_w, renderer.Config().tile_h);
    }
    uint8_t* d = nullptr;
    if (cudaMalloc(&d, (size_t)w * h * 4) != cudaSuccess) return 5;
    gauss_render::RenderStats stats;
    if (renderer.Render(cam, d, stats) != GS_OK) return 6;
    std::vector<uint8_t> img((size_t)w * h * 4);
    cudaMemcpy(img.data(), d, img.size(), cudaMemcpyDeviceToHost);
    cudaFree(d);
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 7;
    std::fwrite(img.data(), 1, img.size(), f);
    std::fclose(f);
    if (gauss_render::SaveImage(std::string(argv[2]) + ".png", img.data(), w, h) != GS_OK) return 9;
    std::printf("stats project %.3f build %.3f sort %.3f raster %.3f total %.3f ms\n", stats.project_ms,
                stats.build_tile_ms, stats.sort_ms, stats.raster_ms, stats.total_ms);
    return 0;
}
