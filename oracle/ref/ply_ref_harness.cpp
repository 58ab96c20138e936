// Reference harness for PLY ingest: a C-ABI around the reference's own
// parsePly (core/ply_parser.cpp:241-393), compiled from the reference
// sources into oracle/_ref/libplyref.so by oracle/ref/build_ref.sh.
// TEST INFRASTRUCTURE ONLY: the tests compare gs_ply_read against it.
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "ply_parser.h"

namespace {
std::vector<float4> g_pos, g_sr, g_col;
std::vector<float> g_sh;
int g_deg = 0, g_count = 0, g_n = 0;
glm::vec3 g_min, g_max;
std::string g_err;
}  // namespace

extern "C" {

// Parses `path`; returns the vertex count (or -1, message in plyref_error()).
int plyref_parse(const char* path)
{
    try {
        g_pos.clear();
        g_sr.clear();
        g_col.clear();
        g_sh.clear();
        g_n = parsePly(path, g_pos, g_sr, g_col, g_sh, g_deg, g_count, g_min, g_max);
        return g_n;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

const char* plyref_error() { return g_err.c_str(); }

// deg, shCount (3 + f_rest count), bounds[6]
void plyref_info(int* deg, int* sh_count, float* bounds)
{
    *deg = g_deg;
    *sh_count = g_count;
    bounds[0] = g_min.x;
    bounds[1] = g_min.y;
    bounds[2] = g_min.z;
    bounds[3] = g_max.x;
    bounds[4] = g_max.y;
    bounds[5] = g_max.z;
}

// pos/sr/col: 4*n floats; sh: n*sh_count floats (per-Gaussian, RGB
// interleaved as parsePly leaves them), may be null.
void plyref_copy(float* pos, float* sr, float* col, float* sh)
{
    std::memcpy(pos, g_pos.data(), g_pos.size() * sizeof(float4));
    std::memcpy(sr, g_sr.data(), g_sr.size() * sizeof(float4));
    std::memcpy(col, g_col.data(), g_col.size() * sizeof(float4));
    if (sh && !g_sh.empty()) std::memcpy(sh, g_sh.data(), g_sh.size() * sizeof(float));
}
}
