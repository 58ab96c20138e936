// PLY ingest and export for gs_b200 (replaces parsePly/savePly,
// core/ply_parser.cpp:15-393, and LoadPly, core/ply_loader.cpp:105-278).
//
// The file is memory-mapped (no copy of the vertex data, no zero-filled
// staging buffer) and the vertex records are transformed in parallel (one
// std::thread per hardware thread over contiguous vertex ranges, each
// faulting in its own part of the file), straight into the device
// layouts: position/opacity, scale + quantised rotation, DC colour, and
// the SH coefficients interleaved per coefficient and regrouped by 256
// (app/main.cpp:147-177).  The per-vertex transforms are the reference's:
// normalised quaternion -> 8-bit encoding, exp(scale), sigmoid(opacity),
// DC * C0 + 0.5.  This file is compiled with -ffp-contract=off so its
// float arithmetic matches the reference host code (no contraction).
#include "../../include/gs_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace {

thread_local std::string g_ply_error;

struct PlyHeader {
    std::vector<std::string> props;
    int64_t count = -1;
    size_t data_offset = 0;
};

// parseHeader (ply_parser.cpp:15-100): binary_little_endian, one vertex
// element, float properties only, no duplicates, at most 256 header lines.
PlyHeader parse_header(std::ifstream& in)
{
    PlyHeader h;
    bool little = false;
    std::string line;
    int iteration = 0;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::stringstream ss(line);
        std::string word;
        if (!(ss >> word)) throw std::invalid_argument("Unexpected empty line.");
        if (word == "ply") continue;
        if (word == "format") {
            little = (ss >> word) && word == "binary_little_endian";
        } else if (word == "element") {
            if (!((ss >> word) && word == "vertex")) throw std::invalid_argument("Unexpected element type.");
            if (!(ss >> word)) throw std::invalid_argument("Unexpected element count.");
            h.count = std::stoll(word);
        } else if (word == "property") {
            if (!((ss >> word) && word == "float"))
                throw std::invalid_argument("Unexpected property format, expected float.");
            if (!(ss >> word)) throw std::invalid_argument("Unexpected property, missing name.");
            if (std::find(h.props.begin(), h.props.end(), word) != h.props.end())
                throw std::invalid_argument("Duplicated property \"" + word + "\".");
            h.props.push_back(word);
        } else if (word == "end_header") {
            if (!little || h.count < 0) throw std::invalid_argument("Invalid header. Format or vertex count not found.");
            h.data_offset = (size_t)in.tellg();
            return h;
        }
        if (++iteration > 256) throw std::invalid_argument("Invalid header. End not found.");
    }
    throw std::invalid_argument("Invalid header. End not found.");
}

int index_of(const PlyHeader& h, const std::string& name)
{
    auto it = std::find(h.props.begin(), h.props.end(), name);
    if (it == h.props.end()) throw std::invalid_argument("Missing property \"" + name + "\".");
    return (int)(it - h.props.begin());
}

struct Layout {
    int off[14];
    std::vector<int> rest;
    int degree = 0;
    int sh_count = 3;
};

// f_rest_* count -> SH degree (ply_parser.cpp:275-309)
Layout layout_of(const PlyHeader& h)
{
    Layout L;
    const char* names[14] = {"x", "y", "z", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2",
                             "f_dc_0", "f_dc_1", "f_dc_2", "opacity"};
    for (int i = 0; i < 14; ++i) L.off[i] = index_of(h, names[i]);
    for (int k = 0;; ++k) {
        auto it = std::find(h.props.begin(), h.props.end(), "f_rest_" + std::to_string(k));
        if (it == h.props.end()) break;
        L.rest.push_back((int)(it - h.props.begin()));
    }
    const int extra = (int)L.rest.size();
    int expected = 0;
    L.degree = 0;
    while (expected < extra) {
        expected += (2 * (L.degree + 1) + 1) * 3;
        ++L.degree;
    }
    if (expected != extra)
        throw std::invalid_argument("Expected degree " + std::to_string(L.degree) + ", " + std::to_string(expected) +
                                    " extra spherical harmonics. Found " + std::to_string(extra) + ".");
    L.sh_count = extra + 3;
    if (L.degree > 3) throw std::invalid_argument("SH degree above 3 is not supported.");
    return L;
}

// sigmoid (ply_parser.cpp:10-13) calls the unqualified C exp on a float,
// which is the double-precision exp: the expression is evaluated in double
// and rounded to float once, on return.
inline float sigmoidf(float x) { return (float)(1.0 / (1.0 + std::exp((double)(-x)))); }

inline float clamp01(float v) { return std::min(std::max(v, 0.0f), 1.0f); }

// encodeVec4 (ply_parser.cpp:231-239)
inline uint32_t encode_vec4(float x, float y, float z, float w)
{
    return ((uint32_t)(clamp01(x) * 255.0f) << 24u) | ((uint32_t)(clamp01(y) * 255.0f) << 16u) |
           ((uint32_t)(clamp01(z) * 255.0f) << 8u) | ((uint32_t)(clamp01(w) * 255.0f));
}

template <class F>
void parallel_for(int64_t n, F&& f)
{
    const int nt = (int)std::max<unsigned>(1, std::min<unsigned>(std::thread::hardware_concurrency(), 64));
    if (n < 65536 || nt == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) {
        const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
        th.emplace_back([&f, lo, hi] { f(lo, hi); });
    }
    for (auto& x : th) x.join();
}

// A read-only mapping of the whole file; the vertex data starts at
// `data`, at any byte offset (values are read with memcpy).
struct PlyFile {
    PlyHeader h;
    Layout L;
    const char* map = nullptr;
    size_t map_bytes = 0;
    const char* data = nullptr;  // count x props little-endian floats
    PlyFile() = default;
    PlyFile(const PlyFile&) = delete;
    PlyFile& operator=(const PlyFile&) = delete;
    ~PlyFile()
    {
        if (map) munmap(const_cast<char*>(map), map_bytes);
    }
    // property k of vertex i
    float at(int64_t i, int k) const
    {
        float v;
        std::memcpy(&v, data + ((size_t)i * h.props.size() + (size_t)k) * sizeof(float), sizeof(float));
        return v;
    }
};

void read_ply(const char* path, bool with_data, PlyFile& f)
{
    {
        std::ifstream in(path, std::ios::binary);
        if (!in.is_open()) throw std::invalid_argument(std::string("cannot open ") + path);
        f.h = parse_header(in);
    }
    f.L = layout_of(f.h);
    if (!with_data) return;
    const size_t bytes = (size_t)f.h.count * f.h.props.size() * sizeof(float);
    const int fd = open(path, O_RDONLY);
    if (fd < 0) throw std::invalid_argument(std::string("cannot open ") + path);
    struct stat sb;
    if (fstat(fd, &sb) != 0 || (size_t)sb.st_size < f.h.data_offset + bytes) {
        close(fd);
        throw std::invalid_argument("truncated vertex data");
    }
    if (bytes == 0) {
        close(fd);
        return;
    }
    void* m = mmap(nullptr, (size_t)sb.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);  // the mapping keeps the file
    if (m == MAP_FAILED) throw std::invalid_argument(std::string("cannot map ") + path);
    f.map = static_cast<const char*>(m);
    f.map_bytes = (size_t)sb.st_size;
    f.data = f.map + f.h.data_offset;
}

}  // namespace

extern "C" {

GS_API int gs_ply_info(const char* path, int64_t* out_n, int32_t* out_sh_degree)
{
    try {
        if (!path) return GS_ERR_INVALID;
        PlyFile f;
        read_ply(path, false, f);
        if (out_n) *out_n = f.h.count;
        if (out_sh_degree) *out_sh_degree = f.L.degree;
        return GS_OK;
    } catch (const std::exception& e) {
        g_ply_error = e.what();
        return GS_ERR_INVALID;
    }
}

GS_API const char* gs_ply_last_error(void) { return g_ply_error.c_str(); }

GS_API int gs_ply_read(const char* path, float* h_position, float* h_scale_rotation, float* h_color,
                       float* h_sh_grouped, float* bounds)
{
    try {
        if (!path) return GS_ERR_INVALID;
        PlyFile f;
        read_ply(path, true, f);
        const int64_t n = f.h.count;
        const Layout& L = f.L;
        const int sc = L.sh_count;
        const int rgb = (sc - 3) / 3;
        parallel_for(n, [&](int64_t lo, int64_t hi) {
            for (int64_t i = lo; i < hi; ++i) {
                const auto r = [&f, i](int k) { return f.at(i, k); };
                // glm::quat(w = rot_0, x = rot_1, y = rot_2, z = rot_3), normalised
                float qw = r(L.off[3]), qx = r(L.off[4]), qy = r(L.off[5]), qz = r(L.off[6]);
                const float len = std::sqrt((qw * qw + qx * qx) + (qy * qy + qz * qz));
                if (len <= 0.0f) {
                    qw = 1.0f;
                    qx = qy = qz = 0.0f;
                } else {
                    const float inv = 1.0f / len;
                    qw *= inv;
                    qx *= inv;
                    qy *= inv;
                    qz *= inv;
                }
                const float opacity = sigmoidf(r(L.off[13]));
                if (h_position) {
                    float* p = h_position + 4 * i;
                    p[0] = r(L.off[0]);
                    p[1] = r(L.off[1]);
                    p[2] = r(L.off[2]);
                    p[3] = opacity;
                }
                if (h_scale_rotation) {
                    float* s = h_scale_rotation + 4 * i;
                    s[0] = std::exp(r(L.off[7]));
                    s[1] = std::exp(r(L.off[8]));
                    s[2] = std::exp(r(L.off[9]));
                    const uint32_t bits = encode_vec4((qx + 1.0f) * 0.5f, (qy + 1.0f) * 0.5f, (qz + 1.0f) * 0.5f,
                                                      (qw + 1.0f) * 0.5f);
                    std::memcpy(&s[3], &bits, 4);
                }
                if (h_color) {
                    const float C0 = 0.28209479177387814f;
                    float* c = h_color + 4 * i;
                    c[0] = r(L.off[10]) * C0 + 0.5f;
                    c[1] = r(L.off[11]) * C0 + 0.5f;
                    c[2] = r(L.off[12]) * C0 + 0.5f;
                    c[3] = opacity;
                }
                if (h_sh_grouped && L.degree > 0) {
                    // [group][coefficient][256]; coefficient k holds RGB at 3k..3k+2,
                    // f_rest is channel-major in the file (ply_parser.cpp:332-348)
                    const int64_t g = i / 256, t = i % 256;
                    float* base = h_sh_grouped + (size_t)g * 256 * sc + t;
                    base[0 * 256] = r(L.off[10]);
                    base[1 * 256] = r(L.off[11]);
                    base[2 * 256] = r(L.off[12]);
                    for (int j = 0; j < rgb; ++j)
                        for (int c = 0; c < 3; ++c) base[(size_t)(3 + 3 * j + c) * 256] = r(L.rest[c * rgb + j]);
                }
            }
        });
        if (h_sh_grouped && L.degree > 0) {
            // zero the padding of the last group
            const int64_t groups = (n + 255) / 256;
            for (int64_t i = n; i < groups * 256; ++i) {
                const int64_t g = i / 256, t = i % 256;
                for (int k = 0; k < sc; ++k) h_sh_grouped[(size_t)g * 256 * sc + (size_t)k * 256 + t] = 0.0f;
            }
        }
        if (bounds) {
            // boundsMin/Max (ply_parser.cpp:351-381); the max starts at the
            // smallest positive float, as in the reference
            float mn[3], mx[3];
            for (int c = 0; c < 3; ++c) {
                mn[c] = std::numeric_limits<float>::max();
                mx[c] = std::numeric_limits<float>::min();
            }
            for (int64_t i = 0; i < n; ++i)
                for (int c = 0; c < 3; ++c) {
                    const float v = f.at(i, L.off[c]);
                    mn[c] = (v < mn[c]) ? v : mn[c];
                    mx[c] = (mx[c] < v) ? v : mx[c];
                }
            for (int c = 0; c < 3; ++c) {
                bounds[c] = mn[c];
                bounds[3 + c] = mx[c];
            }
        }
        return GS_OK;
    } catch (const std::exception& e) {
        g_ply_error = e.what();
        return GS_ERR_INVALID;
    }
}

GS_API int gs_ply_write(const char* path, int64_t n, const float* h_position, const float* h_scale_rotation,
                        const float* h_color, const float* h_sh_grouped, int32_t sh_degree)
{
    // savePly (ply_parser.cpp:143-219), extended with f_rest_* for SH scenes.
    if (!path || n <= 0 || !h_position || !h_scale_rotation || sh_degree < 0 || sh_degree > 3)
        return GS_ERR_INVALID;
    if (sh_degree == 0 && !h_color) return GS_ERR_INVALID;
    if (sh_degree > 0 && !h_sh_grouped) return GS_ERR_INVALID;
    std::ofstream out(path, std::ios::binary);
    if (!out.is_open()) return GS_ERR_INVALID;
    const int sc = 3 * (sh_degree + 1) * (sh_degree + 1);
    const int rgb = (sc - 3) / 3;
    out << "ply\nformat binary_little_endian 1.0\nelement vertex " << n << "\n";
    const char* names[] = {"x", "y", "z", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2",
                           "f_dc_0", "f_dc_1", "f_dc_2"};
    for (const char* nm : names) out << "property float " << nm << "\n";
    for (int k = 0; k < 3 * rgb; ++k) out << "property float f_rest_" << k << "\n";
    out << "property float opacity\nend_header\n";
    const float C0 = 0.28209479177387814f;
    std::vector<float> rec(14 + 3 * rgb);
    for (int64_t i = 0; i < n; ++i) {
        const float* p = h_position + 4 * i;
        const float* s = h_scale_rotation + 4 * i;
        uint32_t bits;
        std::memcpy(&bits, &s[3], 4);
        float q[4];
        for (int c = 0; c < 4; ++c) q[c] = (float)((bits >> (24 - 8 * c)) & 0xFFu) / 255.0f * 2.0f - 1.0f;
        size_t k = 0;
        rec[k++] = p[0];
        rec[k++] = p[1];
        rec[k++] = p[2];
        // rot_0..3 = (w, x, y, z), the order parsePly reads (ply_parser.cpp:360-364);
        // the reference's savePly writes (x, y, z, w) there instead, so its
        // files do not read back with the same rotation
        rec[k++] = q[3];
        rec[k++] = q[0];
        rec[k++] = q[1];
        rec[k++] = q[2];
        rec[k++] = std::log(s[0]);
        rec[k++] = std::log(s[1]);
        rec[k++] = std::log(s[2]);
        if (sh_degree > 0) {
            const int64_t g = i / 256, t = i % 256;
            const float* base = h_sh_grouped + (size_t)g * 256 * sc + t;
            rec[k++] = base[0];
            rec[k++] = base[256];
            rec[k++] = base[512];
            for (int c = 0; c < 3; ++c)
                for (int j = 0; j < rgb; ++j) rec[k++] = base[(size_t)(3 + 3 * j + c) * 256];
        } else {
            for (int c = 0; c < 3; ++c) rec[k++] = (h_color[4 * i + c] - 0.5f) / C0;
        }
        float o = std::min(std::max(p[3], 0.001f), 0.999f);
        rec[k++] = std::log(o / (1.0f - o));
        out.write(reinterpret_cast<const char*>(rec.data()), (std::streamsize)(k * sizeof(float)));
    }
    return out.good() ? GS_OK : GS_ERR_INVALID;
}

}  // extern "C"
