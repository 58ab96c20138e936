// gs_stage_sort_noalloc: the tile-list sort with no device allocation.
//
// gs_stage_sort keeps its scratch (per-tile look-back words, digit
// histograms, tile counters, error word) in a gs_ctx that grows with the
// input, which means cudaMalloc on the first call and whenever the list
// grows.  Some callers cannot allocate: a renderer embedded in a host
// application whose device memory is handed out by its own pool or budget
// (every byte must come from that pool), and real-time frame loops that
// must not hit cudaMalloc/cudaFree, which synchronise the whole device and
// stall other streams mid-frame.  This entry point serves them: its scratch
// is one file-scope device array of fixed size, reserved when the library
// is loaded, and the call itself allocates nothing.
//
// Limits and sharing:
//  * at most kNoAllocMaxKeys (4,194,304) keys per call; larger inputs are
//    rejected with GS_ERR_CAPACITY.  The array takes a little over 2 MiB on
//    every GPU that loads the library, until the process exits;
//  * every call, from any thread or stream, uses the same array, which keeps
//    the previous call's contents: each call clears the words that must
//    start at zero.  Calls whose work overlaps on the GPU race and corrupt
//    each other's results: serialise them (one stream, or one call at a time);
//  * every call looks up the array's device address with
//    cudaGetSymbolAddress; the first call on a device also loads the module,
//    so make that first call before any stream capture.  After a
//    cudaDeviceReset the module comes back with a fresh array at a possibly
//    new address, which the next call picks up.
#include "gs_kernels.h"
#include "../../include/gs_b200.h"

#include <mutex>
#include <string>

namespace {

constexpr int64_t kNoAllocMaxKeys = 1ll << 22;
constexpr int64_t kNoAllocMaxTiles = kNoAllocMaxKeys / gs::kSortTile;  // 1024

struct NoAllocScratch {
    uint64_t status[kNoAllocMaxTiles * gs::kRadix];  // look-back words (epoch-tagged)
    uint32_t hist[gs::kMaxPasses * gs::kRadix];
    unsigned long long counters[gs::kMaxPasses];
    int err;
};

// Zero-initialised when the module loads; the status words are epoch-tagged,
// so zero reads as "not yet published" for every epoch.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;

struct DeviceState {
    NoAllocScratch* ptr = nullptr;  // device address of g_noalloc_scratch on this device
    uint32_t epoch = 1;
};

std::mutex g_mu;
DeviceState g_dev[kMaxDevices];
thread_local std::string g_err;

}  // namespace

extern "C" {

GS_API const char* gs_stage_sort_noalloc_error(void) { return g_err.c_str(); }

GS_API int64_t gs_stage_sort_noalloc_max_keys(void) { return kNoAllocMaxKeys; }

GS_API int gs_stage_sort_noalloc(int64_t num_keys, int32_t key_bits, uint64_t* d_keys, int32_t* d_values,
                                 uint64_t* d_keys_alt, int32_t* d_values_alt, int32_t* out_selector, void* stream)
{
    if (!out_selector || num_keys < 0 || key_bits < 1 || key_bits > 64) {
        g_err = "bad argument";
        return GS_ERR_INVALID;
    }
    *out_selector = 0;
    if (num_keys > kNoAllocMaxKeys) {
        g_err = "gs_stage_sort_noalloc: " + std::to_string(num_keys) + " keys exceed the fixed scratch limit of " +
                std::to_string(kNoAllocMaxKeys) + "; use gs_stage_sort";
        return GS_ERR_CAPACITY;
    }
    if (num_keys == 0) return GS_OK;
    if (!d_keys || !d_values || !d_keys_alt || !d_values_alt) {
        g_err = "null buffer";
        return GS_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        g_err = "no current CUDA device";
        return GS_ERR_NO_DEVICE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int passes = gs::sort_passes(key_bits);
    uint32_t epoch;
    NoAllocScratch* s;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        DeviceState& d = g_dev[dev];
        // with this device current: the host-side name of the array is not a
        // device address.  The first call on a device loads the module; later
        // calls only read the address back, and a changed address (the
        // context was reset, which reloads the module with a zeroed array)
        // restarts the epochs.
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            g_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return GS_ERR_CUDA;
        }
        if (d.ptr != static_cast<NoAllocScratch*>(p)) {
            d.ptr = static_cast<NoAllocScratch*>(p);
            d.epoch = 1;
        }
        s = d.ptr;
        if (d.epoch + (uint32_t)passes > 0xFFFFu) {
            // the 16-bit epoch wraps: clear the look-back words once
            if (cudaMemsetAsync(s->status, 0, sizeof(s->status), st) != cudaSuccess) {
                g_err = "status clear failed";
                return GS_ERR_CUDA;
            }
            d.epoch = 1;
        }
        epoch = d.epoch;
        d.epoch += (uint32_t)passes;
    }
    // the error word must start at zero (histograms and counters are cleared
    // by the sort launcher itself)
    if (cudaMemsetAsync(&s->err, 0, sizeof(int), st) != cudaSuccess) {
        g_err = "error word clear failed";
        return GS_ERR_CUDA;
    }
    gs::SortScratch ss;
    ss.hist = s->hist;
    ss.status = s->status;
    ss.counters = s->counters;
    ss.err = &s->err;
    ss.max_tiles = kNoAllocMaxTiles;
    const int done = gs::launch_sort(d_keys, d_values, d_keys_alt, d_values_alt, num_keys, nullptr, key_bits, ss, epoch,
                                     gs::device_sm_count(), st);
    cudaError_t e = cudaGetLastError();
    int err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, &s->err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        g_err = std::string("sort: ") + cudaGetErrorString(e);
        return GS_ERR_CUDA;
    }
    if (err) {
        g_err = "sort look-back timed out";
        return GS_ERR_DEVICE_TIMEOUT;
    }
    *out_selector = done % 2;
    return GS_OK;
}

}  // extern "C"
