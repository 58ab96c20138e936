// Continuous-batching render server of gs_b200 (declared in include/gs_b200.h).
//
// Several scenes stay resident in HBM.  Clients submit view requests
// (scene, camera, host output buffer) from any thread; a scheduler thread
// groups pending requests of one scene into a batched frame and hands it
// to the next free worker.  Each worker owns a context (its own frame
// buffers) and a CUDA stream, so batches of different workers overlap on
// the device; requests that arrive while batches run are admitted as soon
// as a worker frees up -- the batch is formed at dispatch time, not when
// the previous batch started.  Admission is against a device-memory
// budget: resident scenes plus every worker's frame buffers, with the
// next batch sized from the scene's observed keys per Gaussian.
//
// Latency of a request = submit -> its image is in the host buffer.
#include "../../include/gs_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id;
    int32_t scene;
    gs_camera cam;
    uint8_t* out;  // host, 4*W*H bytes
    Clock::time_point submitted;
};

struct Done {
    int status;
    double latency_ms;
};

struct SceneEntry {
    gs_scene* scene = nullptr;
    int64_t n = 0;
    int64_t bytes = 0;
    double keys_per_gaussian = 2.0;  // refined from every rendered batch
    double ms_per_mpixel = 0.0;      // batch time per million output pixels, refined likewise
};

struct Worker {
    gs_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::thread th;
    std::vector<Request> batch;
    bool has_batch = false;
    uint8_t* images = nullptr;  // device images of the current batch
    size_t image_bytes = 0;
};

}  // namespace

struct gs_server {
    int device = 0;
    gs_server_cfg cfg{};
    gs_ctx* owner = nullptr;  // scenes are created through this context
    std::map<int32_t, SceneEntry> scenes;
    int32_t next_scene = 0;
    std::deque<Request> pending;
    std::map<int64_t, Done> done;
    std::atomic<int64_t> next_id{1};
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::vector<std::unique_ptr<Worker>> workers;
    std::thread scheduler;
    bool stop = false;
    bool paused = false;  // gs_server_pause: requests queue, none is dispatched
    int64_t resident_bytes = 0;
    // statistics
    std::vector<double> latencies;
    int64_t views_done = 0, batches_done = 0, max_batch_seen = 0;
    Clock::time_point first_submit{}, last_done{};
    bool any_submit = false;
};

namespace {

size_t frame_bytes_estimate(const SceneEntry& s, const std::vector<Request>& reqs)
{
    size_t px = 0;
    for (const Request& r : reqs) px += 4 * (size_t)r.cam.width * r.cam.height;
    const double views = (double)reqs.size();
    // per (view, Gaussian) splat buffers + tile lists (keys/values, double
    // buffered) + images
    return (size_t)(views * s.n * 76.0 + views * s.n * s.keys_per_gaussian * 24.0) + px;
}

void worker_loop(gs_server* S, Worker* w)
{
    cudaSetDevice(S->device);
    for (;;) {
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_sched.wait(lk, [&] { return S->stop || w->has_batch; });
            if (!w->has_batch && S->stop) return;
            batch.swap(w->batch);
        }
        const Clock::time_point t0 = Clock::now();
        const int32_t sid = batch.front().scene;
        gs_scene* scene = nullptr;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            scene = S->scenes[sid].scene;
        }
        std::vector<gs_camera> cams;
        std::vector<size_t> offs;
        size_t total = 0;
        for (const Request& r : batch) {
            cams.push_back(r.cam);
            offs.push_back(total);
            total += 4 * (size_t)r.cam.width * r.cam.height;
        }
        int status = GS_OK;
        if (total > w->image_bytes) {
            // grow-only, with headroom, so steady state never allocates
            if (w->images) cudaFree(w->images);
            w->images = nullptr;
            w->image_bytes = 0;
            const size_t want = total + total / 2;
            if (cudaMalloc(&w->images, want) == cudaSuccess)
                w->image_bytes = want;
            else
                status = GS_ERR_OOM;
        }
        gs_stats st{};
        if (status == GS_OK) {
            std::vector<uint8_t*> outs;
            for (size_t o : offs) outs.push_back(w->images + o);
            status = gs_render_batch(w->ctx, scene, cams.data(), (int32_t)cams.size(), &S->cfg.render, outs.data(),
                                     &st, w->stream);
        }
        if (status == GS_OK) {
            // every view straight into its request's host buffer
            for (size_t k = 0; k < batch.size(); ++k) {
                const size_t b = 4 * (size_t)batch[k].cam.width * batch[k].cam.height;
                if (cudaMemcpyAsync(batch[k].out, w->images + offs[k], b, cudaMemcpyDeviceToHost, w->stream) !=
                    cudaSuccess)
                    status = GS_ERR_CUDA;
            }
            if (cudaStreamSynchronize(w->stream) != cudaSuccess) status = GS_ERR_CUDA;
        }
        const Clock::time_point now = Clock::now();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (const Request& r : batch) {
                const double ms = std::chrono::duration<double, std::milli>(now - r.submitted).count();
                S->done[r.id] = Done{status, ms};
                if (status == GS_OK) S->latencies.push_back(ms);
            }
            if (status == GS_OK) {
                SceneEntry& se = S->scenes[sid];
                if (se.n > 0 && st.num_keys > 0)
                    se.keys_per_gaussian = 0.5 * se.keys_per_gaussian +
                                           0.5 * (double)st.num_keys / ((double)se.n * (double)batch.size());
                const double mp = (double)total / 4.0 / 1e6;
                const double batch_ms = std::chrono::duration<double, std::milli>(now - t0).count();
                if (mp > 0) {
                    const double x = batch_ms / mp;
                    se.ms_per_mpixel = se.ms_per_mpixel > 0 ? 0.7 * se.ms_per_mpixel + 0.3 * x : x;
                }
                S->views_done += (int64_t)batch.size();
                S->batches_done += 1;
                S->max_batch_seen = std::max<int64_t>(S->max_batch_seen, (int64_t)batch.size());
                S->last_done = now;
            }
            w->has_batch = false;
        }
        S->cv_done.notify_all();
        S->cv_sched.notify_all();
    }
}

int64_t workers_bytes(gs_server* S)
{
    int64_t b = 0;
    for (auto& w : S->workers) b += gs_ctx_device_bytes(w->ctx);
    return b;
}

void scheduler_loop(gs_server* S)
{
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_sched.wait(lk, [&] {
            if (S->stop) return true;
            if (S->pending.empty() || S->paused) return false;
            for (auto& w : S->workers)
                if (!w->has_batch) return true;
            return false;
        });
        if (S->stop) return;
        if (S->paused) continue;
        Worker* free_w = nullptr;
        for (auto& w : S->workers)
            if (!w->has_batch) {
                free_w = w.get();
                break;
            }
        if (!free_w || S->pending.empty()) continue;
        // oldest request decides the scene; take that scene's pending
        // requests in arrival order up to the batch limit and the budget
        const int32_t sid = S->pending.front().scene;
        const SceneEntry& se = S->scenes[sid];
        std::vector<Request> batch;
        const int64_t headroom = S->cfg.budget_bytes - S->resident_bytes - workers_bytes(S);
        for (auto it = S->pending.begin(); it != S->pending.end();) {
            if ((int)batch.size() >= S->cfg.max_batch_views) break;
            if (it->scene != sid) {
                ++it;
                continue;
            }
            batch.push_back(*it);
            if (batch.size() > 1 && (int64_t)frame_bytes_estimate(se, batch) > std::max<int64_t>(headroom, 0)) {
                batch.pop_back();
                break;
            }
            // keep the batch within the latency target, from the scene's
            // measured cost per output pixel
            if (batch.size() > 1 && se.ms_per_mpixel > 0 && S->cfg.batch_target_ms > 0) {
                double mp = 0;
                for (const Request& q : batch) mp += (double)q.cam.width * q.cam.height / 1e6;
                if (mp * se.ms_per_mpixel > S->cfg.batch_target_ms) {
                    batch.pop_back();
                    break;
                }
            }
            it = S->pending.erase(it);
        }
        if (batch.empty()) {
            // a single view always goes (the budget only limits batch growth)
            batch.push_back(S->pending.front());
            S->pending.pop_front();
        }
        free_w->batch.swap(batch);
        free_w->has_batch = true;
        S->cv_sched.notify_all();
    }
}

}  // namespace

extern "C" {

GS_API void gs_server_default_cfg(gs_server_cfg* cfg)
{
    if (!cfg) return;
    cfg->budget_bytes = 150ll << 30;
    cfg->max_batch_views = 16;
    cfg->num_workers = 2;
    cfg->batch_target_ms = 8.0;
    gs_default_cfg(&cfg->render);
    // the batches a server forms rarely repeat (scene, view sizes and output
    // offsets all vary), so capturing graphs would mostly add capture time
    // to request latency: plain stream launches
    cfg->render.graph = 0;
}

GS_API int gs_server_create(int device, const gs_server_cfg* cfg, gs_server** out)
{
    if (!cfg || !out || cfg->num_workers < 1 || cfg->num_workers > 8 || cfg->max_batch_views < 1)
        return GS_ERR_INVALID;
    *out = nullptr;
    gs_server* S = new gs_server();
    S->device = device;
    S->cfg = *cfg;
    int rc = gs_ctx_create(device, &S->owner);
    if (rc) {
        delete S;
        return rc;
    }
    for (int i = 0; i < cfg->num_workers; ++i) {
        auto w = std::make_unique<Worker>();
        rc = gs_ctx_create(device, &w->ctx);
        if (rc == GS_OK && cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess)
            rc = GS_ERR_CUDA;
        if (rc) {
            if (w->ctx) gs_ctx_destroy(w->ctx);
            S->stop = true;
            for (auto& x : S->workers) {
                gs_ctx_destroy(x->ctx);
                cudaStreamDestroy(x->stream);
            }
            gs_ctx_destroy(S->owner);
            delete S;
            return rc;
        }
        S->workers.push_back(std::move(w));
    }
    for (auto& w : S->workers) w->th = std::thread(worker_loop, S, w.get());
    S->scheduler = std::thread(scheduler_loop, S);
    *out = S;
    return GS_OK;
}

GS_API int gs_server_destroy(gs_server* S)
{
    if (!S) return GS_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_sched.notify_all();
    if (S->scheduler.joinable()) S->scheduler.join();
    for (auto& w : S->workers)
        if (w->th.joinable()) w->th.join();
    for (auto& w : S->workers) {
        gs_ctx_destroy(w->ctx);
        cudaStreamDestroy(w->stream);
        if (w->images) cudaFree(w->images);
    }
    for (auto& kv : S->scenes) gs_scene_destroy(kv.second.scene);
    gs_ctx_destroy(S->owner);
    delete S;
    return GS_OK;
}

GS_API int gs_server_add_scene(gs_server* S, int64_t n, const float* h_position, const float* h_scale_rotation,
                               const float* h_color, const float* h_sh, int32_t sh_degree, int32_t* out_scene_id)
{
    if (!S || !out_scene_id) return GS_ERR_INVALID;
    const int64_t groups = (n + 255) / 256;
    const int64_t need = 32 * n + (h_color ? 16 * n : 0) +
                         (sh_degree > 0 ? (int64_t)4 * groups * 256 * 3 * (sh_degree + 1) * (sh_degree + 1) : 0);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->resident_bytes + need + workers_bytes(S) > S->cfg.budget_bytes) return GS_ERR_CAPACITY;
    }
    gs_scene* sc = nullptr;
    int rc = gs_scene_create(S->owner, n, h_position, h_scale_rotation, h_color, h_sh, sh_degree, &sc);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(S->mu);
    SceneEntry e;
    e.scene = sc;
    e.n = n;
    e.bytes = gs_scene_device_bytes(sc);
    S->resident_bytes += e.bytes;
    const int32_t id = S->next_scene++;
    S->scenes[id] = e;
    *out_scene_id = id;
    return GS_OK;
}

GS_API int gs_server_submit(gs_server* S, int32_t scene_id, const gs_camera* cam, uint8_t* h_rgba, int64_t* out_id)
{
    if (!S || !cam || !h_rgba || !out_id || cam->width <= 0 || cam->height <= 0) return GS_ERR_INVALID;
    Request r;
    r.scene = scene_id;
    r.cam = *cam;
    r.out = h_rgba;
    r.submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (!S->scenes.count(scene_id)) return GS_ERR_INVALID;
        r.id = S->next_id++;
        if (!S->any_submit) {
            S->first_submit = r.submitted;
            S->any_submit = true;
        }
        S->pending.push_back(r);
    }
    S->cv_sched.notify_all();
    *out_id = r.id;
    return GS_OK;
}

GS_API int gs_server_wait(gs_server* S, int64_t id, double timeout_ms, double* out_latency_ms)
{
    if (!S) return GS_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                        [&] { return S->done.count(id) > 0; });
    if (!ok) return GS_ERR_DEVICE_TIMEOUT;
    const Done d = S->done[id];
    S->done.erase(id);
    if (out_latency_ms) *out_latency_ms = d.latency_ms;
    return d.status;
}

GS_API int gs_server_cancel(gs_server* S, int64_t id)
{
    if (!S) return GS_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = std::find_if(S->pending.begin(), S->pending.end(), [&](const Request& r) { return r.id == id; });
        // already handed to a worker (its batch is on the device), finished,
        // or unknown: nothing to cancel
        if (it == S->pending.end()) return GS_ERR_INVALID;
        const double ms = std::chrono::duration<double, std::milli>(Clock::now() - it->submitted).count();
        S->done[id] = Done{GS_ERR_CANCELLED, ms};
        S->pending.erase(it);
    }
    S->cv_done.notify_all();
    return GS_OK;
}

GS_API int gs_server_pause(gs_server* S, int32_t paused)
{
    if (!S) return GS_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->paused = paused != 0;
    }
    S->cv_sched.notify_all();
    return GS_OK;
}

GS_API int gs_server_get_stats(gs_server* S, gs_server_stats* out)
{
    if (!S || !out) return GS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    std::vector<double> l = S->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
        if (l.empty()) return 0.0;
        const size_t k = std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5));
        return l[k];
    };
    out->views_done = S->views_done;
    out->batches_done = S->batches_done;
    out->max_batch = S->max_batch_seen;
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->mean_ms = l.empty() ? 0.0 : [&] {
        double s = 0;
        for (double x : l) s += x;
        return s / l.size();
    }();
    const double span = S->any_submit ? std::chrono::duration<double>(S->last_done - S->first_submit).count() : 0.0;
    out->views_per_s = span > 0 ? S->views_done / span : 0.0;
    out->resident_bytes = S->resident_bytes;
    out->frame_bytes = workers_bytes(S);
    out->pending = (int64_t)S->pending.size();
    return GS_OK;
}

GS_API int gs_server_reset_stats(gs_server* S)
{
    if (!S) return GS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    S->latencies.clear();
    S->views_done = S->batches_done = S->max_batch_seen = 0;
    S->any_submit = false;
    return GS_OK;
}

}  // extern "C"
