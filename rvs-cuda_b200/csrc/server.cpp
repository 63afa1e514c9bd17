// Serving loop: virtual-camera requests on resident scenes, continuous
// batching over independent lanes, admission by an HBM budget.
//
// The reference renders the frames of a configuration one after another
// (Application::execute, rvs/src/Application.cpp:53-65).  Here requests
// arrive at any time.  A worker thread owns `lanes` batch cores, each with
// its own stream: whenever a lane is free and requests are waiting, it
// launches all of them that fit (up to the batch size, in arrival order,
// while the workspace bytes of the requests in flight stay within the
// budget), so requests that arrive while others run join the next free
// lane instead of waiting for a full batch, and the lanes' work overlaps on
// the device.  Completion is detected by polling each lane's event; every
// request records its submit, launch and completion times.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "camera.hpp"
#include "engine.hpp"
#include "frontend.hpp"
#include "rvsb.h"

using namespace rvsb;

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
    uint64_t id;
    int scene;
    SlotRequest req;
    size_t bytes;
    double submit_s;
};

struct Lane {
    std::unique_ptr<BatchCore> core;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<Pending> reqs;
    double start_s = 0.0;
    size_t bytes = 0;
};

}  // namespace

struct rvsb_server {
    rvsb_context* ctx = nullptr;
    int max_batch = 1;
    size_t budget = 0;
    std::vector<rvsb_scene*> scenes;
    std::vector<std::unique_ptr<Lane>> lanes;
    Clock::time_point epoch = Clock::now();

    std::mutex mu;
    std::condition_variable cv;
    std::deque<Pending> pending;
    std::vector<rvsb_request_result> finished;
    size_t in_flight_bytes = 0;
    int in_flight_requests = 0;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    std::string worker_error;

    double now() const { return std::chrono::duration<double>(Clock::now() - epoch).count(); }
    void loop();
};

void rvsb_server::loop() {
    cudaSetDevice(ctx->device);
    std::vector<SlotRequest> batch;
    while (true) {
        bool any_busy = false;
        bool progressed = false;
        // Retire finished lanes.
        for (auto& lp : lanes) {
            Lane& L = *lp;
            if (!L.busy) continue;
            const cudaError_t q = cudaEventQuery(L.done);
            if (q == cudaErrorNotReady) {
                any_busy = true;
                continue;
            }
            const double t = now();
            std::lock_guard<std::mutex> lock(mu);
            for (const Pending& p : L.reqs) {
                rvsb_request_result r{};
                r.id = p.id;
                r.status = q == cudaSuccess ? RVSB_OK : RVSB_E_CUDA;
                r.batch_size = (int32_t)L.reqs.size();
                r.submit_s = p.submit_s;
                r.start_s = L.start_s;
                r.done_s = t;
                finished.push_back(r);
            }
            if (q != cudaSuccess) cudaGetLastError();
            in_flight_bytes -= L.bytes;
            in_flight_requests -= (int)L.reqs.size();
            L.reqs.clear();
            L.bytes = 0;
            L.busy = false;
            progressed = true;
        }
        // Admit waiting requests to free lanes.
        for (auto& lp : lanes) {
            Lane& L = *lp;
            if (L.busy) continue;
            {
                std::lock_guard<std::mutex> lock(mu);
                while (!pending.empty() && (int)L.reqs.size() < max_batch) {
                    const Pending& p = pending.front();
                    if (in_flight_bytes + L.bytes + p.bytes > budget && (in_flight_bytes + L.bytes) > 0) break;
                    L.bytes += p.bytes;
                    L.reqs.push_back(p);
                    pending.pop_front();
                }
                in_flight_bytes += L.bytes;
                in_flight_requests += (int)L.reqs.size();
            }
            if (L.reqs.empty()) {
                L.bytes = 0;
                break;  // nothing admissible: later lanes would admit nothing either
            }
            HostRange range("rvsb: serve (launch a lane's batch)");
            batch.clear();
            for (const Pending& p : L.reqs) batch.push_back(p.req);
            L.start_s = now();
            try {
                L.core->run(batch.data(), (int)batch.size(), L.stream);
                check(cudaEventRecord(L.done, L.stream), "record completion");
            } catch (const std::exception& e) {
                std::lock_guard<std::mutex> lock(mu);
                worker_error = e.what();
                for (const Pending& p : L.reqs) {
                    rvsb_request_result r{};
                    r.id = p.id;
                    r.status = RVSB_E_CUDA;
                    r.submit_s = p.submit_s;
                    r.start_s = r.done_s = now();
                    finished.push_back(r);
                }
                in_flight_bytes -= L.bytes;
                in_flight_requests -= (int)L.reqs.size();
                L.reqs.clear();
                L.bytes = 0;
                continue;
            }
            L.busy = true;
            any_busy = true;
            progressed = true;
        }
        std::unique_lock<std::mutex> lock(mu);
        if (stop && pending.empty() && in_flight_requests == 0) break;
        if (progressed) continue;
        if (any_busy) {
            // Lanes in flight: poll again shortly.
            lock.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        } else {
            cv.wait_for(lock, std::chrono::milliseconds(50),
                        [&] { return stop || !pending.empty(); });
        }
    }
}

extern "C" {

rvsb_status rvsb_server_create(rvsb_context* ctx, int lanes, int max_batch, size_t hbm_budget_bytes,
                               rvsb_server** out) {
    if (!ctx || !out || lanes <= 0 || lanes > 64 || max_batch <= 0 || max_batch > 256) return RVSB_E_ARG;
    *out = nullptr;
    try {
        check(cudaSetDevice(ctx->device), "cudaSetDevice");
        auto s = std::make_unique<rvsb_server>();
        s->ctx = ctx;
        s->max_batch = max_batch;
        s->budget = hbm_budget_bytes ? hbm_budget_bytes : ctx->budget;
        for (int k = 0; k < lanes; ++k) {
            auto L = std::make_unique<Lane>();
            L->core = std::make_unique<BatchCore>(ctx, max_batch);
            check(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            check(cudaEventCreateWithFlags(&L->done, cudaEventDisableTiming), "cudaEventCreate");
            s->lanes.push_back(std::move(L));
        }
        rvsb_server* raw = s.get();
        s->worker = std::thread([raw] { raw->loop(); });
        *out = s.release();
        return RVSB_OK;
    } catch (const BudgetError& e) {
        ctx->last_error = e.what();
        return RVSB_E_OOM_BUDGET;
    } catch (const std::exception& e) {
        ctx->last_error = e.what();
        return RVSB_E_CUDA;
    }
}

rvsb_status rvsb_server_add_scene(rvsb_server* s, rvsb_scene* scene, int* scene_id) {
    if (!s || !scene || !scene_id || scene->ctx != s->ctx) return RVSB_E_ARG;
    for (size_t v = 0; v < scene->cams.size(); ++v)
        if (!scene->uploaded[v]) {
            s->ctx->last_error = "input view " + std::to_string(v) + " was not uploaded";
            return RVSB_E_ARG;
        }
    std::lock_guard<std::mutex> lock(s->mu);
    s->scenes.push_back(scene);
    *scene_id = (int)s->scenes.size() - 1;
    return RVSB_OK;
}

rvsb_status rvsb_server_reserve(rvsb_server* s, int scene_id, int max_width, int max_height) {
    if (!s || max_width <= 0 || max_height <= 0) return RVSB_E_ARG;
    rvsb_scene* scene;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (scene_id < 0 || scene_id >= (int)s->scenes.size()) return RVSB_E_NOT_FOUND;
        if (!s->pending.empty() || s->in_flight_requests > 0) return RVSB_E_BUSY;
        scene = s->scenes[scene_id];
    }
    try {
        check(cudaSetDevice(s->ctx->device), "cudaSetDevice");
        for (auto& L : s->lanes)
            for (int k = 0; k < L->core->slots(); ++k) L->core->workspace(k).ensure(s->ctx, scene, max_width, max_height);
        return RVSB_OK;
    } catch (const BudgetError& e) {
        s->ctx->last_error = e.what();
        return RVSB_E_OOM_BUDGET;
    } catch (const std::exception& e) {
        s->ctx->last_error = e.what();
        return RVSB_E_CUDA;
    }
}

rvsb_status rvsb_server_submit(rvsb_server* s, int scene_id, const rvsb_camera* virt,
                               const rvsb_synth_params* params, const rvsb_yuv420* out, uint64_t* request_id) {
    if (!s || !virt || !params || !out || !out->y || !out->u || !out->v) return RVSB_E_ARG;
    if (const char* why = camera_problem(*virt, true)) {
        s->ctx->last_error = std::string("virtual camera: ") + why;
        return RVSB_E_ARG;
    }
    if (!std::isfinite(params->blending_factor) || params->blending_factor == 0.f ||
        params->reserved[0] != 0 || params->reserved[1] != 0 ||
        (params->blending_method != RVSB_BLEND_SIMPLE && params->blending_method != RVSB_BLEND_MULTISPECTRAL) ||
        (params->chroma_rounding != RVSB_CHROMA_TIES_EVEN && params->chroma_rounding != RVSB_CHROMA_TIES_UP))
        return RVSB_E_UNSUPPORTED;
    RasterDims rd;
    try {
        rd = raster_dims(*virt, *params);
    } catch (const std::exception& e) {
        s->ctx->last_error = e.what();
        return RVSB_E_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (scene_id < 0 || scene_id >= (int)s->scenes.size()) return RVSB_E_NOT_FOUND;
    if (s->stop) return RVSB_E_BUSY;
    Pending p;
    p.id = s->next_id++;
    p.scene = scene_id;
    p.req.scene = s->scenes[scene_id];
    p.req.virt = *virt;
    p.req.params = *params;
    p.req.out = *out;
    p.bytes = SlotWorkspace::bytes_for(p.req.scene, rd.w, rd.h, rd.rescale);
    if (p.bytes > s->budget) {
        s->ctx->last_error = "request needs more than the server's HBM budget";
        return RVSB_E_OOM_BUDGET;
    }
    p.submit_s = s->now();
    s->pending.push_back(p);
    if (request_id) *request_id = p.id;
    s->cv.notify_one();
    return RVSB_OK;
}

int rvsb_server_poll(rvsb_server* s, rvsb_request_result* out, int max_results) {
    if (!s || !out || max_results <= 0) return 0;
    std::lock_guard<std::mutex> lock(s->mu);
    const int n = std::min(max_results, (int)s->finished.size());
    std::copy(s->finished.begin(), s->finished.begin() + n, out);
    s->finished.erase(s->finished.begin(), s->finished.begin() + n);
    return n;
}

rvsb_status rvsb_server_drain(rvsb_server* s, int timeout_ms) {
    if (!s) return RVSB_E_ARG;
    const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    while (true) {
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (s->pending.empty() && s->in_flight_requests == 0) return RVSB_OK;
        }
        if (Clock::now() >= deadline) return RVSB_E_TIMEOUT;
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

double rvsb_server_clock(const rvsb_server* s) { return s ? s->now() : 0.0; }

void rvsb_server_destroy(rvsb_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->pending.clear();
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    for (auto& L : s->lanes) {
        if (L->stream) cudaStreamSynchronize(L->stream);
        L->core.reset();
        if (L->done) cudaEventDestroy(L->done);
        if (L->stream) cudaStreamDestroy(L->stream);
    }
    delete s;
}

}  // extern "C"
