// C ABI of the B200 synthesis backend (include/rvsb.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "camera.hpp"
#include "engine.hpp"
#include "frontend.hpp"
#include "kernels.hpp"
#include "rvsb.h"

using namespace rvsb;

struct rvsb_batch {
    rvsb_scene* scene = nullptr;
    std::unique_ptr<BatchCore> core;
};

// Pipelined host frames: three sets of raw device planes and output staging
// used in turn; uploads on `copy`, synthesis on `compute`, downloads on
// `down` (a second upload stream gains nothing: the uploads are bound by
// the host link).  With three sets the upload of frame k waits only for frame k-3,
// long finished, so the copy engine and the synthesis both stay busy.
// A set's planes lie back to back in one device block (per view y, u, v,
// depth), so planes that are also adjacent in host memory (a frame read
// into one buffer) go up in one copy: one large copy runs at the link's
// full rate, many small ones about 12% below it.
struct rvsb_host_stream {
    struct Set {
        DevMem frame;                 // every view's y, u, v, depth planes, back to back
        DevMem out;
        cudaEvent_t uploaded = nullptr, computed = nullptr, downloaded = nullptr;
        uint64_t ticket = 0;
        bool busy = false;
    };
    rvsb_context* ctx = nullptr;
    rvsb_scene* scene = nullptr;  // cameras, decoded colour, slot workspace
    static constexpr int kDepth = 3;
    Set sets[kDepth];
    std::vector<size_t> plane_off;  // byte offset of plane 4 * view + k in a set's block
    std::vector<size_t> plane_len;
    cudaStream_t copy = nullptr, compute = nullptr, down = nullptr;
    cudaEvent_t ordered = nullptr;  // the caller's stream at submit time
    uint64_t next = 0;
    ~rvsb_host_stream();
};

namespace {

rvsb_status fail(rvsb_context* ctx, rvsb_status s, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return s;
}

template <class F>
rvsb_status guarded(rvsb_context* ctx, F&& f) {
    try {
        return f();
    } catch (const ArgError& e) {
        return fail(ctx, RVSB_E_ARG, e.what());
    } catch (const ConfigError& e) {
        return fail(ctx, RVSB_E_CONFIG, e.what());
    } catch (const Unsupported& e) {
        return fail(ctx, RVSB_E_UNSUPPORTED, e.what());
    } catch (const IoError& e) {
        return fail(ctx, RVSB_E_IO, e.what());
    } catch (const BudgetError& e) {
        return fail(ctx, RVSB_E_OOM_BUDGET, e.what());
    } catch (const CudaError& e) {
        return fail(ctx, RVSB_E_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(ctx, RVSB_E_OOM_BUDGET, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, RVSB_E_ARG, e.what());
    }
}

size_t plane_bytes(const rvsb_camera& c, int k) {
    const size_t n = (size_t)c.width * c.height;
    return (k == 1 || k == 2) ? (size_t)(c.width / 2) * (c.height / 2) * 2 : n * 2;
}

// Copies planes that are back to back on both sides: parts[i] = (dst, src,
// bytes), each part starting where the previous one ends.  One copy moves
// them all at the link's full rate; but planes adjacent in host memory can
// belong to different pinned allocations, and the runtime refuses a copy
// across them (invalid value, reported at the call), so then each part is
// copied on its own.
struct CopyPart {
    void* dst;
    const void* src;
    size_t bytes;
};
void copy_run(const CopyPart* parts, int n, cudaMemcpyKind kind, cudaStream_t s, const char* what) {
    if (n > 1) {
        size_t total = 0;
        for (int i = 0; i < n; ++i) total += parts[i].bytes;
        const cudaError_t e = cudaMemcpyAsync(parts[0].dst, parts[0].src, total, kind, s);
        if (e == cudaSuccess) return;
        if (e != cudaErrorInvalidValue) check(e, what);
        (void)cudaGetLastError();  // the refused copy: clear it and copy per part
    }
    for (int i = 0; i < n; ++i) check(cudaMemcpyAsync(parts[i].dst, parts[i].src, parts[i].bytes, kind, s), what);
}

// Copies planes parts[0..n) in runs of parts that are adjacent on both
// sides (the library's side is adjacent by construction; the caller's when
// its planes are one buffer).
void copy_planes(const CopyPart* parts, int n, cudaMemcpyKind kind, cudaStream_t s, const char* what) {
    auto follows = [](const void* next, const void* prev, size_t bytes) {
        return static_cast<const char*>(next) == static_cast<const char*>(prev) + bytes;
    };
    for (int k = 0; k < n;) {
        int e = k + 1;
        while (e < n && follows(parts[e].src, parts[e - 1].src, parts[e - 1].bytes) &&
               follows(parts[e].dst, parts[e - 1].dst, parts[e - 1].bytes))
            ++e;
        copy_run(parts + k, e - k, kind, s, what);
        k = e;
    }
}

// Copies a YUV420 result from device staging (Y, U, V back to back, ny and
// nc bytes) to the caller's host planes: one copy when those are one frame
// buffer as well, else one per plane.
void download_yuv(const rvsb_yuv420* host, const rvsb_yuv420& dev, size_t ny, size_t nc, cudaStream_t s) {
    const CopyPart parts[3] = {{host->y, dev.y, ny}, {host->u, dev.u, nc}, {host->v, dev.v, nc}};
    copy_planes(parts, 3, cudaMemcpyDeviceToHost, s, "download");
}

void validate_params(const rvsb_synth_params* p) {
    if (!p) throw ArgError("null synthesis parameters");
    if (!std::isfinite(p->blending_factor) || p->blending_factor == 0.f)
        throw Unsupported("BlendingFactor must be a finite nonzero number (negative: blend by maximum)");
    if (!std::isfinite(p->precision) || !(p->precision > 0.f)) throw Unsupported("Precision must be positive");
    if (p->chroma_rounding != RVSB_CHROMA_TIES_EVEN && p->chroma_rounding != RVSB_CHROMA_TIES_UP)
        throw ArgError("chroma_rounding must be RVSB_CHROMA_TIES_EVEN or RVSB_CHROMA_TIES_UP");
    if (p->reserved[0] != 0 || p->reserved[1] != 0) throw ArgError("reserved synthesis parameters must be 0");
    if (p->blending_method != RVSB_BLEND_SIMPLE && p->blending_method != RVSB_BLEND_MULTISPECTRAL)
        throw ArgError("blending_method must be RVSB_BLEND_SIMPLE or RVSB_BLEND_MULTISPECTRAL");
    if (p->blending_method == RVSB_BLEND_MULTISPECTRAL &&
        (!std::isfinite(p->low_freq_factor) || p->low_freq_factor == 0.f || !std::isfinite(p->high_freq_factor) ||
         p->high_freq_factor == 0.f))
        throw Unsupported("Multispectral blending factors must be finite and nonzero");
}

void validate_request(const rvsb_scene* sc, const rvsb_camera* virt, const rvsb_synth_params* params,
                      const rvsb_yuv420* out) {
    if (!virt || !out || !out->y || !out->u || !out->v) throw ArgError("null camera or output planes");
    validate_params(params);
    if (const char* why = camera_problem(*virt, true)) throw ArgError(std::string("virtual camera: ") + why);
    raster_dims(*virt, *params);
    (void)sc;
}

BatchCore& single_core(rvsb_scene* sc) {
    if (!sc->single) sc->single = std::make_unique<BatchCore>(sc->ctx, 1);
    return *sc->single;
}

// `frame` (optional): raw device planes of every input view for this call;
// their colour is decoded into the scene and their depth read in place.
rvsb_status synthesize_impl(rvsb_scene* sc, const rvsb_camera* virt, const rvsb_synth_params* params,
                            const rvsb_yuv420* out, const rvsb_debug_out* dbg_out, void* stream,
                            const rvsb_view_planes* frame = nullptr, const rvsb_aux_out* aux = nullptr) {
    if (!sc) return RVSB_E_ARG;
    rvsb_context* ctx = sc->ctx;
    HostRange range("rvsb: synthesize");
    return guarded(ctx, [&]() -> rvsb_status {
        validate_request(sc, virt, params, out);
        if (frame) {
            for (size_t v = 0; v < sc->cams.size(); ++v)
                if (!frame[v].y || !frame[v].u || !frame[v].v || !frame[v].depth) throw ArgError("null plane");
        } else {
            for (size_t v = 0; v < sc->cams.size(); ++v)
                if (!sc->uploaded[v]) throw ArgError("input view " + std::to_string(v) + " was not uploaded");
        }
        check(cudaSetDevice(ctx->device), "cudaSetDevice");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        BatchCore& core = single_core(sc);
        int decodes = 0;
        if (frame) {
            DecodeJobs jobs{};
            int max_w = 0, max_h = 0;
            for (size_t v = 0; v < sc->cams.size(); ++v) {
                const rvsb_camera& c = sc->cams[v];
                jobs.v[v] = DecodeJob{frame[v].y, frame[v].u, frame[v].v, sc->color[v]->as<uint64_t>(), c.width,
                                      c.height};
                max_w = std::max(max_w, c.width);
                max_h = std::max(max_h, c.height);
            }
            launch_decode_views(jobs, (int)sc->cams.size(), max_w, max_h, s);
            decodes = 1;
            check(cudaPeekAtLastError(), "decode colour");
            // Depth ranges of the ERP views' vertex tiles, from this frame's depth.
            TileDepthJobs tj{};
            int n_erp = 0, ew = 0, eh = 0;
            for (size_t v = 0; v < sc->cams.size(); ++v) {
                const rvsb_camera& c = sc->cams[v];
                if (c.projection != RVSB_PROJ_EQUIRECTANGULAR) continue;
                tj.v[n_erp++] = TileDepthJob{frame[v].depth, sc->depth_lut[v]->as<float4>(),
                                             sc->tile_depth[v]->as<float2>(), c.width, c.height};
                ew = std::max(ew, c.width);
                eh = std::max(eh, c.height);
            }
            if (n_erp > 0) {
                launch_tile_depth(tj, n_erp, ew, eh, s);
                decodes = 2;
                check(cudaPeekAtLastError(), "tile depth ranges");
            }
        }
        SlotRequest r;
        r.scene = sc;
        r.virt = *virt;
        r.params = *params;
        r.out = *out;
        r.frame = frame;
        if (aux) {
            if (aux->masked.y || aux->masked.u || aux->masked.v)
                if (!aux->masked.y || !aux->masked.u || !aux->masked.v)
                    throw ArgError("masked colour needs all three planes");
            if (aux->mask || aux->masked.y || aux->depth || aux->masked_depth) r.aux = aux;
        }
        if (dbg_out) {
            r.dbg.warped_uvz = dbg_out->warped_uvz;
            r.dbg.view_color = dbg_out->view_color;
            r.dbg.view_depth = dbg_out->view_depth;
            r.dbg.view_validity = dbg_out->view_validity;
            r.dbg.blend_color = dbg_out->blend_color;
            r.dbg.blend_quality = dbg_out->blend_quality;
            r.dbg.inpaint_source = dbg_out->inpaint_source;
        }
        const int launches = core.run(&r, 1, s);
        if (r.dbg.warped_uvz) {
            size_t off = 0;
            SlotWorkspace& ws = core.workspace(0);
            for (size_t v = 0; v < sc->cams.size(); ++v) {
                const size_t nv = (size_t)sc->cams[v].width * sc->cams[v].height;
                check(cudaMemcpyAsync(r.dbg.warped_uvz + off * 4, ws.vert.as<float4>() + off, nv * sizeof(float4),
                                      cudaMemcpyDeviceToDevice, s),
                      "copy warped vertices");
                off += nv;
            }
        }
        sc->last_launches = launches + decodes;
        return RVSB_OK;
    });
}

}  // namespace

extern "C" {

const char* rvsb_status_string(rvsb_status s) {
    switch (s) {
        case RVSB_OK: return "ok";
        case RVSB_E_ARG: return "invalid argument";
        case RVSB_E_CONFIG: return "configuration rejected";
        case RVSB_E_IO: return "i/o error";
        case RVSB_E_OOM_BUDGET: return "HBM budget exceeded";
        case RVSB_E_CUDA: return "CUDA error";
        case RVSB_E_TIMEOUT: return "timeout";
        case RVSB_E_UNSUPPORTED: return "unsupported option";
        case RVSB_E_BUSY: return "busy";
        case RVSB_E_NOT_FOUND: return "not found";
    }
    return "unknown status";
}

rvsb_status rvsb_create(int device, size_t hbm_budget_bytes, rvsb_context** out) {
    if (!out) return RVSB_E_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return RVSB_E_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return RVSB_E_CUDA;
    auto* ctx = new (std::nothrow) rvsb_context;
    if (!ctx) return RVSB_E_OOM_BUDGET;
    ctx->device = device;
    ctx->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)60 << 30;
    *out = ctx;
    return RVSB_OK;
}

void rvsb_destroy(rvsb_context* ctx) {
    if (!ctx) return;
    if (ctx->host_scene) rvsb_scene_destroy(ctx->host_scene);
    if (ctx->host_out) {
        cudaSetDevice(ctx->device);
        cudaFree(ctx->host_out);
    }
    delete ctx;
}

const char* rvsb_last_error(const rvsb_context* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

size_t rvsb_memory_in_use(const rvsb_context* ctx) { return ctx ? ctx->in_use : 0; }

rvsb_status rvsb_relative_pose(const rvsb_camera* input, const rvsb_camera* virt, float R[9], float t[3]) {
    if (!input || !virt || !R || !t) return RVSB_E_ARG;
    relative_pose(*input, *virt, R, t);
    return RVSB_OK;
}

rvsb_status rvsb_scene_create(rvsb_context* ctx, const rvsb_camera* inputs, int n_inputs, rvsb_scene** out) {
    if (!ctx || !inputs || !out || n_inputs <= 0 || n_inputs > MAX_VIEWS) return RVSB_E_ARG;
    *out = nullptr;
    return guarded(ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(ctx->device), "cudaSetDevice");
        auto sc = std::make_unique<rvsb_scene>();
        sc->ctx = ctx;
        for (int v = 0; v < n_inputs; ++v) {
            if (const char* why = camera_problem(inputs[v], false))
                throw ArgError("input camera " + std::to_string(v) + ": " + why);
            sc->cams.push_back(inputs[v]);
        }
        for (int v = 0; v < n_inputs; ++v) {
            auto m = std::make_unique<DevMem>();
            m->alloc(ctx, plane_bytes(inputs[v], 0) + 2 * plane_bytes(inputs[v], 1) + plane_bytes(inputs[v], 3));
            sc->raw.push_back(std::move(m));
            auto r = std::make_unique<DevMem>();
            auto c = std::make_unique<DevMem>();
            auto cone = std::make_unique<DevMem>();
            auto tdep = std::make_unique<DevMem>();
            if (inputs[v].projection == RVSB_PROJ_EQUIRECTANGULAR) {
                std::vector<float> rows, cols, cones;
                erp_tables(inputs[v], rows, cols);
                r->alloc(ctx, rows.size() * sizeof(float));
                c->alloc(ctx, cols.size() * sizeof(float));
                check(cudaMemcpy(r->ptr, rows.data(), rows.size() * sizeof(float), cudaMemcpyHostToDevice),
                      "upload ERP rows");
                check(cudaMemcpy(c->ptr, cols.data(), cols.size() * sizeof(float), cudaMemcpyHostToDevice),
                      "upload ERP columns");
                erp_tile_cones(inputs[v], rows, cols, WARP_TILE, cones);
                cone->alloc(ctx, cones.size() * sizeof(float));
                check(cudaMemcpy(cone->ptr, cones.data(), cones.size() * sizeof(float), cudaMemcpyHostToDevice),
                      "upload ERP tile cones");
                tdep->alloc(ctx, cones.size() / 4 * sizeof(float2));
            }
            sc->erp_cone.push_back(std::move(cone));
            sc->tile_depth.push_back(std::move(tdep));
            sc->erp.push_back(std::move(r));
            sc->erp.push_back(std::move(c));
            auto col = std::make_unique<DevMem>();
            col->alloc(ctx, (size_t)inputs[v].width * inputs[v].height * sizeof(uint64_t));
            sc->color.push_back(std::move(col));
            auto lut = std::make_unique<DevMem>();
            lut->alloc(ctx, 65536 * sizeof(float4));
            const rvsb_camera& cam = inputs[v];
            launch_depth_lut(cam.depth_range[0], cam.depth_range[1],
                             1.0f / (float)((1u << cam.bit_depth_depth) - 1u), cam.has_invalid_depth,
                             cam.focal[0], cam.focal[1], lut->as<float4>(), nullptr);
            check(cudaPeekAtLastError(), "depth table");
            sc->depth_lut.push_back(std::move(lut));
        }
        // The depth tables must be complete before any stream uses them.
        check(cudaStreamSynchronize(nullptr), "depth tables");
        sc->uploaded.assign(n_inputs, false);
        *out = sc.release();
        return RVSB_OK;
    });
}

void rvsb_scene_destroy(rvsb_scene* scene) {
    if (!scene) return;
    cudaSetDevice(scene->ctx->device);
    cudaDeviceSynchronize();
    delete scene;
}

rvsb_status rvsb_scene_upload(rvsb_scene* sc, int view, const rvsb_view_planes* planes, int planes_on_device,
                              void* stream) {
    if (!sc) return RVSB_E_ARG;
    HostRange range("rvsb: scene upload");
    return guarded(sc->ctx, [&]() -> rvsb_status {
        if (!planes || view < 0 || view >= (int)sc->cams.size()) throw ArgError("bad view index or planes");
        const void* src[4] = {planes->y, planes->u, planes->v, planes->depth};
        for (int k = 0; k < 4; ++k)
            if (!src[k]) throw ArgError("null plane");
        check(cudaSetDevice(sc->ctx->device), "cudaSetDevice");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const rvsb_camera& c = sc->cams[view];
        const cudaMemcpyKind kind = planes_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        CopyPart parts[4];
        for (int k = 0; k < 4; ++k) parts[k] = {sc->plane(view, k), src[k], plane_bytes(c, k)};
        copy_planes(parts, 4, kind, s, "upload planes");
        launch_decode_color(sc->plane(view, 0), sc->plane(view, 1), sc->plane(view, 2), c.width, c.height,
                            sc->color[view]->as<uint64_t>(), s);
        check(cudaPeekAtLastError(), "decode colour");
        if (c.projection == RVSB_PROJ_EQUIRECTANGULAR) {
            TileDepthJobs jobs{};
            jobs.v[0] = TileDepthJob{sc->plane(view, 3), sc->depth_lut[view]->as<float4>(),
                                     sc->tile_depth[view]->as<float2>(), c.width, c.height};
            launch_tile_depth(jobs, 1, c.width, c.height, s);
            check(cudaPeekAtLastError(), "tile depth ranges");
        }
        sc->uploaded[view] = true;
        return RVSB_OK;
    });
}

rvsb_status rvsb_synthesize(rvsb_scene* scene, const rvsb_camera* virt, const rvsb_synth_params* params,
                            const rvsb_yuv420* out, void* stream) {
    return synthesize_impl(scene, virt, params, out, nullptr, stream);
}

rvsb_status rvsb_synthesize_aux(rvsb_scene* scene, const rvsb_camera* virt, const rvsb_synth_params* params,
                                const rvsb_yuv420* out, const rvsb_aux_out* aux, void* stream) {
    return synthesize_impl(scene, virt, params, out, nullptr, stream, nullptr, aux);
}

rvsb_status rvsb_synthesize_debug(rvsb_scene* scene, const rvsb_camera* virt, const rvsb_synth_params* params,
                                  const rvsb_yuv420* out, const rvsb_debug_out* dbg, void* stream) {
    return synthesize_impl(scene, virt, params, out, dbg, stream);
}

rvsb_status rvsb_synthesize_frame(rvsb_scene* scene, const rvsb_view_planes* device_planes,
                                  const rvsb_camera* virt, const rvsb_synth_params* params,
                                  const rvsb_yuv420* out, void* stream) {
    if (!device_planes) return RVSB_E_ARG;
    return synthesize_impl(scene, virt, params, out, nullptr, stream, device_planes);
}

int rvsb_scene_last_launch_count(const rvsb_scene* scene) { return scene ? scene->last_launches : 0; }

rvsb_status rvsb_scene_set_profiling(rvsb_scene* sc, int enable) {
    if (!sc) return RVSB_E_ARG;
    return guarded(sc->ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(sc->ctx->device), "cudaSetDevice");
        single_core(sc).set_profiling(enable != 0);
        return RVSB_OK;
    });
}

int rvsb_scene_stage_times(rvsb_scene* sc, float* ms, int max_stages) {
    if (!sc || !ms || !sc->single) return -1;
    return sc->single->stage_times(ms, max_stages);
}

// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------

rvsb_status rvsb_batch_create(rvsb_scene* scene, int max_slots, rvsb_batch** out) {
    if (!scene || !out || max_slots <= 0 || max_slots > 1024) return RVSB_E_ARG;
    *out = nullptr;
    return guarded(scene->ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(scene->ctx->device), "cudaSetDevice");
        auto b = std::make_unique<rvsb_batch>();
        b->scene = scene;
        b->core = std::make_unique<BatchCore>(scene->ctx, max_slots);
        *out = b.release();
        return RVSB_OK;
    });
}

void rvsb_batch_destroy(rvsb_batch* batch) {
    if (!batch) return;
    cudaSetDevice(batch->scene->ctx->device);
    cudaDeviceSynchronize();
    delete batch;
}

rvsb_status rvsb_batch_reserve(rvsb_batch* batch, int max_width, int max_height) {
    if (!batch || max_width <= 0 || max_height <= 0) return RVSB_E_ARG;
    return guarded(batch->scene->ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(batch->scene->ctx->device), "cudaSetDevice");
        for (int k = 0; k < batch->core->slots(); ++k)
            batch->core->workspace(k).ensure(batch->scene->ctx, batch->scene, max_width, max_height);
        return RVSB_OK;
    });
}

rvsb_status rvsb_batch_set_graphs(rvsb_batch* batch, int enable) {
    if (!batch) return RVSB_E_ARG;
    batch->core->set_graphs(enable != 0);
    return RVSB_OK;
}

rvsb_status rvsb_batch_set_autotune(rvsb_batch* batch, int enable) {
    if (!batch) return RVSB_E_ARG;
    batch->core->set_autotune(enable != 0);
    return RVSB_OK;
}

rvsb_status rvsb_batch_set_raster_variant(rvsb_batch* batch, int variant) {
    if (!batch || variant < -1 || variant >= NUM_RASTER_VARIANTS) return RVSB_E_ARG;
    batch->core->force_variant(variant);
    return RVSB_OK;
}

int rvsb_batch_last_raster_variant(const rvsb_batch* batch) { return batch ? batch->core->last_variant() : -1; }

rvsb_status rvsb_scene_set_autotune(rvsb_scene* sc, int enable) {
    if (!sc) return RVSB_E_ARG;
    return guarded(sc->ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(sc->ctx->device), "cudaSetDevice");
        single_core(sc).set_autotune(enable != 0);
        return RVSB_OK;
    });
}

rvsb_status rvsb_scene_set_raster_variant(rvsb_scene* sc, int variant) {
    if (!sc || variant < -1 || variant >= NUM_RASTER_VARIANTS) return RVSB_E_ARG;
    return guarded(sc->ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(sc->ctx->device), "cudaSetDevice");
        single_core(sc).force_variant(variant);
        return RVSB_OK;
    });
}

rvsb_status rvsb_batch_set_profiling(rvsb_batch* batch, int enable) {
    if (!batch) return RVSB_E_ARG;
    return guarded(batch->scene->ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(batch->scene->ctx->device), "cudaSetDevice");
        batch->core->set_profiling(enable != 0);
        return RVSB_OK;
    });
}

int rvsb_batch_stage_times(rvsb_batch* batch, float* ms, int max_stages) {
    return batch ? batch->core->stage_times(ms, max_stages) : -1;
}

int rvsb_batch_last_launch_count(const rvsb_batch* batch) { return batch ? batch->core->last_launches() : 0; }

rvsb_status rvsb_synthesize_batch(rvsb_batch* batch, const rvsb_camera* virts, int n,
                                  const rvsb_synth_params* params, const rvsb_yuv420* outs, void* stream) {
    if (!batch || !virts || !outs || n <= 0) return RVSB_E_ARG;
    rvsb_scene* sc = batch->scene;
    return guarded(sc->ctx, [&]() -> rvsb_status {
        for (size_t v = 0; v < sc->cams.size(); ++v)
            if (!sc->uploaded[v]) throw ArgError("input view " + std::to_string(v) + " was not uploaded");
        for (int k = 0; k < n; ++k) validate_request(sc, &virts[k], params, &outs[k]);
        check(cudaSetDevice(sc->ctx->device), "cudaSetDevice");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        BatchCore& core = *batch->core;
        std::vector<SlotRequest> reqs(std::min(n, core.slots()));
        for (int k0 = 0; k0 < n; k0 += core.slots()) {
            const int m = std::min(core.slots(), n - k0);
            for (int k = 0; k < m; ++k) {
                reqs[k].scene = sc;
                reqs[k].virt = virts[k0 + k];
                reqs[k].params = *params;
                reqs[k].out = outs[k0 + k];
            }
            core.run(reqs.data(), m, s);
        }
        return RVSB_OK;
    });
}

const char* rvsb_stage_name(int stage) {
    static const char* names[NUM_STAGES] = {"warp", "bin", "raster", "inpaint", "total"};
    return (stage >= 0 && stage < NUM_STAGES) ? names[stage] : "";
}

rvsb_status rvsb_synthesize_host(rvsb_context* ctx, const rvsb_camera* inputs, int n_inputs,
                                 const rvsb_view_planes* host_planes, const rvsb_camera* virt,
                                 const rvsb_synth_params* params, const rvsb_yuv420* out_host, void* stream) {
    if (!ctx || !inputs || !host_planes || !virt || !out_host || n_inputs <= 0) return RVSB_E_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    // Reuse the scene of the previous call when the input cameras match.
    rvsb_scene* sc = ctx->host_scene;
    if (!sc || sc->cams.size() != (size_t)n_inputs ||
        std::memcmp(sc->cams.data(), inputs, sizeof(rvsb_camera) * n_inputs) != 0) {
        if (sc) rvsb_scene_destroy(sc);
        ctx->host_scene = nullptr;
        rvsb_status st = rvsb_scene_create(ctx, inputs, n_inputs, &sc);
        if (st != RVSB_OK) return st;
        ctx->host_scene = sc;
    }
    for (int v = 0; v < n_inputs; ++v) {
        rvsb_status st = rvsb_scene_upload(sc, v, &host_planes[v], 0, stream);
        if (st != RVSB_OK) return st;
    }
    return guarded(ctx, [&]() -> rvsb_status {
        if (!out_host->y || !out_host->u || !out_host->v) throw ArgError("null output planes");
        const size_t ny = (size_t)virt->width * virt->height * 2;
        const size_t nc = (size_t)(virt->width / 2) * (virt->height / 2) * 2;
        // Device output staging owned by the context.
        if (ctx->host_out_bytes < ny + 2 * nc) {
            if (ctx->host_out) {
                cudaFree(ctx->host_out);
                ctx->in_use -= ctx->host_out_bytes;
                ctx->host_out = nullptr;
                ctx->host_out_bytes = 0;
            }
            if (ctx->in_use + ny + 2 * nc > ctx->budget) throw BudgetError("output staging exceeds the HBM budget");
            check(cudaMalloc(&ctx->host_out, ny + 2 * nc), "cudaMalloc");
            ctx->host_out_bytes = ny + 2 * nc;
            ctx->in_use += ny + 2 * nc;
        }
        rvsb_yuv420 dev;
        char* base = static_cast<char*>(ctx->host_out);
        dev.y = reinterpret_cast<uint16_t*>(base);
        dev.u = reinterpret_cast<uint16_t*>(base + ny);
        dev.v = reinterpret_cast<uint16_t*>(base + ny + nc);
        rvsb_status st = synthesize_impl(sc, virt, params, &dev, nullptr, stream);
        if (st != RVSB_OK) return st;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        download_yuv(out_host, dev, ny, nc, s);
        check(cudaStreamSynchronize(s), "synchronize");
        return RVSB_OK;
    });
}

rvsb_host_stream::~rvsb_host_stream() {
    cudaSetDevice(ctx->device);
    for (Set& s : sets)
        if (s.busy) cudaEventSynchronize(s.downloaded);
    for (Set& s : sets)
        for (cudaEvent_t e : {s.uploaded, s.computed, s.downloaded})
            if (e) cudaEventDestroy(e);
    for (cudaStream_t st : {copy, compute, down})
        if (st) cudaStreamDestroy(st);
    if (ordered) cudaEventDestroy(ordered);
    if (scene) rvsb_scene_destroy(scene);
}

rvsb_status rvsb_host_stream_create(rvsb_context* ctx, const rvsb_camera* inputs, int n_inputs,
                                    rvsb_host_stream** out) {
    if (!ctx || !inputs || !out || n_inputs <= 0) return RVSB_E_ARG;
    *out = nullptr;
    auto hs = std::make_unique<rvsb_host_stream>();
    hs->ctx = ctx;
    rvsb_status st = rvsb_scene_create(ctx, inputs, n_inputs, &hs->scene);
    if (st != RVSB_OK) return st;
    return guarded(ctx, [&]() -> rvsb_status {
        check(cudaSetDevice(ctx->device), "cudaSetDevice");
        size_t total = 0;
        for (int v = 0; v < n_inputs; ++v)
            for (int k = 0; k < 4; ++k) {
                hs->plane_off.push_back(total);
                hs->plane_len.push_back(plane_bytes(inputs[v], k));
                total += plane_bytes(inputs[v], k);
            }
        for (auto& s : hs->sets) {
            s.frame.alloc(ctx, total);
            for (cudaEvent_t* e : {&s.uploaded, &s.computed, &s.downloaded})
                check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
        }
        for (cudaStream_t* sp : {&hs->copy, &hs->compute, &hs->down})
            check(cudaStreamCreateWithFlags(sp, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaEventCreateWithFlags(&hs->ordered, cudaEventDisableTiming), "cudaEventCreate");
        *out = hs.release();
        return RVSB_OK;
    });
}

void rvsb_host_stream_destroy(rvsb_host_stream* hs) { delete hs; }

rvsb_status rvsb_host_stream_submit(rvsb_host_stream* hs, const rvsb_view_planes* host_planes,
                                    const rvsb_camera* virt, const rvsb_synth_params* params,
                                    const rvsb_yuv420* out_host, void* stream, uint64_t* ticket) {
    if (!hs || !host_planes || !virt || !out_host || !ticket) return RVSB_E_ARG;
    rvsb_context* ctx = hs->ctx;
    HostRange range("rvsb: host frame (upload, synthesis, download)");
    return guarded(ctx, [&]() -> rvsb_status {
        if (!out_host->y || !out_host->u || !out_host->v) throw ArgError("null output planes");
        rvsb_scene* sc = hs->scene;
        const int n = (int)sc->cams.size();
        for (int v = 0; v < n; ++v)
            if (!host_planes[v].y || !host_planes[v].u || !host_planes[v].v || !host_planes[v].depth)
                throw ArgError("null plane");
        validate_request(sc, virt, params, out_host);
        check(cudaSetDevice(ctx->device), "cudaSetDevice");
        rvsb_host_stream::Set& S = hs->sets[hs->next % rvsb_host_stream::kDepth];
        // The set's previous frame (three submits ago) must be complete
        // before its planes and staging are reused.
        if (S.busy) {
            check(cudaEventSynchronize(S.downloaded), "wait for an earlier frame");
            S.busy = false;
        }
        const size_t ny = (size_t)virt->width * virt->height * 2;
        const size_t nc = (size_t)(virt->width / 2) * (virt->height / 2) * 2;
        if (S.out.bytes < ny + 2 * nc) S.out.alloc(ctx, ny + 2 * nc);
        check(cudaEventRecord(hs->ordered, static_cast<cudaStream_t>(stream)), "record caller stream");
        check(cudaStreamWaitEvent(hs->copy, hs->ordered, 0), "order after caller stream");
        std::vector<rvsb_view_planes> dev(n);
        char* block = static_cast<char*>(S.frame.ptr);
        std::vector<CopyPart> parts(4 * n);
        for (int p = 0; p < 4 * n; ++p) {
            const rvsb_view_planes& hp = host_planes[p / 4];
            const void* srcs[4] = {hp.y, hp.u, hp.v, hp.depth};
            parts[p] = {block + hs->plane_off[p], srcs[p % 4], hs->plane_len[p]};
        }
        copy_planes(parts.data(), 4 * n, cudaMemcpyHostToDevice, hs->copy, "upload planes");
        for (int v = 0; v < n; ++v) {
            dev[v].y = reinterpret_cast<uint16_t*>(block + hs->plane_off[v * 4 + 0]);
            dev[v].u = reinterpret_cast<uint16_t*>(block + hs->plane_off[v * 4 + 1]);
            dev[v].v = reinterpret_cast<uint16_t*>(block + hs->plane_off[v * 4 + 2]);
            dev[v].depth = reinterpret_cast<uint16_t*>(block + hs->plane_off[v * 4 + 3]);
        }
        check(cudaEventRecord(S.uploaded, hs->copy), "record upload");
        check(cudaStreamWaitEvent(hs->compute, S.uploaded, 0), "wait for upload");
        rvsb_yuv420 o;
        char* base = static_cast<char*>(S.out.ptr);
        o.y = reinterpret_cast<uint16_t*>(base);
        o.u = reinterpret_cast<uint16_t*>(base + ny);
        o.v = reinterpret_cast<uint16_t*>(base + ny + nc);
        rvsb_status st = synthesize_impl(sc, virt, params, &o, nullptr, hs->compute, dev.data());
        if (st != RVSB_OK) return st;
        check(cudaEventRecord(S.computed, hs->compute), "record synthesis");
        check(cudaStreamWaitEvent(hs->down, S.computed, 0), "wait for synthesis");
        download_yuv(out_host, o, ny, nc, hs->down);
        check(cudaEventRecord(S.downloaded, hs->down), "record download");
        S.ticket = hs->next;
        S.busy = true;
        *ticket = hs->next++;
        return RVSB_OK;
    });
}

rvsb_status rvsb_host_stream_wait(rvsb_host_stream* hs, uint64_t ticket) {
    if (!hs || ticket >= hs->next) return RVSB_E_ARG;
    return guarded(hs->ctx, [&]() -> rvsb_status {
        for (auto& s : hs->sets)
            if (s.busy && s.ticket == ticket) {
                check(cudaEventSynchronize(s.downloaded), "wait for frame");
                s.busy = false;
            }
        return RVSB_OK;  // older frames completed before their set was reused
    });
}

rvsb_status rvsb_host_stream_join(rvsb_host_stream* hs, void* stream) {
    if (!hs) return RVSB_E_ARG;
    return guarded(hs->ctx, [&]() -> rvsb_status {
        for (auto& s : hs->sets)
            if (s.busy)
                check(cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), s.downloaded, 0), "join");
        return RVSB_OK;
    });
}

// ---------------------------------------------------------------------------
// Front end
// ---------------------------------------------------------------------------

struct rvsb_config {
    Config cfg;
};

static void copy_err(char* err, size_t len, const char* msg) {
    if (err && len) {
        std::strncpy(err, msg, len - 1);
        err[len - 1] = 0;
    }
}

rvsb_status rvsb_camera_from_json(const char* text, rvsb_camera* out, char* err, size_t err_len) {
    if (!text || !out) return RVSB_E_ARG;
    try {
        *out = parse_camera(json::Node::parse(text));
        return RVSB_OK;
    } catch (const Unsupported& e) {
        copy_err(err, err_len, e.what());
        return RVSB_E_UNSUPPORTED;
    } catch (const std::exception& e) {
        copy_err(err, err_len, e.what());
        return RVSB_E_CONFIG;
    }
}

rvsb_status rvsb_config_load(const char* path, rvsb_config** out, char* err, size_t err_len) {
    if (!path || !out) return RVSB_E_ARG;
    *out = nullptr;
    try {
        auto c = std::make_unique<rvsb_config>();
        c->cfg = load_config(path);
        *out = c.release();
        return RVSB_OK;
    } catch (const IoError& e) {
        copy_err(err, err_len, e.what());
        return RVSB_E_IO;
    } catch (const Unsupported& e) {
        copy_err(err, err_len, e.what());
        return RVSB_E_UNSUPPORTED;
    } catch (const std::exception& e) {
        copy_err(err, err_len, e.what());
        return RVSB_E_CONFIG;
    }
}

void rvsb_config_free(rvsb_config* cfg) { delete cfg; }
int rvsb_config_num_inputs(const rvsb_config* c) { return c ? (int)c->cfg.params_real.size() : 0; }
int rvsb_config_num_virtual(const rvsb_config* c) { return c ? (int)c->cfg.params_virtual.size() : 0; }

rvsb_status rvsb_config_input_camera(const rvsb_config* c, int i, rvsb_camera* out) {
    if (!c || !out || i < 0 || i >= (int)c->cfg.params_real.size()) return RVSB_E_ARG;
    *out = c->cfg.params_real[i];
    return RVSB_OK;
}

rvsb_status rvsb_config_virtual_camera(const rvsb_config* c, int i, rvsb_camera* out) {
    if (!c || !out || i < 0 || i >= (int)c->cfg.params_virtual.size()) return RVSB_E_ARG;
    *out = c->cfg.params_virtual[i];
    return RVSB_OK;
}

static rvsb_status crop_of(const std::vector<CropRegion>& v, int i, int32_t region[4], int32_t padded_size[2]) {
    if (!region || !padded_size || i < 0 || i >= (int)v.size()) return RVSB_E_ARG;
    const CropRegion& r = v[i];
    region[0] = r.x;
    region[1] = r.y;
    region[2] = r.w;
    region[3] = r.h;
    padded_size[0] = r.padded_w;
    padded_size[1] = r.padded_h;
    return RVSB_OK;
}

rvsb_status rvsb_config_virtual_crop(const rvsb_config* c, int i, int32_t region[4], int32_t padded_size[2]) {
    return c ? crop_of(c->cfg.crop_virtual, i, region, padded_size) : RVSB_E_ARG;
}

rvsb_status rvsb_config_input_crop(const rvsb_config* c, int i, int32_t region[4], int32_t padded_size[2]) {
    return c ? crop_of(c->cfg.crop_real, i, region, padded_size) : RVSB_E_ARG;
}

const char* rvsb_config_texture_path(const rvsb_config* c, int i) {
    return (c && i >= 0 && i < (int)c->cfg.texture_names.size()) ? c->cfg.texture_names[i].c_str() : nullptr;
}
const char* rvsb_config_depth_path(const rvsb_config* c, int i) {
    return (c && i >= 0 && i < (int)c->cfg.depth_names.size()) ? c->cfg.depth_names[i].c_str() : nullptr;
}
const char* rvsb_config_output_path(const rvsb_config* c, int i) {
    return (c && i >= 0 && i < (int)c->cfg.outfilenames.size()) ? c->cfg.outfilenames[i].c_str() : nullptr;
}

void rvsb_config_frames(const rvsb_config* c, int* start, int* n, int* nout) {
    if (!c) return;
    if (start) *start = c->cfg.start_frame;
    if (n) *n = c->cfg.number_of_frames;
    if (nout) *nout = c->cfg.number_of_output_frames;
}

const char* rvsb_config_output_file(const rvsb_config* c, int kind, int i) {
    if (!c) return nullptr;
    const std::vector<std::string>* v = nullptr;
    switch (kind) {
        case RVSB_OUT_COLOR: v = &c->cfg.outfilenames; break;
        case RVSB_OUT_MASKED_COLOR: v = &c->cfg.outmaskedfilenames; break;
        case RVSB_OUT_MASK: v = &c->cfg.outmaskfilenames; break;
        case RVSB_OUT_DEPTH: v = &c->cfg.outdepthfilenames; break;
        case RVSB_OUT_MASKED_DEPTH: v = &c->cfg.outmaskdepthfilenames; break;
        default: return nullptr;
    }
    return (i >= 0 && i < (int)v->size()) ? (*v)[i].c_str() : nullptr;
}

float rvsb_config_validity_threshold(const rvsb_config* c) { return c ? c->cfg.validity_threshold : 5000.f; }

void rvsb_config_synth_params(const rvsb_config* c, rvsb_synth_params* out) {
    if (!c || !out) return;
    std::memset(out, 0, sizeof(*out));
    out->blending_factor = c->cfg.blending_factor;
    out->precision = c->cfg.precision;
    out->chroma_rounding = RVSB_CHROMA_TIES_EVEN;
    if (c->cfg.blending_method == "Multispectral") {
        out->blending_method = RVSB_BLEND_MULTISPECTRAL;
        out->low_freq_factor = c->cfg.blending_low_freq_factor;
        out->high_freq_factor = c->cfg.blending_high_freq_factor;
    }
}

rvsb_status rvsb_config_virtual_camera_at(const rvsb_config* c, int i, int frame, rvsb_camera* out) {
    if (!c || !out || i < 0 || i >= (int)c->cfg.params_virtual.size() || frame < 0) return RVSB_E_ARG;
    *out = c->cfg.params_virtual[i];
    if (!c->cfg.pose_trace.empty()) {
        if (frame >= (int)c->cfg.pose_trace.size()) return RVSB_E_ARG;
        const Pose& p = c->cfg.pose_trace[frame];
        for (int k = 0; k < 3; ++k) out->position[k] = out->position[k] + p.position[k];
        for (int k = 0; k < 3; ++k) out->rotation[k] = p.rotation[k];
    }
    return RVSB_OK;
}

}  // extern "C"
