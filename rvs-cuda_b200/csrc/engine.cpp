// Host engine: device memory, slot workspaces, slot tables and batch launches.
#include "engine.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "camera.hpp"
#include "frontend.hpp"

namespace rvsb {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

void DevMem::alloc(rvsb_context* c, size_t n) {
    release();
    if (n == 0) n = 16;
    {
        std::lock_guard<std::mutex> lock(c->mem_mu);
        if (c->in_use + n > c->budget)
            throw BudgetError("request of " + std::to_string(n) + " bytes exceeds the HBM budget (" +
                              std::to_string(c->in_use) + " of " + std::to_string(c->budget) + " in use)");
        c->in_use += n;
    }
    const cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        std::lock_guard<std::mutex> lock(c->mem_mu);
        c->in_use -= n;
        check(e, "cudaMalloc");
    }
    ctx = c;
    bytes = n;
}

void DevMem::release() {
    if (ptr) {
        cudaFree(ptr);
        std::lock_guard<std::mutex> lock(ctx->mem_mu);
        ctx->in_use -= bytes;
    }
    ptr = nullptr;
    bytes = 0;
}

RasterDims raster_dims(const rvsb_camera& virt, const rvsb_synth_params& p) {
    if (!std::isfinite(p.precision) || !(p.precision > 0.f)) throw Unsupported("Precision must be positive");
    if (p.precision == 1.f) return {virt.width, virt.height, false};
    const int w = (int)(0.5f + (float)virt.width * p.precision);
    const int h = (int)(0.5f + (float)virt.height * p.precision);
    if (w < 2 || h < 2 || w > 32768 || h > 32768)
        throw Unsupported("Precision " + std::to_string(p.precision) + " gives a raster size of " +
                          std::to_string(w) + "x" + std::to_string(h) +
                          "; only sizes of at least 2 and at most 32768 are supported");
    return {w, h, true};
}

int nblocks_x(int w) { return (w - 1 + BLOCK_W - 1) / BLOCK_W; }
int nblocks_y(int h) { return (h - 1 + BLOCK_H - 1) / BLOCK_H; }

namespace {

struct SlotNeeds {
    size_t vert, bbox, out, bins, list;
};

SlotNeeds needs_of(const rvsb_scene* sc, int wo, int ho) {
    SlotNeeds n{};
    for (const auto& c : sc->cams) {
        n.vert += (size_t)c.width * c.height;
        n.bbox += (size_t)nblocks_x(c.width) * nblocks_y(c.height);
    }
    n.out = (size_t)wo * ho;
    n.bins = (size_t)((wo + MIN_TILE_W - 1) / MIN_TILE_W) * ((ho + MIN_TILE_H - 1) / MIN_TILE_H) * sc->cams.size();
    n.list = std::min<size_t>(INT32_MAX / 2, std::max<size_t>(1 << 16, n.bbox * 8 + n.bins));
    return n;
}

}  // namespace

size_t SlotWorkspace::bytes_for(const rvsb_scene* sc, int wo, int ho, bool rescale) {
    const SlotNeeds n = needs_of(sc, wo, ho);
    return sizeof(DevStatus) + n.vert * sizeof(float4) + n.bbox * sizeof(int4) + 3 * n.bins * sizeof(int) +
           n.list * sizeof(int) + n.out * (sizeof(uint64_t) * 5 + 1) +
           inpaint_seg_words(wo) * sizeof(uint64_t) +
           n.bins / std::max<size_t>(1, sc->cams.size()) * sizeof(int) +
           (rescale ? n.out * (sizeof(float4) + 2 * sizeof(int32_t)) : 0);
}

void SlotWorkspace::ensure_rescale(rvsb_context* ctx, int wo, int ho) {
    const size_t n = (size_t)wo * ho;
    if (n > cap_rescale) {
        pcolor.alloc(ctx, n * sizeof(float4));
        psrc.alloc(ctx, n * 2 * sizeof(int32_t));
        cap_rescale = n;
    }
}

void SlotWorkspace::ensure(rvsb_context* ctx, const rvsb_scene* sc, int wo, int ho) {
    const SlotNeeds n = needs_of(sc, wo, ho);
    if (!status.ptr) status.alloc(ctx, sizeof(DevStatus));
    if (n.vert > cap_vert) {
        vert.alloc(ctx, n.vert * sizeof(float4));
        cap_vert = n.vert;
    }
    if (n.bbox > cap_bbox) {
        bbox.alloc(ctx, n.bbox * sizeof(int4));
        cap_bbox = n.bbox;
    }
    if (n.bins > cap_bins) {
        counts.alloc(ctx, n.bins * sizeof(int));
        offsets.alloc(ctx, n.bins * sizeof(int));
        cursor.alloc(ctx, n.bins * sizeof(int));
        cap_bins = n.bins;
    }
    if (n.list > cap_list) {
        list.alloc(ctx, n.list * sizeof(int));
        cap_list = n.list;
    }
    const size_t tiles = (size_t)((wo + MIN_TILE_W - 1) / MIN_TILE_W) * ((ho + MIN_TILE_H - 1) / MIN_TILE_H);
    if (tiles > cap_tiles) {
        tile_order.alloc(ctx, tiles * sizeof(int));
        cap_tiles = tiles;
    }
    const size_t seg_words = inpaint_seg_words(wo);
    if (seg_words > cap_seg_words) {
        inpaint_seg.alloc(ctx, seg_words * sizeof(uint64_t));
        cap_seg_words = seg_words;
    }
    if (n.out > cap_out) {
        codes.alloc(ctx, n.out * sizeof(uint64_t));
        holes.alloc(ctx, n.out);
        for (auto& s : scan) s.alloc(ctx, n.out * sizeof(uint64_t));
        cap_out = n.out;
    }
}

void SlotWorkspace::ensure_aux(rvsb_context* ctx, int wo, int ho) {
    const size_t n = (size_t)wo * ho;
    if (n > cap_aux) {
        aux_depth.alloc(ctx, n * sizeof(float));
        aux_valid.alloc(ctx, n * sizeof(float));
        cap_aux = n;
    }
}

void SlotWorkspace::ensure_ms(rvsb_context* ctx, int n_views, int wo, int ho) {
    const size_t n = (size_t)n_views * wo * ho;
    if (n > cap_ms) {
        ms_view.alloc(ctx, n * sizeof(float4));
        ms_hsum.alloc(ctx, n * sizeof(double));
        ms_hcnt.alloc(ctx, n * sizeof(int));
        ms_blur.alloc(ctx, n * sizeof(float));
        cap_ms = n;
    }
}

BatchCore::BatchCore(rvsb_context* ctx, int slots) : ctx_(ctx), slots_(slots) {
    if (slots <= 0) throw ArgError("a batch needs at least one slot");
    prepare_kernels();
    for (int k = 0; k < slots; ++k) ws_.push_back(std::make_unique<SlotWorkspace>());
    tables_.alloc(ctx, sizeof(SlotTable) * (size_t)slots);
    for (int b = 0; b < 2; ++b) {
        void* p = nullptr;
        check(cudaHostAlloc(&p, sizeof(SlotTable) * (size_t)slots, cudaHostAllocDefault), "cudaHostAlloc");
        staging_[b] = static_cast<SlotTable*>(p);
        check(cudaEventCreateWithFlags(&copied_[b], cudaEventDisableTiming), "cudaEventCreate");
    }
    check(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : tune_ev_) check(cudaEventCreate(&e), "cudaEventCreate");
}

BatchCore::~BatchCore() {
    for (auto& g : graphs_) cudaGraphExecDestroy(g.second.exec);
    for (int b = 0; b < 2; ++b) {
        if (copied_[b]) {
            cudaEventSynchronize(copied_[b]);
            cudaEventDestroy(copied_[b]);
        }
        if (staging_[b]) cudaFreeHost(staging_[b]);
    }
    for (auto& e : events_)
        if (e) cudaEventDestroy(e);
    if (capture_) cudaStreamDestroy(capture_);
    for (auto& e : tune_ev_)
        if (e) cudaEventDestroy(e);
}

void BatchCore::set_profiling(bool on) {
    if (on && !events_[0])
        for (auto& e : events_) check(cudaEventCreate(&e), "cudaEventCreate");
    profiling_ = on;
}

int BatchCore::stage_times(float* ms, int max_stages) const {
    if (!profiled_ || !ms) return -1;
    const int n = std::min(max_stages, (int)NUM_STAGES);
    for (int k = 0; k < n; ++k) {
        if (cudaEventElapsedTime(&ms[k], events_[2 * k], events_[2 * k + 1]) != cudaSuccess) {
            cudaGetLastError();
            return -1;
        }
    }
    return n;
}

namespace {
int log2i(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}
}  // namespace

void BatchCore::fill(SlotTable& T, int k, const SlotRequest& r, int variant) {
    std::memset(&T, 0, sizeof(T));
    const rvsb_scene* sc = r.scene;
    SlotWorkspace& ws = *ws_[k];
    const rvsb_camera& virt = r.virt;
    const rvsb_synth_params& p = r.params;
    const int n = (int)sc->cams.size();
    size_t voff = 0, boff = 0;
    for (int v = 0; v < n; ++v) {
        const rvsb_camera& c = sc->cams[v];
        DevView& V = T.v[v];
        V.w = c.width;
        V.h = c.height;
        V.proj = c.projection;
        V.bits_color = c.bit_depth_color;
        V.f0 = c.focal[0];
        V.f1 = c.focal[1];
        V.p0 = c.principle_point[0];
        V.p1 = c.principle_point[1];
        V.near_ = c.depth_range[0];
        V.far_ = c.depth_range[1];
        V.depth_scale = 1.0f / (float)((1u << c.bit_depth_depth) - 1u);
        V.has_invalid = c.has_invalid_depth;
        V.color_scale = 1.0f / (float)((1u << c.bit_depth_color) - 1u);
        V.cw = c.width / 2;
        V.ch = c.height / 2;
        V.chroma_sx = (float)V.cw / c.width;
        V.chroma_sy = (float)V.ch / c.height;
        relative_pose(c, virt, V.R, V.t);
        V.py = sc->plane(v, 0);
        V.pu = sc->plane(v, 1);
        V.pv = sc->plane(v, 2);
        V.pd = r.frame ? r.frame[v].depth : sc->plane(v, 3);
        if (c.projection == RVSB_PROJ_EQUIRECTANGULAR) {
            V.erp_row = sc->erp[v * 2 + 0]->as<float>();
            V.erp_col = sc->erp[v * 2 + 1]->as<float>();
            V.erp_cone = sc->erp_cone[v]->as<float4>();
            V.tile_depth = sc->tile_depth[v]->as<float2>();
        }
        V.color = sc->color[v]->as<uint64_t>();
        V.depth_lut = sc->depth_lut[v]->as<float4>();
        V.vert = ws.vert.as<float4>() + voff;
        V.bbox = ws.bbox.as<int4>() + boff;
        V.tri_shift = 2;
        while ((1 << (V.tri_shift - 2)) < c.width - 1) ++V.tri_shift;
        V.nbx = nblocks_x(c.width);
        V.nby = nblocks_y(c.height);
        voff += (size_t)c.width * c.height;
        boff += (size_t)V.nbx * V.nby;
    }
    DevTarget& D = T.t;
    const RasterDims rd = raster_dims(virt, p);
    D.wo = rd.w;
    D.ho = rd.h;
    D.out_w = virt.width;
    D.out_h = virt.height;
    D.precision = p.precision;
    if (rd.rescale) {
        D.rescale = 1;
        D.uv_sx = (float)rd.w / (float)virt.width;
        D.uv_sy = (float)rd.h / (float)virt.height;
        // cv::resize from the raster size to W x H: an exact 2x reduction
        // is an area mean, everything else bilinear.
        D.rs_scale_x = 1.0 / ((double)virt.width / rd.w);
        D.rs_scale_y = 1.0 / ((double)virt.height / rd.h);
        const int ix = (int)std::lrint(D.rs_scale_x), iy = (int)std::lrint(D.rs_scale_y);
        D.rs_area = std::fabs(D.rs_scale_x - ix) < 2.220446049250313e-16 &&
                    std::fabs(D.rs_scale_y - iy) < 2.220446049250313e-16 && ix == 2 && iy == 2;
    }
    D.proj = virt.projection;
    D.wrap = (virt.projection == RVSB_PROJ_EQUIRECTANGULAR && virt.full_hor_range) ? 1 : 0;
    D.f0 = virt.focal[0];
    D.f1 = virt.focal[1];
    D.p0 = virt.principle_point[0];
    D.p1 = virt.principle_point[1];
    if (virt.projection == RVSB_PROJ_EQUIRECTANGULAR) erp_projector_constants(virt, D.u0, D.v0, D.du_dphi, D.dv_dtheta);
    // ERP input tiles wholly beyond a side of a perspective output are
    // skipped, except when the warped vertices themselves are asked for.
    if (virt.projection == RVSB_PROJ_PERSPECTIVE && p.precision == 1.f && !r.dbg.warped_uvz) {
        const float f0 = virt.focal[0], f1 = virt.focal[1], p0 = virt.principle_point[0], p1 = virt.principle_point[1];
        const float W = (float)virt.width, H = (float)virt.height;
        const float planes[4][3] = {{-(p0 + 1.f), f0, 0.f},      // u < -1
                                    {p0 - W - 1.f, -f0, 0.f},    // u > W + 1
                                    {-(p1 + 1.f), 0.f, f1},      // v < -1
                                    {p1 - H - 1.f, 0.f, -f1}};   // v > H + 1
        std::memcpy(D.cull_plane, planes, sizeof(planes));
        D.cull = 1;
    }
    D.bits = virt.bit_depth_color;
    D.max_val = (1u << virt.bit_depth_color) - 1u;
    D.blend_exp = p.blending_factor;
    D.inv_blend_exp = 1.0f / p.blending_factor;
    D.blend_exp_int = 0;
    if (p.blending_factor == std::floor(p.blending_factor) && p.blending_factor >= 2.f && p.blending_factor <= 16.f)
        D.blend_exp_int = (int)p.blending_factor;
    D.chroma_ties_up = p.chroma_rounding == RVSB_CHROMA_TIES_UP;
    D.blend_max = p.blending_factor < 0.f ? 1 : 0;
    auto exp_int = [](float e) {
        return (e == std::floor(e) && e >= 2.f && e <= 16.f) ? (int)e : 0;
    };
    if (p.blending_method == RVSB_BLEND_MULTISPECTRAL) {
        // The raster's own blend follows the low band: its quality, holes,
        // depth and validity are the multispectral blender's.
        D.blend_exp = p.low_freq_factor;
        D.inv_blend_exp = 1.0f / p.low_freq_factor;
        D.blend_exp_int = exp_int(p.low_freq_factor);
        D.blend_max = p.low_freq_factor < 0.f ? 1 : 0;
        MsPtrs& M = T.ms;
        M.view = ws.ms_view.as<float4>();
        M.hsum = ws.ms_hsum.as<double>();
        M.hcnt = ws.ms_hcnt.as<int>();
        M.blur = ws.ms_blur.as<float>();
        M.on = 1;
        M.rad = std::max(rd.w, rd.h) / 20;
        M.low_exp = p.low_freq_factor;
        M.high_exp = p.high_freq_factor;
        M.low_int = exp_int(p.low_freq_factor);
        M.high_int = exp_int(p.high_freq_factor);
    }
    const RasterVariant& rv = kRasterVariants[variant];
    D.tile_wl = log2i(rv.tw);
    D.tile_hl = log2i(rv.th);
    D.ntx = (rd.w + rv.tw - 1) / rv.tw;
    D.nty = (rd.h + rv.th - 1) / rv.th;
    D.n_views = n;
    D.bin_capacity = (int)ws.cap_list;
    SlotBuffers& B = T.b;
    B.status = ws.status.as<DevStatus>();
    B.counts = ws.counts.as<int>();
    B.offsets = ws.offsets.as<int>();
    B.cursor = ws.cursor.as<int>();
    B.list = ws.list.as<int>();
    B.capacity = (int)ws.cap_list;
    B.codes = ws.codes.as<uint64_t>();
    B.holes = ws.holes.as<uint8_t>();
    for (int s = 0; s < 4; ++s) B.scan[s] = ws.scan[s].as<uint64_t>();
    B.inpaint_seg = ws.inpaint_seg.as<uint64_t>();
    B.tile_order = ws.tile_order.as<int>();
    if (rd.rescale) {
        B.pcolor = ws.pcolor.as<float4>();
        B.psrc = r.dbg.inpaint_source ? r.dbg.inpaint_source : ws.psrc.as<int32_t>();
    }
    T.out_y = r.out.y;
    T.out_u = r.out.u;
    T.out_v = r.out.v;
    T.dbg = r.dbg;
    if (r.aux) {
        AuxPtrs& A = T.aux;
        A.mask = r.aux->mask;
        A.masked_y = r.aux->masked.y;
        A.masked_u = r.aux->masked.u;
        A.masked_v = r.aux->masked.v;
        A.depth = r.aux->depth;
        A.masked_depth = r.aux->masked_depth;
        A.acc_depth = ws.aux_depth.as<float>();
        A.acc_valid = ws.aux_valid.as<float>();
        A.threshold = r.aux->validity_threshold;
        A.on = 1;
        A.depth_near = virt.depth_range[0];
        A.depth_far = virt.depth_range[1];
        A.depth_max = (1u << virt.bit_depth_depth) - 1u;
    }
}

BatchShape BatchCore::shape_of(const SlotRequest* reqs, int n, int variant) const {
    const RasterVariant& rv = kRasterVariants[variant];
    BatchShape sh;
    sh.slots = n;
    sh.variant = variant;
    for (int k = 0; k < n; ++k) {
        if (reqs[k].aux) sh.aux = 1;
        if (reqs[k].params.blending_method == RVSB_BLEND_MULTISPECTRAL) sh.ms = 1;
        if (reqs[k].params.precision != 1.f) sh.rescale = 1;
    }
    for (int k = 0; k < n; ++k) {
        const SlotRequest& r = reqs[k];
        const int nv = (int)r.scene->cams.size();
        sh.max_views = std::max(sh.max_views, nv);
        for (const auto& c : r.scene->cams) {
            sh.max_w = std::max(sh.max_w, c.width);
            sh.max_h = std::max(sh.max_h, c.height);
            sh.max_blocks = std::max(sh.max_blocks, nblocks_x(c.width) * nblocks_y(c.height));
        }
        const RasterDims rd = raster_dims(r.virt, r.params);
        const int ntiles = ((rd.w + rv.tw - 1) / rv.tw) * ((rd.h + rv.th - 1) / rv.th);
        sh.max_wo = std::max(sh.max_wo, rd.w);
        sh.max_ho = std::max(sh.max_ho, rd.h);
        sh.max_out_w = std::max(sh.max_out_w, r.virt.width);
        sh.max_out_h = std::max(sh.max_out_h, r.virt.height);
        sh.max_tiles = std::max(sh.max_tiles, ntiles);
        sh.max_bins = std::max(sh.max_bins, ntiles * nv);
    }
    return sh;
}

int BatchCore::launch_variant(const SlotRequest* reqs, int n, int variant, cudaStream_t s) {
    const BatchShape sh = shape_of(reqs, n, variant);
    if (n == 1 && !use_graphs_) {
        // A single synthesis: the table travels as a kernel parameter.
        TableParam tp;
        fill(tp.t, 0, reqs[0], variant);
        const int launches = launch_batch(tp, sh, s, profiling_ ? events_ : nullptr);
        if (launches < 0) check(cudaGetLastError(), "kernel launch");
        return launches;
    }
    // The staging buffer is reused every other call: its previous copy must
    // have been consumed.
    check(cudaEventSynchronize(copied_[cur_]), "wait for table staging");
    for (int k = 0; k < n; ++k) fill(staging_[cur_][k], k, reqs[k], variant);
    check(cudaMemcpyAsync(tables_.ptr, staging_[cur_], sizeof(SlotTable) * (size_t)n, cudaMemcpyHostToDevice, s),
          "upload slot tables");
    check(cudaEventRecord(copied_[cur_], s), "record table upload");
    cur_ ^= 1;
    const TablePtr tabs{tables_.as<SlotTable>()};
    if (use_graphs_ && !profiling_) {
        const std::vector<int> key = {sh.slots,  sh.variant, sh.max_views, sh.max_w,    sh.max_h,
                                      sh.max_blocks, sh.max_wo, sh.max_ho, sh.max_tiles, sh.max_bins, sh.aux, sh.ms,
                                      sh.rescale, sh.max_out_w, sh.max_out_h};
        auto it = graphs_.find(key);
        if (it == graphs_.end()) {
            cudaGraph_t g = nullptr;
            check(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal), "begin capture");
            const int nl = launch_batch(tabs, sh, capture_, nullptr);
            const cudaError_t ec = cudaStreamEndCapture(capture_, &g);
            if (nl < 0) check(cudaGetLastError(), "kernel launch (capture)");
            check(ec, "end capture");
            cudaGraphExec_t exec = nullptr;
            const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            check(ei, "graph instantiate");
            it = graphs_.emplace(key, Graph{exec, nl}).first;
        }
        check(cudaGraphLaunch(it->second.exec, s), "graph launch");
        return it->second.launches;
    }
    const int launches = launch_batch(tabs, sh, s, profiling_ ? events_ : nullptr);
    if (launches < 0) check(cudaGetLastError(), "kernel launch");
    return launches;
}

namespace {

// Pixels per radian at the centre of a camera: the focal length of a
// perspective camera, the width over the horizontal range of an
// equirectangular one.
float pixels_per_radian(const rvsb_camera& c) {
    if (c.projection == RVSB_PROJ_EQUIRECTANGULAR) {
        const float range = (c.hor_range[1] - c.hor_range[0]) * (3.14159265f / 180.f);
        return range > 0.f ? (float)c.width / range : 0.f;
    }
    return c.focal[0];
}

// Raster variant of a run that is neither pinned nor tuned.  An input pixel
// spacing seen m times magnified in the raster gives triangles whose
// candidate boxes hold about (m + 1)^2 pixels, so past m of about 1 most
// leave the small path (at most 4 candidates) and the medium path of variant
// 7 rasterises them faster: 960x540 inputs into a 1920x1080 output (m = 2)
// 0.359 -> 0.285 ms, 4096x2048 equirectangular inputs into 1920x1080
// (m = 1.47) 1.03 -> 0.62 ms; at m <= 1 it is 2 to 26% slower.  An
// equirectangular output stretches its rows by 1 / cos(latitude), sqrt(2) at
// the median row, which its m includes (equirectangular to equirectangular
// at m = 1: 4.30 -> 3.25 ms).  The largest m of the batch decides.
// At m <= 1.1 variant 4 (64x32 tiles, all four views in one z-buffer
// group, 1024-thread CTAs, one per SM) runs: a binning block lands in 1.35
// of its tiles instead of 1.53 of 32x32, the bins are half as many, and a
// tile's 32 warps finish it in about half the time of 16, which keeps the
// last wave short.  Against variant 0 (ms per view, median of 36 calls):
// 4 x 1920x1080 into 1920x1080 0.648 -> 0.621, into 960x540 0.459 -> 0.453,
// into an equirectangular 4096x2048 1.027 -> 0.943; 2 x 960x540 into
// 960x540 0.153 -> 0.150.  A perspective output minified to m <= 0.6 has
// many small triangles per tile, and the 32x32 tiles of variant 2 (also
// 1024-thread CTAs) rasterise it faster: 4 x 1920x1080 into 960x540 (m =
// 0.5) 0.450 -> 0.406 ms, into 640x360 (m = 0.33) 0.521 -> 0.440 ms; at m =
// 0.67 variant 4 is ahead again (0.452 against 0.466).  A batch of many
// slots has tiles enough that the last wave does not matter, and there two
// 512-thread CTAs per SM, one working while the other waits at a barrier,
// do better: variant 1 (64x32 tiles of two views) runs 16 poses of the
// 1080p scene at 1806 views/s and the 64-target mixed batch at 771,
// against 755 for variant 4.
constexpr int kMagnifiedVariant = 7;
constexpr int kDefaultVariant = 4;
constexpr int kMinifiedVariant = 2;
constexpr int kBatchVariant = 1;
constexpr int kBatchVariantMinSlots = 8;
static_assert(kRasterVariants[kMagnifiedVariant].med > kRasterVariants[kMagnifiedVariant].small,
              "the magnified default has the medium-triangle path");
static_assert(kRasterVariants[kDefaultVariant].tw == 64 && kRasterVariants[kDefaultVariant].vg == 4 &&
                  kRasterVariants[kDefaultVariant].threads == 1024,
              "the default holds 64x32 tiles of four views in 1024-thread CTAs");
static_assert(kRasterVariants[kMinifiedVariant].tw == 32 && kRasterVariants[kMinifiedVariant].threads == 1024,
              "the minified default holds 32x32 tiles in 1024-thread CTAs");
static_assert(kRasterVariants[kBatchVariant].threads == 512 && kRasterVariants[kBatchVariant].med == 0,
              "the batch default runs two CTAs per SM");

int default_variant(const SlotRequest* reqs, int n) {
    float m = 0.f;
    bool erp_out = false;
    for (int k = 0; k < n; ++k) {
        const SlotRequest& r = reqs[k];
        float in = 0.f;
        for (const rvsb_camera& c : r.scene->cams) in = std::max(in, pixels_per_radian(c));
        const RasterDims rd = raster_dims(r.virt, r.params);
        float out = pixels_per_radian(r.virt) * (float)rd.w / (float)r.virt.width;
        if (r.virt.projection == RVSB_PROJ_EQUIRECTANGULAR) {
            out *= 1.41421356f;
            erp_out = true;
        }
        if (in > 0.f) m = std::max(m, out / in);
    }
    if (m > 1.1f) return kMagnifiedVariant;
    if (!erp_out && m <= 0.6f) return kMinifiedVariant;
    return n >= kBatchVariantMinSlots ? kBatchVariant : kDefaultVariant;
}

}  // namespace

int BatchCore::tune(const SlotRequest* reqs, int n, cudaStream_t s) {
    const bool graphs = use_graphs_, prof = profiling_;
    use_graphs_ = false;
    profiling_ = false;
    // A warm-up run of every variant (first use of its module), then five
    // rounds that time each variant once, in turn, so that a drift of the
    // device's state affects them alike; the variant with the smallest median
    // wins if it beats the untuned default's median by at least 2%, else the
    // default stays.  One run alone is too noisy to rank variants a few
    // percent apart, and among variants within the noise of each other the
    // pick would otherwise be arbitrary (measured: a 1.7% slower one picked
    // for the plain 1080p view).
    constexpr int kRounds = 5;
    for (int v = 0; v < NUM_RASTER_VARIANTS; ++v) launch_variant(reqs, n, v, s);
    float t[NUM_RASTER_VARIANTS][kRounds];
    for (int r = 0; r < kRounds; ++r)
        for (int v = 0; v < NUM_RASTER_VARIANTS; ++v) {
            check(cudaEventRecord(tune_ev_[0], s), "record");
            launch_variant(reqs, n, v, s);
            check(cudaEventRecord(tune_ev_[1], s), "record");
            check(cudaEventSynchronize(tune_ev_[1]), "synchronize");
            check(cudaEventElapsedTime(&t[v][r], tune_ev_[0], tune_ev_[1]), "elapsed");
        }
    int best = 0;
    float best_ms = 0.f, med[NUM_RASTER_VARIANTS];
    for (int v = 0; v < NUM_RASTER_VARIANTS; ++v) {
        std::sort(t[v], t[v] + kRounds);
        med[v] = t[v][kRounds / 2];
        if (v == 0 || med[v] < best_ms) {
            best = v;
            best_ms = med[v];
        }
    }
    const int fallback = default_variant(reqs, n);
    if (best_ms > 0.98f * med[fallback]) best = fallback;
    use_graphs_ = graphs;
    profiling_ = prof;
    return best;
}

int BatchCore::run(const SlotRequest* reqs, int n, cudaStream_t s) {
    HostRange range("rvsb: batch (tables, launches)");
    if (n <= 0 || n > slots_) throw ArgError("batch of " + std::to_string(n) + " requests for " +
                                             std::to_string(slots_) + " slots");
    int ms_wo = 0;
    for (int k = 0; k < n; ++k) {
        const SlotRequest& r = reqs[k];
        const RasterDims rd = raster_dims(r.virt, r.params);
        if (rd.rescale && r.aux && r.aux->masked.y)
            throw Unsupported("MaskedOutputFiles needs Precision 1: the reference masks the raster-sized colour "
                              "with the mask resized to the output size (Pipeline.cpp:314-318), which OpenCV "
                              "rejects");
        ws_[k]->ensure(ctx_, r.scene, rd.w, rd.h);
        if (r.aux) ws_[k]->ensure_aux(ctx_, rd.w, rd.h);
        if (rd.rescale) ws_[k]->ensure_rescale(ctx_, rd.w, rd.h);
        if (r.params.blending_method == RVSB_BLEND_MULTISPECTRAL) {
            ws_[k]->ensure_ms(ctx_, (int)r.scene->cams.size(), rd.w, rd.h);
            ms_wo = std::max(ms_wo, rd.w);
        }
    }
    if (ms_wo > 0) prepare_ms_kernels(ms_wo);
    int variant = default_variant(reqs, n);
    if (forced_variant_ >= 0) {
        variant = forced_variant_;
    } else if (autotune_) {
        // The shape the tuner keys on: the batch size bucket and, over the
        // batch, the largest input set and output and the projections.
        const BatchShape sh = shape_of(reqs, n, 0);
        int proj_in = 0, proj_out = 0;
        for (int k = 0; k < n; ++k) {
            proj_in |= 1 << reqs[k].scene->cams[0].projection;
            proj_out |= 1 << reqs[k].virt.projection;
        }
        const int bucket = n == 1 ? 1 : n <= 4 ? 4 : n <= 16 ? 16 : 64;
        const std::vector<int> sig = {bucket, sh.max_views, sh.max_w, sh.max_h, sh.max_wo, sh.max_ho,
                                      proj_in, proj_out, sh.max_out_w, sh.max_out_h};
        auto it = tuned_.find(sig);
        if (it == tuned_.end()) it = tuned_.emplace(sig, tune(reqs, n, s)).first;
        variant = it->second;
    }
    const int launches = launch_variant(reqs, n, variant, s);
    profiled_ = profiling_;
    last_launches_ = launches;
    last_variant_ = variant;
    return launches;
}

}  // namespace rvsb
