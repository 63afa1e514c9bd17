// Host engine under the C ABI: device memory accounting, input scenes,
// slot workspaces and batch launches (slot tables, CUDA graphs).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.hpp"
#include "rvsb.h"

namespace rvsb {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct BudgetError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ArgError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char* what);

// An NVTX range over a host stage (header-only NVTX 3: a no-op unless a
// profiler such as Nsight Systems is attached), so the host side of a
// synthesis shows beside its kernels on a timeline.
struct HostRange {
    explicit HostRange(const char* name) { nvtxRangePushA(name); }
    ~HostRange() { nvtxRangePop(); }
    HostRange(const HostRange&) = delete;
    HostRange& operator=(const HostRange&) = delete;
};

}  // namespace rvsb

struct rvsb_context {
    int device = 0;
    size_t budget = 0;
    size_t in_use = 0;
    std::string last_error;
    std::mutex mu;                     // serialises rvsb_synthesize_host
    std::mutex mem_mu;                 // guards in_use
    rvsb_scene* host_scene = nullptr;  // scene reused by rvsb_synthesize_host
    void* host_out = nullptr;          // device output staging of rvsb_synthesize_host
    size_t host_out_bytes = 0;
};

namespace rvsb {

// Device allocation counted against the context's HBM budget.
struct DevMem {
    rvsb_context* ctx = nullptr;
    void* ptr = nullptr;
    size_t bytes = 0;

    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { release(); }

    void alloc(rvsb_context* c, size_t n);
    void release();
    template <class T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

// Buffers of one synthesis slot, grown on demand to the largest request
// seen: the warped vertices and block boxes of every input view, the bins,
// and the output-sized codes, hole mask and inpainting scratch.
struct SlotWorkspace {
    DevMem status, counts, offsets, cursor, list, codes, holes, scan[4], vert, bbox;
    DevMem aux_depth, aux_valid;  // blended depth / validity (auxiliary outputs only)
    DevMem inpaint_seg;           // column-group minima of the inpainting passes
    DevMem tile_order;            // raster launch order of the output tiles
    size_t cap_tiles = 0;
    DevMem ms_view, ms_hsum, ms_hcnt, ms_blur;  // multispectral blending only
    size_t cap_ms = 0;            // view-pixels the multispectral buffers hold
    void ensure_ms(rvsb_context* ctx, int n_views, int wo, int ho);
    DevMem pcolor, psrc;          // Precision != 1: raster-size colour and inpainting sources
    size_t cap_rescale = 0;
    void ensure_rescale(rvsb_context* ctx, int wo, int ho);
    size_t cap_vert = 0, cap_bbox = 0, cap_out = 0, cap_bins = 0, cap_list = 0, cap_aux = 0, cap_seg_words = 0;
    void ensure_aux(rvsb_context* ctx, int wo, int ho);

    // Bytes a slot needs for `scene` at raster size wo x ho (rescale: plus
    // the buffers of a Precision != 1 synthesis).
    static size_t bytes_for(const rvsb_scene* scene, int wo, int ho, bool rescale = false);
    void ensure(rvsb_context* ctx, const rvsb_scene* scene, int wo, int ho);
};

// Raster size of a synthesis: the virtual camera's size, or for Precision
// P != 1 int(0.5 + W * P) x int(0.5 + H * P) (SynthesizedView.cpp:326-329),
// rasterised with uv scaled by raster size / W and H and resized to W x H
// when written.  Throws Unsupported for a P that is not finite and positive
// or for a raster size that is not even in both dimensions (the raster's
// 4:2:0 tile writer and inpainting work on 2x2 blocks).
struct RasterDims {
    int w, h;
    bool rescale;
};
RasterDims raster_dims(const rvsb_camera& virt, const rvsb_synth_params& p);

// Number of binning blocks of a view (BLOCK_W x BLOCK_H quads).
int nblocks_x(int w);
int nblocks_y(int h);

// One synthesis request of a batch.
struct SlotRequest {
    const rvsb_scene* scene = nullptr;
    rvsb_camera virt{};
    rvsb_synth_params params{};
    rvsb_yuv420 out{};
    DebugPtrs dbg{};
    const rvsb_view_planes* frame = nullptr;  // optional raw device planes (depth read in place)
    const rvsb_aux_out* aux = nullptr;        // optional auxiliary outputs
};

// Slot tables in device memory, their pinned host staging, and the launch
// of a batch of up to `slots` requests.  Calls on one core must be ordered
// (one stream, or the caller waits): the device tables are reused.
class BatchCore {
public:
    BatchCore(rvsb_context* ctx, int slots);
    ~BatchCore();
    BatchCore(const BatchCore&) = delete;
    BatchCore& operator=(const BatchCore&) = delete;

    int slots() const { return slots_; }
    SlotWorkspace& workspace(int k) { return *ws_[k]; }

    // Sizes the slot workspaces for the requests, fills and uploads their
    // tables and issues the batch on `stream`.  Returns the kernel launches.
    int run(const SlotRequest* reqs, int n, cudaStream_t stream);

    void set_graphs(bool on) { use_graphs_ = on; }
    // Time every raster variant on the first batch of each new shape and
    // keep the fastest (all variants give identical results).
    void set_autotune(bool on) { autotune_ = on; }
    // Use raster variant v for every run (-1: default or tuned).
    void force_variant(int v) { forced_variant_ = v; }
    // Variant used by the last run, and the tuner's choices so far.
    int last_variant() const { return last_variant_; }
    void set_profiling(bool on);
    // Milliseconds per stage of the last profiled run (stream complete).
    int stage_times(float* ms, int max_stages) const;
    int last_launches() const { return last_launches_; }

private:
    void fill(SlotTable& t, int k, const SlotRequest& r, int variant);
    BatchShape shape_of(const SlotRequest* reqs, int n, int variant) const;
    int launch_variant(const SlotRequest* reqs, int n, int variant, cudaStream_t s);
    int tune(const SlotRequest* reqs, int n, cudaStream_t s);

    rvsb_context* ctx_;
    int slots_;
    std::vector<std::unique_ptr<SlotWorkspace>> ws_;
    DevMem tables_;
    SlotTable* staging_[2] = {nullptr, nullptr};
    cudaEvent_t copied_[2] = {nullptr, nullptr};
    int cur_ = 0;
    bool use_graphs_ = false;
    cudaStream_t capture_ = nullptr;  // private stream the graphs are captured on
    struct Graph {
        cudaGraphExec_t exec;
        int launches;
    };
    std::map<std::vector<int>, Graph> graphs_;
    bool profiling_ = false;
    bool profiled_ = false;
    cudaEvent_t events_[2 * NUM_STAGES] = {};
    int last_launches_ = 0;
    bool autotune_ = false;
    int forced_variant_ = -1;
    int last_variant_ = 0;
    std::map<std::vector<int>, int> tuned_;
    cudaEvent_t tune_ev_[2] = {nullptr, nullptr};
};

}  // namespace rvsb

struct rvsb_scene {
    rvsb_context* ctx = nullptr;
    std::vector<rvsb_camera> cams;
    // 1 per view: the raw y, u, v and depth planes back to back, so that a
    // view whose planes are adjacent in host memory uploads in one copy.
    std::vector<std::unique_ptr<rvsb::DevMem>> raw;
    std::vector<std::unique_ptr<rvsb::DevMem>> erp;     // 2 per view: rows, cols (ERP inputs)
    std::vector<std::unique_ptr<rvsb::DevMem>> color;   // 1 per view: decoded colour words
    std::vector<std::unique_ptr<rvsb::DevMem>> depth_lut;  // 1 per view: 65536 x (d, -d/f0, -d/f1, 0)
    // ERP views: per vertex tile, direction cone and depth range (culling)
    std::vector<std::unique_ptr<rvsb::DevMem>> erp_cone, tile_depth;
    std::vector<bool> uploaded;
    std::unique_ptr<rvsb::BatchCore> single;            // the per-view calls: a batch of one
    int last_launches = 0;

    // Plane k (y, u, v, depth) of view v in its raw block.
    uint16_t* plane(int v, int k) const {
        const rvsb_camera& c = cams[v];
        const size_t ny = (size_t)c.width * c.height, nc = (size_t)(c.width / 2) * (c.height / 2);
        const size_t off[4] = {0, ny, ny + nc, ny + 2 * nc};
        return raw[v]->as<uint16_t>() + off[k];
    }
};
