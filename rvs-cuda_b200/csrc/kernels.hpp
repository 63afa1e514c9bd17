// Host-side interface of the synthesis kernels (kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_types.hpp"

namespace rvsb {

// Grid extents of one batch launch: maxima over its slots.
struct BatchShape {
    int slots = 0;
    int variant = 0;         // raster variant (kRasterVariants)
    int aux = 0;             // some slot wants auxiliary outputs
    int ms = 0;              // some slot blends multispectrally
    int max_views = 0;       // largest n_views
    int max_w = 0, max_h = 0;  // largest input view
    int max_blocks = 0;      // largest nbx * nby of an input view
    int max_wo = 0, max_ho = 0;
    int max_tiles = 0;       // largest ntx * nty
    int max_bins = 0;        // largest ntx * nty * n_views
    int rescale = 0;         // some slot rasterises at Precision != 1
    int max_out_w = 0, max_out_h = 0;  // largest output (virtual camera) size
};

// Where the kernels find the slot tables.  A single synthesis passes its
// table as a kernel parameter (read through the constant bank); a batch
// passes a device array of tables, indexed by the slot grid dimension, so
// its launch sequence does not change from call to call (CUDA graphs).
#ifdef __CUDACC__
#define RVSB_HD __host__ __device__
#else
#define RVSB_HD
#endif
struct TableParam {
    SlotTable t;
    RVSB_HD const SlotTable& at(int) const { return t; }
};
struct TablePtr {
    const SlotTable* p;
    RVSB_HD const SlotTable& at(int slot) const { return p[slot]; }
};
#undef RVSB_HD

// Launches `kernel` after the previous kernel on `s` with programmatic
// dependent launch: its CTAs are scheduled while the previous kernel drains
// and wait in grid_dep_wait() (device_common.cuh) until it has finished, which
// hides the launch gap between the dependent kernels of a synthesis.
template <class... KArgs, class... Args>
void launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Issues one batch of syntheses on `stream`; returns the number of kernel
// launches, or -1 on a launch error (cudaGetLastError holds the cause).
// `events` (optional) holds 2 * NUM_STAGES events recorded around the stages.
constexpr int NUM_STAGES = 5;
template <class Tabs>
int launch_batch(const Tabs& tabs, const BatchShape& shape, cudaStream_t stream, cudaEvent_t* events = nullptr);

// Raster variants the autotuner chooses from: tile width and height, views
// per shared z-buffer group, the candidate count above which a triangle is
// rasterised warp-cooperatively, the bin entries staged per round, and the
// candidate count up to which those triangles are flattened across the warp
// together (med <= small: each one alone, row span by row span).  Every
// variant gives identical results.
struct RasterVariant {
    int tw, th, vg, small, ent, med, threads;
};
constexpr int NUM_RASTER_VARIANTS = 8;
constexpr RasterVariant kRasterVariants[NUM_RASTER_VARIANTS] = {
    {32, 32, 4, 4, 1024, 0, 512},  {64, 32, 2, 4, 1024, 0, 512},   {32, 32, 4, 4, 1024, 0, 1024},
    {32, 32, 4, 8, 1024, 0, 512},  {64, 32, 4, 4, 1024, 0, 1024},  {64, 32, 2, 4, 1024, 32, 1024},
    {32, 32, 4, 2, 1024, 32, 512}, {64, 32, 2, 4, 1024, 32, 512},
};
// The bin arrays are sized for tiles of MIN_TILE_W x MIN_TILE_H.
constexpr bool tiles_at_least_minimum() {
    for (const RasterVariant& v : kRasterVariants)
        if (v.tw < MIN_TILE_W || v.th < MIN_TILE_H) return false;
    return true;
}
static_assert(tiles_at_least_minimum(), "a raster variant's tiles are smaller than the bins are sized for");

// One-time kernel attributes of the current device (the raster kernel's
// dynamic shared memory); call before launching or capturing a batch.
void prepare_kernels();
// Shared memory of the multispectral row sums for outputs up to max_wo wide.
void prepare_ms_kernels(int max_wo);

// Colour planes of up to MAX_VIEWS views decoded in one launch.
struct DecodeJob {
    const uint16_t* y;
    const uint16_t* u;
    const uint16_t* v;
    uint64_t* out;
    int w, h;
};
struct DecodeJobs {
    DecodeJob v[MAX_VIEWS];
};
// Precision != 1: resize of the raster-size colour to the output and its
// 4:2:0 write, one launch for all slots that rescale.
template <class Tabs>
void launch_resize(const Tabs& tabs, const BatchShape& shape, cudaStream_t stream);

void launch_decode_views(const DecodeJobs& jobs, int n, int max_w, int max_h, cudaStream_t s);

// The depth table of one input view: for every 16-bit sample the decoded
// depth d (normalised disparity with near / far,
// rvs_cuda_lib/src/process_input_frame.cu:346-385) and the perspective
// unprojection factors -(d / f0), -(d / f1); 65536 float4.
void launch_depth_lut(float near_, float far_, float depth_scale, int has_invalid, float f0, float f1, float4* out,
                      cudaStream_t s);

// Depth range (min, max) of every WARP_TILE x WARP_TILE vertex tile grown by
// one pixel, for the ERP input culling; up to MAX_VIEWS views in one launch.
struct TileDepthJob {
    const uint16_t* depth;   // raw depth plane
    const float4* lut;       // the view's depth table (decoded depth in .x)
    float2* out;             // one (min, max) per tile, row-major
    int w, h;
};
struct TileDepthJobs {
    TileDepthJob v[MAX_VIEWS];
};
void launch_tile_depth(const TileDepthJobs& jobs, int n, int max_w, int max_h, cudaStream_t s);

// Decodes the colour planes of one input view into packed per-pixel words.
void launch_decode_color(const uint16_t* y, const uint16_t* u, const uint16_t* v, int w, int h, uint64_t* out,
                         cudaStream_t s);

// Inpainting of one image outside a batch (no slot table): the scans over
// `holes` with caller-provided scratch (status, codes and four scan buffers
// of w*h words each); the chosen source of every hole goes to `sources`.
// Words of a slot's inpainting column-minima table for outputs up to wo
// wide (group minima and warp-segment minima of the column pre-passes).
size_t inpaint_seg_words(int wo);

void launch_inpaint_scans(DevStatus* st, const uint8_t* holes, uint64_t* codes, uint64_t* const scan[4], int w,
                          int h, int32_t* sources, cudaStream_t s);

}  // namespace rvsb
