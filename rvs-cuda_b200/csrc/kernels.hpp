// Host-side interface of the synthesis kernels (kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_types.hpp"

namespace rvsb {

// Device buffers of one synthesis workspace.
struct SynthBuffers {
    DevStatus* status = nullptr;   // 1 entry (device)
    int* counts = nullptr;         // ntiles * n_views
    int* offsets = nullptr;        // ntiles * n_views
    int* cursor = nullptr;         // ntiles * n_views
    int* list = nullptr;           // bin list, `capacity` entries
    int capacity = 0;
    uint64_t* codes = nullptr;     // Wo*Ho packed output codes + hole bit
    uint8_t* holes = nullptr;      // Wo*Ho hole mask (1 = no view covers the pixel)
    uint64_t* scan_a = nullptr;    // Wo*Ho inpainting scratch
    uint64_t* scan_b = nullptr;
    uint64_t* scan_c = nullptr;
    uint64_t* scan_d = nullptr;
};

// Optional intermediate outputs (device pointers, may be null).
struct DebugPtrs {
    float* warped_uvz = nullptr;
    float* view_color = nullptr;
    float* view_depth = nullptr;
    float* view_validity = nullptr;
    float* blend_color = nullptr;
    float* blend_quality = nullptr;
    int32_t* inpaint_source = nullptr;
    bool any() const {
        return warped_uvz || view_color || view_depth || view_validity || blend_color ||
               blend_quality || inpaint_source;
    }
};

// Sizes the launch code needs on the host.
struct LaunchShape {
    int n_views;
    int max_w, max_h;        // largest input view
    int max_blocks;          // largest nbx * nby
    int wo, ho;
    int ntx, nty;
    int chroma_ties_up;      // output chroma mean: 1 rounds ties up, 0 to even
    int input_w[MAX_VIEWS];  // per view (for the debug copy of warped vertices)
    int input_h[MAX_VIEWS];
    int64_t vert_offset[MAX_VIEWS];  // element offset of each view's vertices in the vertex arena
};

// Issues the whole synthesis on `stream`; returns the number of kernel
// launches, or -1 on a launch error (cudaGetLastError holds the cause).
// Decodes the colour planes of one input view into packed per-pixel words.
void launch_decode_color(const uint16_t* y, const uint16_t* u, const uint16_t* v, int w, int h, uint64_t* out,
                         cudaStream_t s);

// Inpainting scans only, on caller-provided scratch (see inpaint.cu).
void launch_inpaint_scans(const DevStatus* st, const uint8_t* holes, uint64_t* codes, uint64_t* const scan[4], int w,
                          int h, int32_t* sources, cudaStream_t s);

// `events` (optional) holds 2 * NUM_STAGES events recorded around the stages.
constexpr int NUM_STAGES = 5;
int launch_synthesis(const SynthBuffers& b, const ViewTable& tab, const LaunchShape& shape, const DebugPtrs& dbg,
                     uint16_t* out_y, uint16_t* out_u, uint16_t* out_v, cudaStream_t stream,
                     cudaEvent_t* events = nullptr);

}  // namespace rvsb
