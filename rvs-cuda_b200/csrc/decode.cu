// Colour decode of one input view: the loader's chroma upsample and merge
// (read_color_YUV, rvs/src/image_loading.cpp:74-145; resizeUV and mergeYUV,
// rvs_cuda_lib/src/process_input_frame.cu:22-81, 211-238), stored as exact
// integers per pixel: Y | 4U << 18 | 4V << 36.  4U and 4V are integers
// because the 2x upsample of an even-sized view has weights 0 or 1/2; the
// colour the reference computes is then (Y * s, 4U * 0.25 * s, 4V * 0.25 * s)
// with s = 1 / (2^bits - 1), bit for bit.
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

__global__ void decode_color_kernel(const uint16_t* __restrict__ py, const uint16_t* __restrict__ pu,
                                    const uint16_t* __restrict__ pv, int w, int h, uint64_t* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= w || i >= h) return;
    const int cw = w / 2, ch = h / 2;
    const size_t o = (size_t)i * w + j;
    out[o] = (uint64_t)py[o] | ((uint64_t)chroma4(pu, cw, ch, j, i) << 18) |
             ((uint64_t)chroma4(pv, cw, ch, j, i) << 36);
}

// All views of a frame in one launch: grid (ceil(max_w / 256), max_h, views).
__global__ void decode_views_kernel(const __grid_constant__ DecodeJobs jobs) {
    const DecodeJob& J = jobs.v[blockIdx.z];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= J.w || i >= J.h) return;
    const int cw = J.w / 2, ch = J.h / 2;
    const size_t o = (size_t)i * J.w + j;
    J.out[o] = (uint64_t)J.y[o] | ((uint64_t)chroma4(J.u, cw, ch, j, i) << 18) |
               ((uint64_t)chroma4(J.v, cw, ch, j, i) << 36);
}

}  // namespace

void launch_decode_views(const DecodeJobs& jobs, int n, int max_w, int max_h, cudaStream_t s) {
    decode_views_kernel<<<dim3((max_w + 255) / 256, max_h, n), 256, 0, s>>>(jobs);
}

void launch_decode_color(const uint16_t* y, const uint16_t* u, const uint16_t* v, int w, int h, uint64_t* out,
                         cudaStream_t s) {
    decode_color_kernel<<<dim3((w + 255) / 256, h), 256, 0, s>>>(y, u, v, w, h, out);
}

}  // namespace rvsb
