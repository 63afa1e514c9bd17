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

// One 2x2 block of pixels per thread: the four chroma samples around
// chroma position (bx, by) serve all four pixels (their upsample weights
// are 2, 1 (x) 2, 1 with the block's parity), and the block is stored as two
// 16-byte rows.
__device__ __forceinline__ void decode_block(const uint16_t* __restrict__ py, const uint16_t* __restrict__ pu,
                                             const uint16_t* __restrict__ pv, int w, int h, int bx, int by,
                                             uint64_t* __restrict__ out) {
    const int cw = w / 2, ch = h / 2;
    const int x1 = bx, y1 = by;
    const int x2 = min(x1 + 1, cw - 1), y2 = min(y1 + 1, ch - 1);
    const uint32_t ua = __ldg(pu + y1 * cw + x1), ub = __ldg(pu + y1 * cw + x2);
    const uint32_t uc = __ldg(pu + y2 * cw + x1), ud = __ldg(pu + y2 * cw + x2);
    const uint32_t va = __ldg(pv + y1 * cw + x1), vb = __ldg(pv + y1 * cw + x2);
    const uint32_t vc = __ldg(pv + y2 * cw + x1), vd = __ldg(pv + y2 * cw + x2);
    const size_t o = (size_t)(2 * by) * w + 2 * bx;
    // Luma as single samples: the caller's plane pointers need only the
    // 2-byte alignment of their type.
    const uint32_t ya = __ldg(py + o), yb = __ldg(py + o + 1);
    const uint32_t yc = __ldg(py + o + w), yd = __ldg(py + o + w + 1);
    // chroma4 (device_common.cuh) at the four parities: (ox, oy) =
    // (0,0): 4a; (1,0): 2a+2b; (0,1): 2a+2c; (1,1): a+b+c+d.
    const uint32_t u00 = 4 * ua, u10 = 2 * ua + 2 * ub, u01 = 2 * ua + 2 * uc, u11 = ua + ub + uc + ud;
    const uint32_t v00 = 4 * va, v10 = 2 * va + 2 * vb, v01 = 2 * va + 2 * vc, v11 = va + vb + vc + vd;
    auto word = [](uint32_t yy, uint32_t u4, uint32_t v4) -> unsigned long long {
        return (unsigned long long)yy | ((unsigned long long)u4 << 18) | ((unsigned long long)v4 << 36);
    };
    reinterpret_cast<ulonglong2*>(out + o)[0] = make_ulonglong2(word(ya, u00, v00), word(yb, u10, v10));
    reinterpret_cast<ulonglong2*>(out + o + w)[0] = make_ulonglong2(word(yc, u01, v01), word(yd, u11, v11));
}

__global__ void decode_color_kernel(const uint16_t* __restrict__ py, const uint16_t* __restrict__ pu,
                                    const uint16_t* __restrict__ pv, int w, int h, uint64_t* __restrict__ out) {
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y;
    if (bx >= w / 2 || by >= h / 2) return;
    decode_block(py, pu, pv, w, h, bx, by, out);
}

// All views of a frame in one launch: grid (ceil(max_w / 2 / 128), max_h / 2, views).
__global__ void decode_views_kernel(const __grid_constant__ DecodeJobs jobs) {
    grid_dep_wait();
    const DecodeJob& J = jobs.v[blockIdx.z];
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y;
    if (bx >= J.w / 2 || by >= J.h / 2) return;
    decode_block(J.y, J.u, J.v, J.w, J.h, bx, by, J.out);
}

}  // namespace

void launch_decode_views(const DecodeJobs& jobs, int n, int max_w, int max_h, cudaStream_t s) {
    launch_dependent(decode_views_kernel, dim3((max_w / 2 + 127) / 128, max_h / 2, n), dim3(128), 0, s, jobs);
}

void launch_decode_color(const uint16_t* y, const uint16_t* u, const uint16_t* v, int w, int h, uint64_t* out,
                         cudaStream_t s) {
    decode_color_kernel<<<dim3((w / 2 + 127) / 128, h / 2), 128, 0, s>>>(y, u, v, w, h, out);
}

}  // namespace rvsb
