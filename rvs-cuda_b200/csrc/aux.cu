// Auxiliary outputs of a synthesis (Pipeline.cpp:303-336, CPU mode), after
// inpainting: the validity mask (View::get_validity_mask, View.cpp:206-211),
// the masked colour (colour set to 0.5 where masked, then write_color), the
// blended depth and the masked depth (write_maskedDepth,
// image_writing.cpp:237-268).  One thread per 2x2 output block.
#include <algorithm>

#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

// Normalised disparity of write_maskedDepth, converted with
// convertTo(CV_16U, 2^bits - 1): rounded to nearest (ties to even) and
// saturated; NaN gives 0.
__device__ __forceinline__ uint16_t encode_depth(float depth, const AuxPtrs& A, bool masked) {
    float d;
    if (A.depth_far >= 1000.f)
        d = __fdiv_rn(A.depth_near, depth);
    else
        d = __fdiv_rn(__fsub_rn(__fdiv_rn(__fmul_rn(A.depth_far, A.depth_near), depth), A.depth_near),
                      __fsub_rn(A.depth_far, A.depth_near));
    if (masked) d = 0.f;
    const float v = __fmul_rn(d, (float)A.depth_max);
    if (isnan(v)) return 0;
    const float r = rintf(v);
    return (uint16_t)fminf(65535.f, fmaxf(0.f, r));
}

// Blended depth at output pixel (x, y) of a synthesis rasterised at
// Precision != 1: cv::resize of the raster-sized depth to the output size
// with INTER_LINEAR (Pipeline.cpp:323-333), as resize.cu does for the
// colour: the area mean of an exact 2x reduction, else two linear passes.
__device__ __forceinline__ float resized_depth(const DevTarget& T, const float* d, int x, int y) {
    const int w = T.wo;
    if (T.rs_area) {
        const float a = d[(size_t)(2 * y) * w + 2 * x], b = d[(size_t)(2 * y) * w + 2 * x + 1];
        const float c = d[(size_t)(2 * y + 1) * w + 2 * x], e = d[(size_t)(2 * y + 1) * w + 2 * x + 1];
        return __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(a, b), c), e), 0.25f);
    }
    int sx0, sx1, sy0, sy1;
    float fx, fy;
    linear_tap(x, T.rs_scale_x, T.wo, sx0, sx1, fx);
    linear_tap(y, T.rs_scale_y, T.ho, sy0, sy1, fy);
    const float a0 = __fsub_rn(1.f, fx), b0 = __fsub_rn(1.f, fy);
    const float r0 = lerp2(d[(size_t)sy0 * w + sx0], d[(size_t)sy0 * w + sx1], a0, fx);
    const float r1 = lerp2(d[(size_t)sy1 * w + sx0], d[(size_t)sy1 * w + sx1], a0, fx);
    return lerp2(r0, r1, b0, fy);
}

// Raster index of output index d for cv::resize with INTER_NEAREST
// (resizeNN): min(floor(d * (1 / (out / raster))), raster - 1), in double.
__device__ __forceinline__ int nearest_src(int d, int out, int raster) {
    const double ifx = __drcp_rn(__ddiv_rn((double)out, (double)raster));
    return min((int)floor(__dmul_rn((double)d, ifx)), raster - 1);
}

// One thread per 2x2 block of the output (the virtual camera's size).  At
// Precision != 1 the validity mask and the depth are computed at the raster
// size and resized to the output (Pipeline.cpp:303-333): the mask with
// INTER_NEAREST, the depth with INTER_LINEAR; the masked colour is not
// produced there (the host refuses it).
template <class Tabs>
__global__ void aux_kernel(const __grid_constant__ Tabs tabs) {
    grid_dep_wait();
    const SlotTable& tab = tabs.at(blockIdx.z);
    const AuxPtrs& A = tab.aux;
    if (!A.on) return;
    const DevTarget& T = tab.t;
    const int ow = T.rescale ? T.out_w : T.wo, oh = T.rescale ? T.out_h : T.ho;
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y;
    const int x0 = 2 * bx, y0 = 2 * by;
    if (x0 >= ow || y0 >= oh) return;
    const uint32_t grey = quantize(0.5f, T.max_val);
    uint32_t su = 0, sv = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int x = x0 + (p & 1), y = y0 + (p >> 1);
        const size_t o = (size_t)y * ow + x;
        const size_t ov = T.rescale ? (size_t)nearest_src(y, oh, T.ho) * T.wo + nearest_src(x, ow, T.wo) : o;
        const bool masked = !(A.acc_valid[ov] > A.threshold);
        if (A.mask) A.mask[o] = masked ? 255 : 0;
        if (A.masked_y) {
            const uint64_t c = tab.b.codes[o];
            const uint32_t yy = masked ? grey : (uint32_t)(c & 0xffff);
            su += masked ? grey : (uint32_t)((c >> 16) & 0xffff);
            sv += masked ? grey : (uint32_t)((c >> 32) & 0xffff);
            A.masked_y[o] = (uint16_t)yy;
        }
        if (A.depth || A.masked_depth) {
            const float dep = T.rescale ? resized_depth(T, A.acc_depth, x, y) : A.acc_depth[o];
            if (A.depth) A.depth[o] = encode_depth(dep, A, false);
            if (A.masked_depth) A.masked_depth[o] = encode_depth(dep, A, masked);
        }
    }
    if (A.masked_y) {
        const size_t co = (size_t)by * (T.wo / 2) + bx;
        A.masked_u[co] = quarter_round(su, T.chroma_ties_up);
        A.masked_v[co] = quarter_round(sv, T.chroma_ties_up);
    }
}

}  // namespace

template <class Tabs>
void launch_aux(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    // Output blocks: the raster size, or the output size where a slot
    // rasterises at Precision != 1.
    const int w = std::max(sh.max_wo, sh.max_out_w), h = std::max(sh.max_ho, sh.max_out_h);
    launch_dependent(aux_kernel<Tabs>, dim3((w / 2 + 127) / 128, h / 2, sh.slots), dim3(128), 0, s, tabs);
}

template void launch_aux<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template void launch_aux<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

}  // namespace rvsb
