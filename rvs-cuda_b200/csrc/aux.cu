// Auxiliary outputs of a synthesis (Pipeline.cpp:303-336, CPU mode), after
// inpainting: the validity mask (View::get_validity_mask, View.cpp:206-211),
// the masked colour (colour set to 0.5 where masked, then write_color), the
// blended depth and the masked depth (write_maskedDepth,
// image_writing.cpp:237-268).  One thread per 2x2 output block.
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

template <class Tabs>
__global__ void aux_kernel(const __grid_constant__ Tabs tabs) {
    grid_dep_wait();
    const SlotTable& tab = tabs.at(blockIdx.z);
    const AuxPtrs& A = tab.aux;
    if (!A.on) return;
    const DevTarget& T = tab.t;
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y;
    const int x0 = 2 * bx, y0 = 2 * by;
    if (x0 >= T.wo || y0 >= T.ho) return;
    const uint32_t grey = quantize(0.5f, T.max_val);
    uint32_t su = 0, sv = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int x = x0 + (p & 1), y = y0 + (p >> 1);
        const size_t o = (size_t)y * T.wo + x;
        const bool masked = !(A.acc_valid[o] > A.threshold);
        if (A.mask) A.mask[o] = masked ? 255 : 0;
        if (A.masked_y) {
            const uint64_t c = tab.b.codes[o];
            const uint32_t yy = masked ? grey : (uint32_t)(c & 0xffff);
            su += masked ? grey : (uint32_t)((c >> 16) & 0xffff);
            sv += masked ? grey : (uint32_t)((c >> 32) & 0xffff);
            A.masked_y[o] = (uint16_t)yy;
        }
        if (A.depth || A.masked_depth) {
            const float dep = A.acc_depth[o];
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
    launch_dependent(aux_kernel<Tabs>, dim3((sh.max_wo / 2 + 127) / 128, sh.max_ho / 2, sh.slots), dim3(128), 0, s, tabs);
}

template void launch_aux<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template void launch_aux<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

}  // namespace rvsb
