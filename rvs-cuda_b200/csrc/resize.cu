// Output write of a synthesis rasterised at Precision P != 1: the blended,
// inpainted colour at the raster size is resized to the virtual camera's
// size and written as 4:2:0 (write_color, image_writing.cpp:182-200: cv::resize
// with INTER_LINEAR of the float image, then quantization and the chroma
// 2x2 mean).  The filled colour of a raster pixel is its blended colour, or
// for a hole the blended colour of its inpainting source.
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

struct Filled {
    const float4* color;
    const uint8_t* holes;
    const int32_t* src;
    int w;
    __device__ __forceinline__ float3 at(int x, int y) const {
        size_t o = (size_t)y * w + x;
        if (holes[o]) o = (size_t)src[o * 2 + 1] * w + src[o * 2 + 0];
        const float4 c = color[o];
        return make_float3(c.x, c.y, c.z);
    }
};

// Resized colour of output pixel (x, y).
__device__ __forceinline__ float3 resized(const DevTarget& T, const Filled& F, int x, int y) {
    if (T.rs_area) {
        // resizeAreaFast of an exact 2x reduction: ((a + b) + c + d) / 4
        const float3 a = F.at(2 * x, 2 * y), b = F.at(2 * x + 1, 2 * y);
        const float3 c = F.at(2 * x, 2 * y + 1), d = F.at(2 * x + 1, 2 * y + 1);
        return make_float3(__fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(a.x, b.x), c.x), d.x), 0.25f),
                           __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(a.y, b.y), c.y), d.y), 0.25f),
                           __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(a.z, b.z), c.z), d.z), 0.25f));
    }
    int sx0, sx1, sy0, sy1;
    float fx, fy;
    linear_tap(x, T.rs_scale_x, T.wo, sx0, sx1, fx);
    linear_tap(y, T.rs_scale_y, T.ho, sy0, sy1, fy);
    const float a0 = __fsub_rn(1.f, fx), b0 = __fsub_rn(1.f, fy);
    // horizontal pass on the two source rows, then the vertical pass
    const float3 p00 = F.at(sx0, sy0), p01 = F.at(sx1, sy0), p10 = F.at(sx0, sy1), p11 = F.at(sx1, sy1);
    const float3 r0 = make_float3(lerp2(p00.x, p01.x, a0, fx), lerp2(p00.y, p01.y, a0, fx),
                                  lerp2(p00.z, p01.z, a0, fx));
    const float3 r1 = make_float3(lerp2(p10.x, p11.x, a0, fx), lerp2(p10.y, p11.y, a0, fx),
                                  lerp2(p10.z, p11.z, a0, fx));
    return make_float3(lerp2(r0.x, r1.x, b0, fy), lerp2(r0.y, r1.y, b0, fy), lerp2(r0.z, r1.z, b0, fy));
}

// One thread per 2x2 output block.  Grid (ceil(max_out_w / 2 / 128),
// max_out_h / 2, slots).
template <class Tabs>
__global__ void resize_write_kernel(const __grid_constant__ Tabs tabs) {
    grid_dep_wait();
    const SlotTable& tab = tabs.at(blockIdx.z);
    const DevTarget& T = tab.t;
    if (!T.rescale) return;
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y;
    const int x0 = 2 * bx, y0 = 2 * by;
    if (x0 >= T.out_w || y0 >= T.out_h) return;
    const Filled F{tab.b.pcolor, tab.b.holes, tab.b.psrc, T.wo};
    uint32_t su = 0, sv = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int x = x0 + (p & 1), y = y0 + (p >> 1);
        const float3 c = resized(T, F, x, y);
        tab.out_y[(size_t)y * T.out_w + x] = quantize(c.x, T.max_val);
        su += quantize(c.y, T.max_val);
        sv += quantize(c.z, T.max_val);
    }
    const size_t co = (size_t)by * (T.out_w / 2) + bx;
    tab.out_u[co] = quarter_round(su, T.chroma_ties_up);
    tab.out_v[co] = quarter_round(sv, T.chroma_ties_up);
}

}  // namespace

template <class Tabs>
void launch_resize(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    launch_dependent(resize_write_kernel<Tabs>, dim3((sh.max_out_w / 2 + 127) / 128, sh.max_out_h / 2, sh.slots),
                     dim3(128), 0, s, tabs);
}

template void launch_resize<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template void launch_resize<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

}  // namespace rvsb
