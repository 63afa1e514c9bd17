// Orchestration of one synthesis on a stream.
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {

void launch_warp(const ViewTable& tab, const LaunchShape& sh, cudaStream_t s);
void launch_bin(const SynthBuffers& b, const ViewTable& tab, const LaunchShape& sh, cudaStream_t s);
void launch_raster(const SynthBuffers& b, const ViewTable& tab, const LaunchShape& sh, const DebugPtrs& dbg,
                   uint16_t* out_y, uint16_t* out_u, uint16_t* out_v, cudaStream_t s);
void launch_inpaint(const SynthBuffers& b, const LaunchShape& sh, const DebugPtrs& dbg, uint16_t* out_y,
                    uint16_t* out_u, uint16_t* out_v, cudaStream_t s);

namespace {

__global__ void status_init_kernel(DevStatus* st) {
    st->bin_total = 0;
    st->bin_overflow = 0;
    st->hole_x0 = INT_MAX;
    st->hole_y0 = INT_MAX;
    st->hole_x1 = INT_MIN;
    st->hole_y1 = INT_MIN;
    st->n_holes = 0;
}

}  // namespace

int launch_synthesis(const SynthBuffers& b, const ViewTable& tab, const LaunchShape& sh, const DebugPtrs& dbg,
                     uint16_t* out_y,
                     uint16_t* out_u, uint16_t* out_v, cudaStream_t s, cudaEvent_t* ev) {
    auto mark = [&](int k) {
        if (ev) cudaEventRecord(ev[k], s);
    };
    mark(8);
    status_init_kernel<<<1, 1, 0, s>>>(b.status);
    mark(0);
    launch_warp(tab, sh, s);
    mark(1);
    mark(2);
    launch_bin(b, tab, sh, s);
    mark(3);
    mark(4);
    launch_raster(b, tab, sh, dbg, out_y, out_u, out_v, s);
    mark(5);
    mark(6);
    launch_inpaint(b, sh, dbg, out_y, out_u, out_v, s);
    mark(7);
    mark(9);
    if (cudaPeekAtLastError() != cudaSuccess) return -1;
    return 1 + 1 + 3 + 1 + 6;
}

}  // namespace rvsb
