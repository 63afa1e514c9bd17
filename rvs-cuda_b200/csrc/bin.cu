// Binning of input blocks into output tiles: count per (tile, view),
// exclusive scan, fill.  Bin order does not affect the result (the raster's
// 64-bit atomicMin keys are order independent).
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

__global__ void bin_count_kernel(const __grid_constant__ ViewTable tab, int* __restrict__ counts,
                                 DevStatus* __restrict__ st) {
    const int v = blockIdx.y;
    const DevView& V = tab.v[v];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= V.nbx * V.nby) return;
    const int4 bb = V.bbox[b];
    if (bb.x > bb.z || bb.y > bb.w) return;
    const int ntx = tab.t.ntx, n = tab.t.n_views;
    const int tx0 = bb.x / TILE, tx1 = bb.z / TILE, ty0 = bb.y / TILE, ty1 = bb.w / TILE;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) atomicAdd(&counts[(ty * ntx + tx) * n + v], 1);
    atomicAdd(&st->bin_total, (tx1 - tx0 + 1) * (ty1 - ty0 + 1));
}

// Exclusive scan of the bin counts (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) bin_scan_kernel(const int* __restrict__ counts, int* __restrict__ offsets,
                                                        int* __restrict__ cursor, int n, int capacity,
                                                        DevStatus* __restrict__ st) {
    __shared__ int warp_sums[32];
    const int tid = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int beg = min(n, tid * per), end = min(n, beg + per);
    int local = 0;
    for (int k = beg; k < end; ++k) local += counts[k];
    int x = local;
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    int run = x - local + (warp > 0 ? warp_sums[warp - 1] : 0);
    for (int k = beg; k < end; ++k) {
        offsets[k] = run;
        cursor[k] = run;
        run += counts[k];
    }
    if (tid == 0 && st->bin_total > capacity) st->bin_overflow = 1;
}

__global__ void bin_fill_kernel(const __grid_constant__ ViewTable tab, int* __restrict__ cursor,
                                int* __restrict__ list, const DevStatus* __restrict__ st) {
    if (st->bin_overflow) return;
    const int v = blockIdx.y;
    const DevView& V = tab.v[v];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= V.nbx * V.nby) return;
    const int4 bb = V.bbox[b];
    if (bb.x > bb.z || bb.y > bb.w) return;
    const int ntx = tab.t.ntx, n = tab.t.n_views;
    const int tx0 = bb.x / TILE, tx1 = bb.z / TILE, ty0 = bb.y / TILE, ty1 = bb.w / TILE;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const int pos = atomicAdd(&cursor[(ty * ntx + tx) * n + v], 1);
            list[pos] = ((b / V.nbx) << 11) | (b % V.nbx);  // block row << 11 | block column
        }
}

}  // namespace

void launch_bin(const SynthBuffers& b, const ViewTable& tab, const LaunchShape& sh, cudaStream_t s) {
    const int ntiles = sh.ntx * sh.nty;
    cudaMemsetAsync(b.counts, 0, sizeof(int) * (size_t)ntiles * sh.n_views, s);
    dim3 grid((sh.max_blocks + 255) / 256, sh.n_views);
    bin_count_kernel<<<grid, 256, 0, s>>>(tab, b.counts, b.status);
    bin_scan_kernel<<<1, 1024, 0, s>>>(b.counts, b.offsets, b.cursor, ntiles * sh.n_views, b.capacity, b.status);
    bin_fill_kernel<<<grid, 256, 0, s>>>(tab, b.cursor, b.list, b.status);
}

}  // namespace rvsb
