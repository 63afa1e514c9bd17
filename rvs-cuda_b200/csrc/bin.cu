// Binning of input blocks into output tiles: count per (tile, view) (done
// by the warp kernel as it writes each block's box), exclusive scan, fill.  Bin order does not affect the result (the raster's
// 64-bit atomicMin keys are order independent).
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

// Exclusive scan of one slot's bin counts (one CTA of 1024 threads per slot).
template <class Tabs>
__global__ void __launch_bounds__(1024) bin_scan_kernel(const __grid_constant__ Tabs tabs) {
    dev::grid_dep_wait();
    __shared__ int warp_sums[32];
    const SlotTable& tab = tabs.at(blockIdx.x);
    const int* counts = tab.b.counts;
    int* offsets = tab.b.offsets;
    int* cursor = tab.b.cursor;
    const int n = tab.t.ntx * tab.t.nty * tab.t.n_views;
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
    if (tid == 0 && tab.b.status->bin_total > tab.b.capacity) tab.b.status->bin_overflow = 1;

    // Raster launch order: the tiles with clearly more bin entries than the
    // average (over all views; mostly tiles crossed by stretched triangles)
    // first, then the others, each part in raster order so that
    // neighbouring tiles, which share input blocks, still run together.
    // Tiles are independent, so the order changes only the schedule.
    __syncthreads();
    const int nv = tab.t.n_views, ntiles = tab.t.ntx * tab.t.nty;
    const long long total = tab.b.status->bin_total;
    const int tper = (ntiles + 1023) / 1024;
    const int tb = min(ntiles, tid * tper), te = min(ntiles, tb + tper);
    auto heavy = [&](int t) {
        long long e = 0;
        for (int v = 0; v < nv; ++v) e += counts[t * nv + v];
        return 2 * e * ntiles > 3 * total;  // more than 1.5x the mean
    };
    int nh = 0;
    for (int t = tb; t < te; ++t) nh += heavy(t) ? 1 : 0;
    int hx = nh;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y2 = __shfl_up_sync(0xffffffffu, hx, o);
        if (lane >= o) hx += y2;
    }
    __syncthreads();
    if (lane == 31) warp_sums[warp] = hx;
    __syncthreads();
    if (warp == 0) {
        int s2 = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y2 = __shfl_up_sync(0xffffffffu, s2, o);
            if (lane >= o) s2 += y2;
        }
        warp_sums[lane] = s2;
    }
    __syncthreads();
    const int hbefore = hx - nh + (warp > 0 ? warp_sums[warp - 1] : 0);
    const int nheavy = warp_sums[31];
    int ph = hbefore, pl = nheavy + (tb - hbefore);
    for (int t = tb; t < te; ++t) {
        if (heavy(t))
            tab.b.tile_order[ph++] = t;
        else
            tab.b.tile_order[pl++] = t;
    }
}

// Grid (ceil(max_blocks / 256), max_views, slots): one thread per binning
// block of view blockIdx.y of slot blockIdx.z.
template <class Tabs>
__global__ void bin_fill_kernel(const __grid_constant__ Tabs tabs) {
    dev::grid_dep_wait();
    const SlotTable& tab = tabs.at(blockIdx.z);
    const int v = blockIdx.y;
    if (v >= tab.t.n_views || tab.b.status->bin_overflow) return;
    const DevView& V = tab.v[v];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= V.nbx * V.nby) return;
    const int4 bb = V.bbox[b];
    if (bb.x > bb.z || bb.y > bb.w) return;
    const int ntx = tab.t.ntx, n = tab.t.n_views;
    const int wl = tab.t.tile_wl, hl = tab.t.tile_hl;
    const int tx0 = bb.x >> wl, tx1 = bb.z >> wl, ty0 = bb.y >> hl, ty1 = bb.w >> hl;
    int* cursor = tab.b.cursor;
    int* list = tab.b.list;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const int pos = atomicAdd(&cursor[(ty * ntx + tx) * n + v], 1);
            list[pos] = ((b / V.nbx) << 11) | (b % V.nbx);  // block row << 11 | block column
        }
}

}  // namespace

template <class Tabs>
void launch_bin(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    dim3 grid((sh.max_blocks + 255) / 256, sh.max_views, sh.slots);
    launch_dependent(bin_scan_kernel<Tabs>, dim3(sh.slots), dim3(1024), 0, s, tabs);
    launch_dependent(bin_fill_kernel<Tabs>, grid, dim3(256), 0, s, tabs);
}

template void launch_bin<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template void launch_bin<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

}  // namespace rvsb
