// Binning of input blocks into output tiles: count per (tile, view) (done
// by the warp kernel as it writes each block's box), exclusive scan, fill.  Bin order does not affect the result (the raster's
// 64-bit atomicMin keys are order independent).
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

// Exclusive scan of one slot's bin counts (one CTA of 1024 threads per
// slot), and the raster's launch order of the tiles: those with clearly
// more bin entries than the average (over all views; mostly tiles crossed
// by stretched triangles) first, then the others, each part in raster order
// so that neighbouring tiles, which share input blocks, still run together.
// Tiles are independent, so the order changes only the schedule.  Each
// thread takes a run of whole tiles (all views of each), so one pass over
// the counts yields both its entry sum and its heavy-tile count, and one
// 64-bit scan (entries << 32 | heavy tiles) gives both prefixes.
template <class Tabs>
__global__ void __launch_bounds__(1024) bin_scan_kernel(const __grid_constant__ Tabs tabs) {
    dev::grid_dep_wait();
    __shared__ unsigned long long warp_sums[32];
    const SlotTable& tab = tabs.at(blockIdx.x);
    const int* counts = tab.b.counts;
    int* offsets = tab.b.offsets;
    int* cursor = tab.b.cursor;
    const int nv = tab.t.n_views, ntiles = tab.t.ntx * tab.t.nty;
    const long long total = tab.b.status->bin_total;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tper = (ntiles + 1023) / 1024;
    const int tb = min(ntiles, tid * tper), te = min(ntiles, tb + tper);
    auto heavy = [&](long long e) { return 2 * e * ntiles > 3 * total; };  // more than 1.5x the mean
    unsigned long long local = 0;
    for (int t = tb; t < te; ++t) {
        long long e = 0;
        for (int v = 0; v < nv; ++v) e += counts[t * nv + v];
        local += ((unsigned long long)e << 32) | (heavy(e) ? 1u : 0u);
    }
    unsigned long long x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long s = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    const unsigned long long before = x - local + (warp > 0 ? warp_sums[warp - 1] : 0ull);
    const int nheavy = (int)(warp_sums[31] & 0xffffffffu);
    int run = (int)(before >> 32);
    const int hbefore = (int)(before & 0xffffffffu);
    int ph = hbefore, pl = nheavy + (tb - hbefore);
    for (int t = tb; t < te; ++t) {
        long long e = 0;
        for (int v = 0; v < nv; ++v) {
            const int c = counts[t * nv + v];
            offsets[t * nv + v] = run;
            cursor[t * nv + v] = run;
            run += c;
            e += c;
        }
        if (heavy(e))
            tab.b.tile_order[ph++] = t;
        else
            tab.b.tile_order[pl++] = t;
    }
    if (tid == 0 && total > tab.b.capacity) tab.b.status->bin_overflow = 1;
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
    const int entry = ((b / V.nbx) << 11) | (b % V.nbx);  // block row << 11 | block column
    // Neighbouring blocks (the lanes of a warp) mostly fall in the same
    // single tile: those lanes take their places with one atomic per tile.
    const bool single = tx0 == tx1 && ty0 == ty1;
    const unsigned active = __activemask();
    const int cell = single ? (ty0 * ntx + tx0) * n + v : -1 - (int)(threadIdx.x & 31);
    const unsigned same = __match_any_sync(active, cell);
    if (single) {
        const int lane = threadIdx.x & 31, leader = __ffs(same) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&cursor[cell], __popc(same));
        base = __shfl_sync(same, base, leader);
        list[base + __popc(same & ((1u << lane) - 1u))] = entry;
        return;
    }
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) list[atomicAdd(&cursor[(ty * ntx + tx) * n + v], 1)] = entry;
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
