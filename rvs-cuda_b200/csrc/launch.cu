// Orchestration of one batch of syntheses on a stream.  Every kernel covers
// all slots of the batch in one launch (the slot is a grid dimension), so a
// batch costs the same 11 launches as a single view and the sequence can be
// captured in a CUDA graph.
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {

template <class Tabs>
void launch_warp(const Tabs& tabs, const BatchShape& sh, cudaStream_t s);
template <class Tabs>
void launch_bin(const Tabs& tabs, const BatchShape& sh, cudaStream_t s);
template <class Tabs>
void launch_raster(const Tabs& tabs, const BatchShape& sh, cudaStream_t s);
template <class Tabs>
int launch_inpaint(const Tabs& tabs, const BatchShape& sh, cudaStream_t s);
template <class Tabs>
void launch_aux(const Tabs& tabs, const BatchShape& sh, cudaStream_t s);
template <class Tabs>
int launch_ms(const Tabs& tabs, const BatchShape& sh, cudaStream_t s);

namespace {

// Per slot: the empty status and zero bin counts.  Grid (ceil(max_bins /
// 256), slots).
template <class Tabs>
__global__ void slot_init_kernel(const __grid_constant__ Tabs tabs) {
    dev::grid_dep_wait();
    const SlotTable& tab = tabs.at(blockIdx.y);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nbins = tab.t.ntx * tab.t.nty * tab.t.n_views;
    if (k < nbins) tab.b.counts[k] = 0;
    if (k == 0) {
        DevStatus* st = tab.b.status;
        st->bin_total = 0;
        st->bin_overflow = 0;
        st->hole_x0 = INT_MAX;
        st->hole_y0 = INT_MAX;
        st->hole_x1 = INT_MIN;
        st->hole_y1 = INT_MIN;
        st->n_holes = 0;
        st->pad = 0;
    }
}

}  // namespace

template <class Tabs>
int launch_batch(const Tabs& tabs, const BatchShape& sh, cudaStream_t s, cudaEvent_t* ev) {
    auto mark = [&](int k) {
        if (ev) cudaEventRecord(ev[k], s);
    };
    mark(8);
    launch_dependent(slot_init_kernel<Tabs>, dim3((sh.max_bins + 255) / 256, sh.slots), dim3(256), 0, s, tabs);
    mark(0);
    launch_warp(tabs, sh, s);
    mark(1);
    mark(2);
    launch_bin(tabs, sh, s);
    mark(3);
    mark(4);
    launch_raster(tabs, sh, s);
    const int ms_launches = sh.ms ? launch_ms(tabs, sh, s) : 0;
    mark(5);
    mark(6);
    const int inpaint_launches = launch_inpaint(tabs, sh, s);
    if (sh.aux) launch_aux(tabs, sh, s);
    if (sh.rescale) launch_resize(tabs, sh, s);
    mark(7);
    mark(9);
    if (cudaPeekAtLastError() != cudaSuccess) return -1;
    return 1 + 1 + 2 + 1 + ms_launches + inpaint_launches + (sh.aux ? 1 : 0) + (sh.rescale ? 1 : 0);
}

template int launch_batch<TableParam>(const TableParam&, const BatchShape&, cudaStream_t, cudaEvent_t*);
template int launch_batch<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t, cudaEvent_t*);

}  // namespace rvsb
