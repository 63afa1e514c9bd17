// Raster stage dispatch: the batch's raster variant (see raster.cuh; each
// variant is compiled in its own raster_v*.cu).
#include "kernels.hpp"

namespace rvsb {

#define RVSB_DECLARE_RASTER(N)                                                      \
    void launch_raster_v##N(const TableParam& t, const BatchShape& sh, cudaStream_t s); \
    void launch_raster_v##N(const TablePtr& t, const BatchShape& sh, cudaStream_t s);   \
    void prepare_raster_v##N();
RVSB_DECLARE_RASTER(0)
RVSB_DECLARE_RASTER(1)
RVSB_DECLARE_RASTER(2)
RVSB_DECLARE_RASTER(3)
RVSB_DECLARE_RASTER(4)
RVSB_DECLARE_RASTER(5)
RVSB_DECLARE_RASTER(6)
RVSB_DECLARE_RASTER(7)
#undef RVSB_DECLARE_RASTER
static_assert(NUM_RASTER_VARIANTS == 8, "one declaration per variant");

void prepare_kernels() {
    prepare_raster_v0();
    prepare_raster_v1();
    prepare_raster_v2();
    prepare_raster_v3();
    prepare_raster_v4();
    prepare_raster_v5();
    prepare_raster_v6();
    prepare_raster_v7();
}

template <class Tabs>
void launch_raster(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    switch (sh.variant) {
        case 1: launch_raster_v1(tabs, sh, s); break;
        case 2: launch_raster_v2(tabs, sh, s); break;
        case 3: launch_raster_v3(tabs, sh, s); break;
        case 4: launch_raster_v4(tabs, sh, s); break;
        case 5: launch_raster_v5(tabs, sh, s); break;
        case 6: launch_raster_v6(tabs, sh, s); break;
        case 7: launch_raster_v7(tabs, sh, s); break;
        default: launch_raster_v0(tabs, sh, s); break;
    }
}

template void launch_raster<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template void launch_raster<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

}  // namespace rvsb
