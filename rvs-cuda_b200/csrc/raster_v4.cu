// Raster variant 4: 32x32 tiles, 2 views per z-buffer group,
// warp-cooperative above 4 candidate pixels, 512 bin entries per round.
#include "raster.cuh"

RVSB_RASTER_VARIANT(4, 32, 32, 2, 4, 512, 0)
