// Raster variant 2: 32x32 tiles, 4 views per z-buffer group,
// warp-cooperative above 2 candidate pixels, 1024 bin entries per round.
#include "raster.cuh"

RVSB_RASTER_VARIANT(2, 32, 32, 4, 2, 1024, 0)
