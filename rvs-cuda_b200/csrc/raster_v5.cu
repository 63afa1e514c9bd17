// Raster variant 5: 32x16 tiles, 4 views per z-buffer group,
// warp-cooperative above 4 candidate pixels, 512 bin entries per round.
#include "raster.cuh"

RVSB_RASTER_VARIANT(5, 32, 16, 4, 4, 512, 0)
