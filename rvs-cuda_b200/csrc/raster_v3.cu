// Raster variant 3: 32x32 tiles, 4 views per z-buffer group,
// warp-cooperative above 8 candidate pixels, 1024 bin entries per round,
// 512-thread CTAs (two per SM).
#include "raster.cuh"

RVSB_RASTER_VARIANT(3, 32, 32, 4, 8, 1024, 0, 512)
