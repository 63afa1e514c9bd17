// Raster variant 0: 32x32 tiles, 4 views per z-buffer group,
// warp-cooperative above 4 candidate pixels, 1024 bin entries per round,
// 512-thread CTAs (two per SM).
#include "raster.cuh"

RVSB_RASTER_VARIANT(0, 32, 32, 4, 4, 1024, 0, 512)
