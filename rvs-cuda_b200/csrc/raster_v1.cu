// Raster variant 1: 64x32 tiles, 2 views per z-buffer group,
// warp-cooperative above 4 candidate pixels, 1024 bin entries per round,
// 512-thread CTAs (two per SM).
#include "raster.cuh"

RVSB_RASTER_VARIANT(1, 64, 32, 2, 4, 1024, 0, 512)
