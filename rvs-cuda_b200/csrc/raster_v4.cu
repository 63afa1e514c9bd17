// Raster variant 4: 64x32 tiles, 4 views per z-buffer group (100 KB of
// shared memory), warp-cooperative above 4 candidate pixels, 1024 bin
// entries per round, 1024-thread CTAs (one per SM).
#include "raster.cuh"

RVSB_RASTER_VARIANT(4, 64, 32, 4, 4, 1024, 0, 1024)
