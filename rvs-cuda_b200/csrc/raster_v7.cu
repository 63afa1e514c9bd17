// Raster variant 7: 64x32 tiles, 2 views per z-buffer group,
// warp-cooperative above 4 candidate pixels with triangles of up to 32
// candidates flattened across the warp together, 1024 bin entries per round.
#include "raster.cuh"

RVSB_RASTER_VARIANT(7, 64, 32, 2, 4, 1024, 32)
