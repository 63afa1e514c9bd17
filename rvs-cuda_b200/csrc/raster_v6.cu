// Raster variant 6: 32x32 tiles, 4 views per z-buffer group,
// warp-cooperative above 2 candidate pixels with triangles of up to 32
// candidates flattened across the warp together, 1024 bin entries per round.
#include "raster.cuh"

RVSB_RASTER_VARIANT(6, 32, 32, 4, 2, 1024, 32)
