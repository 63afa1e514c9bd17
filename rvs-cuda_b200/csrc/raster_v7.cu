// Raster variant 7: 64x32 tiles, 2 views per z-buffer group,
// medium triangles (5 to 32 candidate pixels) flattened across the warp,
// larger ones warp-cooperative, 1024 bin entries per round, 512-thread
// CTAs (two per SM).
#include "raster.cuh"

RVSB_RASTER_VARIANT(7, 64, 32, 2, 4, 1024, 32, 512)
