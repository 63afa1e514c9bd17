// Raster variant 6: 32x32 tiles, 4 views per z-buffer group,
// medium triangles (3 to 32 candidate pixels) flattened across the warp,
// larger ones warp-cooperative, 1024 bin entries per round, 512-thread
// CTAs (two per SM).
#include "raster.cuh"

RVSB_RASTER_VARIANT(6, 32, 32, 4, 2, 1024, 32, 512)
