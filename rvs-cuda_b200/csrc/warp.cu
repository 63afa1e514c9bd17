// Warp stage: decode depth, unproject, R*x+t, project every input pixel, and
// the pixel bounding box of each binning block (BLOCK_W x BLOCK_H quads).
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

constexpr int VT_W = 4 * BLOCK_W;  // vertex tile: 32 x 8 vertices per CTA
constexpr int VT_H = 2 * BLOCK_H;
static_assert(VT_W * VT_H == 256, "one vertex per thread");

// A vertex can be part of a rasterised triangle only if it passes the
// emission tests of transform.cpp:161-167 (depth > 0, u > 0) and has finite
// coordinates (a triangle with a non-finite coordinate covers no pixel).
// Seam triangles (horizontal wrap) skip the emission tests.
__device__ __forceinline__ bool bbox_vertex_ok(float4 p, bool wrap) {
    if (!(isfinite(p.x) && isfinite(p.y))) return false;
    return wrap || (p.z > 0.f && p.x > 0.f);
}

__device__ int4 to_pixel_box(float x0, float y0, float x1, float y1, int wo, int ho) {
    if (!(x0 <= x1) || !(y0 <= y1)) return make_int4(1, 1, 0, 0);
    const float fx0 = floorf(x0), fy0 = floorf(y0);
    const float fx1 = ceilf(x1), fy1 = ceilf(y1);
    if (fx0 > (float)(wo - 1) || fy0 > (float)(ho - 1) || fx1 < 0.f || fy1 < 0.f) return make_int4(1, 1, 0, 0);
    int4 r;
    r.x = fx0 < 0.f ? 0 : (int)fx0;
    r.y = fy0 < 0.f ? 0 : (int)fy0;
    r.z = fx1 > (float)(wo - 1) ? wo - 1 : (int)fx1;
    r.w = fy1 > (float)(ho - 1) ? ho - 1 : (int)fy1;
    return r;
}

// Grid (ceil(W/32), ceil(H/8), n_views), 256 threads.  Round 1: one vertex
// per thread, written to the vertex buffer and to shared memory.  Round 2:
// the extra column and row the tile's blocks need (and, for a horizontal
// wrap, column W-1) are computed by the first warps, not written.  Then
// one warp per binning block reduces its (BLOCK_W+1) x (BLOCK_H+1) vertices.
__global__ void __launch_bounds__(256) warp_kernel(const __grid_constant__ ViewTable tab) {
    __shared__ float4 sv[VT_H + 1][VT_W + 1];
    __shared__ float4 sw[VT_H + 1];  // column W-1 (wrap seams)
    const DevView& V = tab.v[blockIdx.z];
    const DevTarget& T = tab.t;
    const int j0 = blockIdx.x * VT_W, i0 = blockIdx.y * VT_H;
    if (j0 >= V.w || i0 >= V.h) return;
    const int tid = threadIdx.x;
    const bool wrap = T.wrap != 0;
    const float4 none = make_float4(qnan(), qnan(), qnan(), 0.f);
    {
        const int tx = tid % VT_W, ty = tid / VT_W;
        const int i = i0 + ty, j = j0 + tx;
        float4 p = none;
        if (i < V.h && j < V.w) {
            p = warp_vertex(V, T, i, j);
            V.vert[(size_t)i * V.w + j] = p;
        }
        sv[ty][tx] = p;
    }
    // Round 2: row VT_H (VT_W + 1 vertices), column VT_W (VT_H vertices),
    // column W-1 (VT_H + 1 vertices, wrap only).
    const int n_extra = (VT_W + 1) + VT_H + ((wrap && blockIdx.x == 0) ? VT_H + 1 : 0);
    if (tid < n_extra) {
        int i, j, ty, tx;
        bool seam = false;
        if (tid <= VT_W) {
            ty = VT_H; tx = tid;
        } else if (tid < VT_W + 1 + VT_H) {
            ty = tid - (VT_W + 1); tx = VT_W;
        } else {
            ty = tid - (VT_W + 1 + VT_H); tx = 0; seam = true;
        }
        i = i0 + ty;
        j = seam ? V.w - 1 : j0 + tx;
        float4 p = none;
        if (i < V.h && j < V.w) p = warp_vertex(V, T, i, j);
        if (seam)
            sw[ty] = p;
        else
            sv[ty][tx] = p;
    }
    __syncthreads();
    // One warp per binning block of the tile (4 x 2 blocks).
    const int warp = tid >> 5, lane = tid & 31;
    const int lbx = warp & 3, lby = warp >> 2;
    const int bx = blockIdx.x * 4 + lbx, by = blockIdx.y * 2 + lby;
    if (bx >= V.nbx || by >= V.nby) return;
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    constexpr int NV = (BLOCK_W + 1) * (BLOCK_H + 1);
    for (int k = lane; k < NV; k += 32) {
        const int r = lby * BLOCK_H + k / (BLOCK_W + 1), c = lbx * BLOCK_W + k % (BLOCK_W + 1);
        const float4 p = sv[r][c];
        if (bbox_vertex_ok(p, wrap)) {
            x0 = fminf(x0, p.x); y0 = fminf(y0, p.y);
            x1 = fmaxf(x1, p.x); y1 = fmaxf(y1, p.y);
        }
    }
    if (wrap && bx == 0 && lane <= BLOCK_H) {
        const float4 p = sw[lby * BLOCK_H + lane];
        if (bbox_vertex_ok(p, wrap)) {
            x0 = fminf(x0, p.x); y0 = fminf(y0, p.y);
            x1 = fmaxf(x1, p.x); y1 = fmaxf(y1, p.y);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane == 0) V.bbox[by * V.nbx + bx] = to_pixel_box(x0, y0, x1, y1, T.wo, T.ho);
}

}  // namespace

void launch_warp(const ViewTable& tab, const LaunchShape& sh, cudaStream_t s) {
    dim3 grid((sh.max_w + VT_W - 1) / VT_W, (sh.max_h + VT_H - 1) / VT_H, sh.n_views);
    warp_kernel<<<grid, 256, 0, s>>>(tab);
}

}  // namespace rvsb
