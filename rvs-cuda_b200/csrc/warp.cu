// Warp stage: decode depth, unproject, R*x+t, project every input pixel, and
// the pixel bounding box of each binning block (BLOCK_W x BLOCK_H quads).
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

constexpr int VT = WARP_TILE;      // vertex tile: 32 x 32 vertices per CTA
constexpr int ROWS = VT / 8;       // vertex rows per thread (8 warps)
static_assert(ROWS == BLOCK_H && VT == 4 * BLOCK_W, "a warp covers one row of 4 binning blocks");

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

// Bounding-box contribution of one vertex: (x, y) when it can belong to a
// rasterised triangle, else NaN (which fminf / fmaxf skip).
__device__ __forceinline__ float2 box_point(float4 p, bool wrap) {
    return bbox_vertex_ok(p, wrap) ? make_float2(p.x, p.y) : make_float2(qnan(), qnan());
}

struct Box {
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    __device__ void add(float2 q) {
        x0 = fminf(x0, q.x); y0 = fminf(y0, q.y);
        x1 = fmaxf(x1, q.x); y1 = fmaxf(y1, q.y);
    }
    __device__ void add(const Box& b) {
        x0 = fminf(x0, b.x0); y0 = fminf(y0, b.y0);
        x1 = fmaxf(x1, b.x1); y1 = fmaxf(y1, b.y1);
    }
    __device__ Box shfl_xor(int o) const {
        Box b;
        b.x0 = __shfl_xor_sync(0xffffffffu, x0, o); b.y0 = __shfl_xor_sync(0xffffffffu, y0, o);
        b.x1 = __shfl_xor_sync(0xffffffffu, x1, o); b.y1 = __shfl_xor_sync(0xffffffffu, y1, o);
        return b;
    }
    __device__ Box shfl_down(int o) const {
        Box b;
        b.x0 = __shfl_down_sync(0xffffffffu, x0, o); b.y0 = __shfl_down_sync(0xffffffffu, y0, o);
        b.x1 = __shfl_down_sync(0xffffffffu, x1, o); b.y1 = __shfl_down_sync(0xffffffffu, y1, o);
        return b;
    }
};

// Grid (ceil(W/32), ceil(H/32), slots * max_views), 256 threads.  Thread (lane, warp)
// warps the vertices of column j0 + lane, rows i0 + 4*warp .. +3, writes
// them and keeps the bounding box of its column.  The row below the tile,
// the column right of it and, for a horizontal wrap, column W-1 are warped
// as well (not written) and exchanged through shared memory.  Warp `warp`
// then reduces the boxes of binning-block row by = 8*blockIdx.y + warp: the
// (BLOCK_W + 1) x (BLOCK_H + 1) vertices of block bx are the columns of
// lanes 8*b .. 8*b + 8, rows 4*warp .. 4*warp + 4.
// Whether vertex tile (blockIdx.x, blockIdx.y) of an ERP input view lies, with
// its one-pixel ring, wholly beyond one of the output's side planes.  A
// vertex is x = z * d (d within the tile's cone, z within its depth range),
// seen by the virtual camera as y = R x + t; beyond plane a when a . y > 0,
// i.e. z * (b . d) + c > 0 with b = R^T a, c = a . t.  Over the cone
// b . d >= b . dc - |b| rho; the smallest value over z is at the near or far
// end of the range.  A relative margin absorbs the float rounding of the
// vertices, and the planes sit one pixel outside the image.
template <class View, class Target>
__device__ __forceinline__ bool tile_culled(const View& V, const Target& T) {
    const int ntx = (V.w + VT - 1) / VT;
    const size_t k = (size_t)blockIdx.y * ntx + blockIdx.x;
    const float4 cone = V.erp_cone[k];
    const float2 zr = V.tile_depth[k];
    if (!(zr.x > 0.f && zr.x <= zr.y)) return false;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const float* a = T.cull_plane[p];
        float b[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) b[j] = a[0] * V.R[j] + a[1] * V.R[3 + j] + a[2] * V.R[6 + j];
        const float c = a[0] * V.t[0] + a[1] * V.t[1] + a[2] * V.t[2];
        const float nb = sqrtf(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        const float m = b[0] * cone.x + b[1] * cone.y + b[2] * cone.z - nb * cone.w;
        const float z = m >= 0.f ? zr.x : zr.y;
        const float L = z * m + c;
        if (L > 1e-3f * (fabsf(c) + z * nb) && isfinite(L)) return true;
    }
    return false;
}

template <class Tabs>
__global__ void __launch_bounds__(256) warp_kernel(const __grid_constant__ Tabs tabs, int max_views) {
    grid_dep_wait();
    __shared__ float2 s_top[8][VT];        // first row of each warp (row 4*w)
    __shared__ float2 s_row[VT + 1];       // row i0 + 32, columns j0 .. j0 + 32
    __shared__ float2 s_col[VT + 1];       // column j0 + 32, rows i0 .. i0 + 32
    __shared__ float2 s_seam[VT + 1];      // column W - 1, rows i0 .. i0 + 32 (wrap)
    const SlotTable& tab = tabs.at(blockIdx.z / max_views);
    const int view = blockIdx.z % max_views;
    const DevTarget& T = tab.t;
    if (view >= T.n_views) return;
    // The view's fields used per vertex, in registers: tab.v[view] is
    // indexed by the grid, so each use would otherwise be a load.
    struct RegView {
        int w, h, proj, nbx, nby;
        float f0, f1, p0, p1;
        float R[9], t[3];
        const uint16_t* pd;
        const float4* depth_lut;
        const float* erp_row;
        const float* erp_col;
        float4* vert;
        int4* bbox;
        const float4* erp_cone;
        const float2* tile_depth;
    } V;
    {
        const DevView& G = tab.v[view];
        V.w = G.w; V.h = G.h; V.proj = G.proj; V.nbx = G.nbx; V.nby = G.nby;
        V.f0 = G.f0; V.f1 = G.f1; V.p0 = G.p0; V.p1 = G.p1;
#pragma unroll
        for (int k = 0; k < 9; ++k) V.R[k] = G.R[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) V.t[k] = G.t[k];
        V.pd = G.pd; V.depth_lut = G.depth_lut; V.erp_row = G.erp_row; V.erp_col = G.erp_col;
        V.vert = G.vert; V.bbox = G.bbox;
        V.erp_cone = G.erp_cone; V.tile_depth = G.tile_depth;
    }
    const int j0 = blockIdx.x * VT, i0 = blockIdx.y * VT;
    if (j0 >= V.w || i0 >= V.h) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (T.cull && V.erp_cone && tile_culled(V, T)) {
        // No triangle with a vertex of this tile can cover an output pixel:
        // every vertex of the tile and of the pixel ring around it lies
        // beyond one side of the output (or behind the camera).  Its
        // vertices are stored as NaN, which no triangle is emitted from, and
        // its blocks get empty boxes.
        const float nan = qnan();
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            const int i = i0 + warp * ROWS + r, j = j0 + lane;
            if (i < V.h && j < V.w) V.vert[(size_t)i * V.w + j] = make_float4(nan, nan, nan, 0.f);
        }
        const int bx = blockIdx.x * 4 + (lane >> 3), by = blockIdx.y * 8 + warp;
        if ((lane & 7) == 0 && bx < V.nbx && by < V.nby) V.bbox[by * V.nbx + bx] = make_int4(1, 1, 0, 0);
        return;
    }
    const bool wrap = T.wrap != 0;
    const bool seam = wrap && blockIdx.x == 0;
    const int j = j0 + lane;
    // The thread's depth samples, then their table entries, before any
    // arithmetic: the dependent gathers of the four rows overlap instead of
    // each waiting behind the previous row's vertex store.
    float4 L[ROWS];
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const int i = i0 + warp * ROWS + r;
        if (i < V.h && j < V.w) L[r] = depth_entry(V, i, j);
    }
    Box col;
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const int i = i0 + warp * ROWS + r;
        float2 q = make_float2(qnan(), qnan());
        if (i < V.h && j < V.w) {
            const float4 p = warp_vertex(V, T, i, j, L[r]);
            V.vert[(size_t)i * V.w + j] = p;
            q = box_point(p, wrap);
        }
        col.add(q);
        if (r == 0) s_top[warp][lane] = q;
    }
    // Extra vertices: warps 0-1 the row below (33), warp 2 the column to the
    // right (32; its row-32 vertex is the row's last), warps 3-4 the seam.
    {
        int i = -1, jj = -1, slot = -1;
        if (tid <= VT) {
            i = i0 + VT; jj = j0 + tid; slot = 0;
        } else if (tid >= 64 && tid < 64 + VT) {
            i = i0 + (tid - 64); jj = j0 + VT; slot = 1;
        } else if (seam && tid >= 96 && tid <= 96 + VT) {
            i = i0 + (tid - 96); jj = V.w - 1; slot = 2;
        }
        if (slot >= 0) {
            float2 q = make_float2(qnan(), qnan());
            if (i < V.h && jj < V.w) q = box_point(warp_vertex(V, T, i, jj), wrap);
            if (slot == 0) {
                s_row[tid] = q;
                if (tid == VT) s_col[VT] = q;
            } else if (slot == 1) {
                s_col[tid - 64] = q;
            } else {
                s_seam[tid - 96] = q;
            }
        }
    }
    __syncthreads();
    // Row 4*warp + 4 of this column closes the column's box.
    col.add(warp < 7 ? s_top[warp + 1][lane] : s_row[lane]);
    // Column 8*b + 8 of each block: the next group's first lane, or the
    // column right of the tile for the last group.
    Box right;
    {
        const Box nb = col.shfl_down(8);
        if (lane < 24) {
            right = nb;
        } else {
#pragma unroll
            for (int r = 0; r <= ROWS; ++r) right.add(s_col[warp * ROWS + r]);
        }
    }
    Box blk = col;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) blk.add(blk.shfl_xor(o));
    const int b = lane >> 3;
    const int bx = blockIdx.x * 4 + b, by = blockIdx.y * 8 + warp;
    int entries = 0;
    if ((lane & 7) == 0 && bx < V.nbx && by < V.nby) {
        Box out = blk;
        out.add(right);
        if (seam && b == 0) {
#pragma unroll
            for (int r = 0; r <= ROWS; ++r) out.add(s_seam[warp * ROWS + r]);
        }
        const int4 bb = to_pixel_box(out.x0, out.y0, out.x1, out.y1, T.wo, T.ho);
        V.bbox[by * V.nbx + bx] = bb;
        // Binning, first pass: one entry per output tile the box touches,
        // counted per (tile, view).
        if (bb.x <= bb.z && bb.y <= bb.w) {
            const int wl = T.tile_wl, hl = T.tile_hl, n = T.n_views, ntx = T.ntx;
            const int tx0 = bb.x >> wl, tx1 = bb.z >> wl, ty0 = bb.y >> hl, ty1 = bb.w >> hl;
            for (int ty = ty0; ty <= ty1; ++ty)
                for (int tx = tx0; tx <= tx1; ++tx) atomicAdd(&tab.b.counts[(ty * ntx + tx) * n + view], 1);
            entries = (tx1 - tx0 + 1) * (ty1 - ty0 + 1);
        }
    }
    entries = __reduce_add_sync(0xffffffffu, entries);
    if (lane == 0 && entries > 0) atomicAdd(&tab.b.status->bin_total, entries);
}

// Range of the decoded depths of one vertex tile grown by one pixel (NaN
// samples ignored).  Grid (tiles x, tiles y, views), 256 threads.
__global__ void tile_depth_kernel(const __grid_constant__ TileDepthJobs jobs) {
    const TileDepthJob& J = jobs.v[blockIdx.z];
    const int ntx = (J.w + WARP_TILE - 1) / WARP_TILE, nty = (J.h + WARP_TILE - 1) / WARP_TILE;
    if ((int)blockIdx.x >= ntx || (int)blockIdx.y >= nty) return;
    const int r0 = max(0, (int)blockIdx.y * WARP_TILE - 1), r1 = min(J.h - 1, (int)blockIdx.y * WARP_TILE + WARP_TILE);
    const int c0 = max(0, (int)blockIdx.x * WARP_TILE - 1), c1 = min(J.w - 1, (int)blockIdx.x * WARP_TILE + WARP_TILE);
    const int cols = c1 - c0 + 1, n = (r1 - r0 + 1) * cols;
    float mn = INFINITY, mx = -INFINITY;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int i = r0 + k / cols, j = c0 + k % cols;
        const float z = __ldg(&J.lut[__ldg(J.depth + (size_t)i * J.w + j)].x);
        mn = fminf(mn, z);
        mx = fmaxf(mx, z);
    }
    __shared__ float s_mn[8], s_mx[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_mn[warp] = mn;
        s_mx[warp] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            mn = fminf(mn, s_mn[k]);
            mx = fmaxf(mx, s_mx[k]);
        }
        J.out[blockIdx.y * ntx + blockIdx.x] = make_float2(mn, mx);
    }
}

// Decoded depth d of every possible 16-bit sample of one view, with the
// two per-sample factors of the perspective unprojection, -(d / f0) and
// -(d / f1) (PerspectiveUnprojector.cpp:75-77), so that the warp reads them
// instead of dividing per pixel.
__global__ void depth_lut_kernel(float near_, float far_, float depth_scale, int has_invalid, float f0, float f1,
                                 float4* out) {
    const uint32_t raw = blockIdx.x * blockDim.x + threadIdx.x;
    if (raw >= 65536u) return;
    const float d = decode_depth_raw(near_, far_, depth_scale, has_invalid, raw);
    out[raw] = make_float4(d, -__fdiv_rn(d, f0), -__fdiv_rn(d, f1), 0.f);
}

}  // namespace

void launch_tile_depth(const TileDepthJobs& jobs, int n, int max_w, int max_h, cudaStream_t s) {
    tile_depth_kernel<<<dim3((max_w + WARP_TILE - 1) / WARP_TILE, (max_h + WARP_TILE - 1) / WARP_TILE, n), 256, 0, s>>>(
        jobs);
}

void launch_depth_lut(float near_, float far_, float depth_scale, int has_invalid, float f0, float f1, float4* out,
                      cudaStream_t s) {
    depth_lut_kernel<<<256, 256, 0, s>>>(near_, far_, depth_scale, has_invalid, f0, f1, out);
}

template <class Tabs>
void launch_warp(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    dim3 grid((sh.max_w + VT - 1) / VT, (sh.max_h + VT - 1) / VT, sh.slots * sh.max_views);
    launch_dependent(warp_kernel<Tabs>, grid, dim3(256), 0, s, tabs, sh.max_views);
}

template void launch_warp<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template void launch_warp<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

}  // namespace rvsb
