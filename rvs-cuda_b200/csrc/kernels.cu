// Synthesis kernels for sm_100a.
//
// One synthesis = warp -> bin -> tile (raster + resolve + blend + quantise)
// -> inpaint scans -> write of the 2x2 blocks that held holes.
//
// Exactness: every float operation whose result decides coverage (the
// warped u, v and the barycentric tests) or feeds the colour is written with
// explicit round-to-nearest intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, ...)
// in the reference's operation order, so nvcc cannot contract them into
// fused multiply-adds.  The translation unit is also built with -fmad=false.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdint>

#include "device_types.hpp"
#include "kernels.hpp"

namespace rvsb {
namespace {

constexpr uint64_t kEmptyKey = ~0ull;
constexpr uint64_t kHoleBit = 1ull << 48;
constexpr uint64_t kCodeMask = (1ull << 48) - 1;
constexpr int kScanBias = 1 << 20;
constexpr uint32_t kInfD = 0xFFFFFFFFu;

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fffffff); }

// static_cast<int>(float) as compiled for x86-64 (cvttss2si): INT_MIN for
// NaN or out-of-range values.
__device__ __forceinline__ int x86_cvt(float x) {
    return (x >= -2147483648.0f && x < 2147483648.0f) ? __float2int_rz(x) : INT_MIN;
}
// std::min / std::max argument order (NaN handling).
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

// ---------------------------------------------------------------------------
// Warp: decode depth, unproject, R*x+t, project.
// ---------------------------------------------------------------------------

// Depth decode of process_input_frame.cu:346-385 (normalize kernel, built by
// nvcc with fused multiply-add: near + d*(far-near) is one fma).
__device__ __forceinline__ float decode_depth(const DevView& V, size_t idx) {
    float dd = __fmul_rn((float)V.pd[idx], V.depth_scale);
    float z;
    if (V.far_ >= 1000.f)
        z = __fdiv_rn(V.near_, dd);
    else
        z = __fdiv_rn(__fmul_rn(V.far_, V.near_), __fmaf_rn(dd, __fsub_rn(V.far_, V.near_), V.near_));
    if (V.has_invalid && z == 0.f) z = qnan();
    return z;
}

// One warped vertex (u, v, virtual depth): SynthesizedView.cpp:320-331 with
// PerspectiveUnprojector.cpp:59-86 / EquirectangularUnprojector.cpp:55-98,
// SynthesizedView.cpp:68-79 and PerspectiveProjector.cpp:59-87 /
// EquirectangularProjector.cpp:60-99.
__device__ float4 warp_vertex(const DevView& V, const DevTarget& T, int i, int j) {
    const size_t idx = (size_t)i * V.w + j;
    const float d = decode_depth(V, idx);
    float x0, x1, x2;
    if (V.proj == 1) {
        const float ct = V.erp_row[2 * i], st = V.erp_row[2 * i + 1];
        const float cp = V.erp_col[2 * j], sp = V.erp_col[2 * j + 1];
        x0 = __fmul_rn(d, __fmul_rn(ct, cp));
        x1 = __fmul_rn(d, __fmul_rn(ct, sp));
        x2 = __fmul_rn(d, st);
    } else {
        const float pu = __fadd_rn((float)j, 0.5f), pv = __fadd_rn((float)i, 0.5f);
        if (d > 0.f) {
            x0 = d;
            x1 = __fmul_rn(-__fdiv_rn(d, V.f0), __fsub_rn(pu, V.p0));
            x2 = __fmul_rn(-__fdiv_rn(d, V.f1), __fsub_rn(pv, V.p1));
        } else {
            x0 = x1 = x2 = qnan();
        }
    }
    float y[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float s = __fadd_rn(0.f, __fmul_rn(V.R[r * 3 + 0], x0));
        s = __fadd_rn(s, __fmul_rn(V.R[r * 3 + 1], x1));
        s = __fadd_rn(s, __fmul_rn(V.R[r * 3 + 2], x2));
        y[r] = __fadd_rn(s, V.t[r]);
    }
    float u, v, z;
    if (T.proj == 1) {
        double s2 = 0.0;
        s2 = __dadd_rn(s2, __dmul_rn((double)y[0], (double)y[0]));
        s2 = __dadd_rn(s2, __dmul_rn((double)y[1], (double)y[1]));
        s2 = __dadd_rn(s2, __dmul_rn((double)y[2], (double)y[2]));
        const float radius = (float)__dsqrt_rn(s2);
        z = radius;
        const float phi = (float)atan2((double)y[1], (double)y[0]);
        const float theta = (float)asin((double)__fdiv_rn(y[2], radius));
        u = __fadd_rn(T.u0, __fmul_rn(T.du_dphi, phi));
        v = __fadd_rn(T.v0, __fmul_rn(T.dv_dtheta, theta));
    } else {
        if (y[0] > 0.f) {
            u = __fadd_rn(__fdiv_rn(__fmul_rn(-T.f0, y[1]), y[0]), T.p0);
            v = __fadd_rn(__fdiv_rn(__fmul_rn(-T.f1, y[2]), y[0]), T.p1);
            z = y[0];
        } else {
            u = v = z = qnan();
        }
    }
    return make_float4(u, v, z, 0.f);
}

struct FBox {
    float x0, y0, x1, y1;
    __device__ void init() { x0 = y0 = INFINITY; x1 = y1 = -INFINITY; }
    __device__ void add(float4 p) {
        x0 = fminf(x0, p.x); y0 = fminf(y0, p.y);
        x1 = fmaxf(x1, p.x); y1 = fmaxf(y1, p.y);
    }
};

// A vertex can be part of a rasterised triangle only if it passes the
// emission tests of transform.cpp:161-167 (depth > 0, u > 0) and has finite
// coordinates (a triangle with a non-finite coordinate covers no pixel).
// Seam triangles (horizontal wrap) skip the emission tests.
__device__ __forceinline__ bool bbox_vertex_ok(float4 p, bool wrap) {
    if (!(isfinite(p.x) && isfinite(p.y))) return false;
    return wrap || (p.z > 0.f && p.x > 0.f);
}

__device__ int4 to_pixel_box(const FBox& b, int wo, int ho) {
    if (!(b.x0 <= b.x1) || !(b.y0 <= b.y1)) return make_int4(1, 1, 0, 0);
    const float fx0 = floorf(b.x0), fy0 = floorf(b.y0);
    const float fx1 = ceilf(b.x1), fy1 = ceilf(b.y1);
    if (fx0 > (float)(wo - 1) || fy0 > (float)(ho - 1) || fx1 < 0.f || fy1 < 0.f)
        return make_int4(1, 1, 0, 0);
    int4 r;
    r.x = fx0 < 0.f ? 0 : (int)fx0;
    r.y = fy0 < 0.f ? 0 : (int)fy0;
    r.z = fx1 > (float)(wo - 1) ? wo - 1 : (int)fx1;
    r.w = fy1 > (float)(ho - 1) ? ho - 1 : (int)fy1;
    return r;
}

__device__ __forceinline__ FBox block_reduce_box(FBox b, float* sm /* 4 * 8 */) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        b.x0 = fminf(b.x0, __shfl_xor_sync(0xffffffffu, b.x0, o));
        b.y0 = fminf(b.y0, __shfl_xor_sync(0xffffffffu, b.y0, o));
        b.x1 = fmaxf(b.x1, __shfl_xor_sync(0xffffffffu, b.x1, o));
        b.y1 = fmaxf(b.y1, __shfl_xor_sync(0xffffffffu, b.y1, o));
    }
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) {
        sm[warp * 4 + 0] = b.x0; sm[warp * 4 + 1] = b.y0;
        sm[warp * 4 + 2] = b.x1; sm[warp * 4 + 3] = b.y1;
    }
    __syncthreads();
    FBox r;
    r.init();
    const int nw = (blockDim.x * blockDim.y) >> 5;
    for (int w = 0; w < nw; ++w) {
        r.x0 = fminf(r.x0, sm[w * 4 + 0]); r.y0 = fminf(r.y0, sm[w * 4 + 1]);
        r.x1 = fmaxf(r.x1, sm[w * 4 + 2]); r.y1 = fmaxf(r.y1, sm[w * 4 + 3]);
    }
    __syncthreads();
    return r;
}

// Grid (ceil(W/16), ceil(H/16), n_views), block 16x16.  Each CTA writes the
// warped vertices of a 16x16 vertex tile and the pixel bounding boxes of the
// two 16x8-quad binning blocks whose quads start in it (the extra vertex row
// and column they need are recomputed, not written).
__global__ void __launch_bounds__(256) warp_kernel(const DevView* __restrict__ views,
                                                   const DevTarget* __restrict__ tgt) {
    __shared__ float sm[2][32];
    const DevView& V = views[blockIdx.z];
    const DevTarget T = *tgt;
    if ((int)blockIdx.x * 16 >= V.w || (int)blockIdx.y * 16 >= V.h) return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int j = blockIdx.x * 16 + tx, i = blockIdx.y * 16 + ty;
    const bool wrap = T.wrap != 0;
    FBox a, b;
    a.init();
    b.init();
    auto add = [&](float4 p, bool to_a, bool to_b) {
        if (!bbox_vertex_ok(p, wrap)) return;
        if (to_a) a.add(p);
        if (to_b) b.add(p);
    };
    if (i < V.h && j < V.w) {
        const float4 p = warp_vertex(V, T, i, j);
        V.vert[(size_t)i * V.w + j] = p;
        add(p, ty <= 8, ty >= 8);
    }
    if (tx == 15 && i < V.h && j + 1 < V.w) add(warp_vertex(V, T, i, j + 1), ty <= 8, ty >= 8);
    if (ty == 15 && i + 1 < V.h && j < V.w) add(warp_vertex(V, T, i + 1, j), false, true);
    if (tx == 15 && ty == 15 && i + 1 < V.h && j + 1 < V.w)
        add(warp_vertex(V, T, i + 1, j + 1), false, true);
    if (wrap && blockIdx.x == 0 && tx == 0) {
        if (i < V.h) add(warp_vertex(V, T, i, V.w - 1), ty <= 8, ty >= 8);
        if (ty == 15 && i + 1 < V.h) add(warp_vertex(V, T, i + 1, V.w - 1), false, true);
    }
    a = block_reduce_box(a, sm[0]);
    b = block_reduce_box(b, sm[1]);
    if (tx == 0 && ty == 0) {
        const int bx = blockIdx.x, by0 = blockIdx.y * 2;
        if (bx < V.nbx) {
            if (by0 < V.nby) V.bbox[by0 * V.nbx + bx] = to_pixel_box(a, T.wo, T.ho);
            if (by0 + 1 < V.nby) V.bbox[(by0 + 1) * V.nbx + bx] = to_pixel_box(b, T.wo, T.ho);
        }
    }
}

// ---------------------------------------------------------------------------
// Binning of input blocks into output tiles.
// ---------------------------------------------------------------------------

__global__ void bin_count_kernel(const DevView* __restrict__ views, const DevTarget* __restrict__ tgt,
                                 int* __restrict__ counts, DevStatus* __restrict__ st) {
    const int v = blockIdx.y;
    const DevView& V = views[v];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= V.nbx * V.nby) return;
    const int4 bb = V.bbox[b];
    if (bb.x > bb.z || bb.y > bb.w) return;
    const int ntx = tgt->ntx, n = tgt->n_views;
    const int tx0 = bb.x / TILE, tx1 = bb.z / TILE, ty0 = bb.y / TILE, ty1 = bb.w / TILE;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) atomicAdd(&counts[(ty * ntx + tx) * n + v], 1);
    atomicAdd(&st->bin_total, (tx1 - tx0 + 1) * (ty1 - ty0 + 1));
}

// Exclusive scan of the bin counts (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) bin_scan_kernel(const int* __restrict__ counts,
                                                        int* __restrict__ offsets,
                                                        int* __restrict__ cursor, int n,
                                                        const DevTarget* __restrict__ tgt,
                                                        DevStatus* __restrict__ st) {
    __shared__ int warp_sums[32];
    const int tid = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int beg = min(n, tid * per), end = min(n, beg + per);
    int local = 0;
    for (int k = beg; k < end; ++k) local += counts[k];
    // block exclusive scan of `local`
    int x = local;
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    int run = x - local + (warp > 0 ? warp_sums[warp - 1] : 0);
    for (int k = beg; k < end; ++k) {
        offsets[k] = run;
        cursor[k] = run;
        run += counts[k];
    }
    if (tid == 0 && st->bin_total > tgt->bin_capacity) st->bin_overflow = 1;
}

__global__ void bin_fill_kernel(const DevView* __restrict__ views, const DevTarget* __restrict__ tgt,
                                int* __restrict__ cursor, int* __restrict__ list,
                                const DevStatus* __restrict__ st) {
    if (st->bin_overflow) return;
    const int v = blockIdx.y;
    const DevView& V = views[v];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= V.nbx * V.nby) return;
    const int4 bb = V.bbox[b];
    if (bb.x > bb.z || bb.y > bb.w) return;
    const int ntx = tgt->ntx, n = tgt->n_views;
    const int tx0 = bb.x / TILE, tx1 = bb.z / TILE, ty0 = bb.y / TILE, ty1 = bb.w / TILE;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const int pos = atomicAdd(&cursor[(ty * ntx + tx) * n + v], 1);
            list[pos] = b;
        }
}

// ---------------------------------------------------------------------------
// Raster + resolve + blend per output tile.
// ---------------------------------------------------------------------------

// Triangle quality of transform.cpp:62-75 (valid_tri): the longest edge by
// cv::norm (double sum of squared float differences, double sqrt), then
// clamp(10000 - 1000 * stretch, 1, 10000) in float.  sqrt is monotone, so
// the square root of the largest squared length equals the largest length.
__device__ __forceinline__ double sq_len(float ax, float ay, float bx, float by) {
    const double dx = (double)__fsub_rn(ax, bx), dy = (double)__fsub_rn(ay, by);
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}
__device__ __forceinline__ float tri_quality(float4 A, float4 B, float4 C) {
    const double m = fmax(sq_len(B.x, B.y, C.x, C.y),
                          fmax(sq_len(A.x, A.y, B.x, B.y), sq_len(A.x, A.y, C.x, C.y)));
    const float stretch = (float)__dsqrt_rn(m);
    float q = __fsub_rn(10000.f, __fmul_rn(1000.f, stretch));
    q = smax(1.f, q);
    q = smin(10000.f, q);
    return q;
}

struct TriSetup {
    float b1c1, c0b0, c1a1, a0c0, den;
    int x0, x1, y0, y1;  // CPU bounding box
};

// Culling and bounding box of colorize_triangle (transform.cpp:82-96).
// Returns false when the triangle covers nothing.
__device__ __forceinline__ bool tri_setup(float4 A, float4 B, float4 C, int wo, int ho, TriSetup& s) {
    s.b1c1 = __fsub_rn(B.y, C.y);
    s.a0c0 = __fsub_rn(A.x, C.x);
    s.c0b0 = __fsub_rn(C.x, B.x);
    s.c1a1 = __fsub_rn(C.y, A.y);
    const float a1c1 = __fsub_rn(A.y, C.y);
    s.den = __fadd_rn(__fmul_rn(s.b1c1, s.a0c0), __fmul_rn(s.c0b0, a1c1));
    // den <= 0 returns; a NaN or infinite den means a non-finite vertex and
    // no pixel can pass the barycentric test.
    if (!(s.den > 0.f) || isinf(s.den)) return false;
    s.x0 = max(0, x86_cvt(floorf(smin(smin(A.x, B.x), C.x))));
    s.y0 = max(0, x86_cvt(floorf(smin(smin(A.y, B.y), C.y))));
    s.x1 = min(wo - 1, x86_cvt(ceilf(smax(smax(A.x, B.x), C.x))));
    s.y1 = min(ho - 1, x86_cvt(ceilf(smax(smax(A.y, B.y), C.y))));
    return !(s.y0 > s.y1 || s.x0 > s.x1);
}

// Barycentric coordinates at pixel (x, y) exactly as transform.cpp:108-111.
__device__ __forceinline__ void barycentric(const TriSetup& s, float4 C, int x, int y, float& l1,
                                            float& l2, float& l3) {
    const float tx = __fsub_rn(__fadd_rn((float)x, 0.5f), C.x);
    const float ty = __fsub_rn(__fadd_rn((float)y, 0.5f), C.y);
    l1 = __fdiv_rn(__fadd_rn(__fmul_rn(s.b1c1, tx), __fmul_rn(s.c0b0, ty)), s.den);
    l2 = __fdiv_rn(__fadd_rn(__fmul_rn(s.c1a1, tx), __fmul_rn(s.a0c0, ty)), s.den);
    l3 = __fsub_rn(__fsub_rn(1.f, l1), l2);
}

__device__ __forceinline__ bool covered(float l1, float l2, float l3) {
    const float eps = 1e-6f;
    return l1 >= -eps && l2 >= -eps && l3 >= -eps;
}

__device__ __forceinline__ float interp(float a, float b, float c, float l1, float l2, float l3) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a, l1), __fmul_rn(b, l2)), __fmul_rn(c, l3));
}

// The CPU keeps, per output pixel, the fragment with the largest
// quality / depth^3 (accepting a later fragment iff (d/D)^3 * Q < q,
// transform.cpp:119-142), the earliest in scan order on ties.  The key packs
// the bits of depth^3 / quality (smaller is better) above the triangle's
// scan index, so a 64-bit atomicMin keeps the same winner independent of
// scheduling order.
__device__ __forceinline__ void raster_tri(float4 A, float4 B, float4 C, uint32_t tri, int wo, int ho,
                                           int tx0, int ty0, unsigned long long* zb) {
    TriSetup s;
    if (!tri_setup(A, B, C, wo, ho, s)) return;
    const int xa = max(s.x0, tx0), xb = min(s.x1, tx0 + TILE - 1);
    const int ya = max(s.y0, ty0), yb = min(s.y1, ty0 + TILE - 1);
    if (xa > xb || ya > yb) return;
    const float q = tri_quality(A, B, C);
    const float invq = __frcp_rn(q);
    for (int y = ya; y <= yb; ++y)
        for (int x = xa; x <= xb; ++x) {
            float l1, l2, l3;
            barycentric(s, C, x, y, l1, l2, l3);
            if (!covered(l1, l2, l3)) continue;
            const float d = interp(A.z, B.z, C.z, l1, l2, l3);
            if (isnan(d)) continue;
            uint32_t hi = 0u;
            if (d > 0.f) hi = __float_as_uint(__fmul_rn(__fmul_rn(__fmul_rn(d, d), d), invq));
            const unsigned long long key = ((unsigned long long)hi << 32) | tri;
            atomicMin(&zb[(y - ty0) * TILE + (x - tx0)], key);
        }
}

// Rasterises the (up to four) triangles of quad (i, j): transform.cpp:159-176.
__device__ __forceinline__ void raster_quad(const DevView& V, int wo, int ho, bool wrap, int i, int j,
                                            int tx0, int ty0, unsigned long long* zb) {
    const float4* vt = V.vert;
    const size_t r0 = (size_t)i * V.w, r1 = r0 + V.w;
    const float4 v01 = vt[r0 + j + 1], v10 = vt[r1 + j];
    if (!(v01.z > 0.f && v10.z > 0.f && v01.x > 0.f && v10.x > 0.f)) return;
    const float4 v00 = vt[r0 + j], v11 = vt[r1 + j + 1];
    const uint32_t quad = (uint32_t)(i * (V.w - 1) + j);
    if (v00.z > 0.f && v00.x > 0.f) raster_tri(v00, v01, v10, quad * 4u + 0u, wo, ho, tx0, ty0, zb);
    if (v11.z > 0.f && v11.x > 0.f) raster_tri(v11, v10, v01, quad * 4u + 1u, wo, ho, tx0, ty0, zb);
    if (wrap && j == 0) {
        const float4 w0 = vt[r0 + V.w - 1], w1 = vt[r1 + V.w - 1];
        raster_tri(w0, v00, w1, quad * 4u + 2u, wo, ho, tx0, ty0, zb);
        raster_tri(v10, w1, v00, quad * 4u + 3u, wo, ho, tx0, ty0, zb);
    }
}

// Colour of input pixel (x, y): mergeYUV of the loader
// (process_input_frame.cu:211-238) after the chroma upsample of resizeUV
// (process_input_frame.cu:22-81).
__device__ __forceinline__ float chroma_at(const uint16_t* p, int cw, float sx, float sy, int ch,
                                           int x, int y) {
    const float srcx = __fmul_rn((float)x, sx), srcy = __fmul_rn((float)y, sy);
    const int x1 = (int)srcx, y1 = (int)srcy;
    const int x2 = (int)fminf((float)(x1 + 1), (float)(cw - 1));
    const int y2 = (int)fminf((float)(y1 + 1), (float)(ch - 1));
    const float dx = __fsub_rn(srcx, (float)x1), dy = __fsub_rn(srcy, (float)y1);
    const float a = p[y1 * cw + x1], b = p[y1 * cw + x2], c = p[y2 * cw + x1], d = p[y2 * cw + x2];
    const float val1 = __fmaf_rn(b, dx, __fmul_rn(a, __fsub_rn(1.f, dx)));
    const float val2 = __fmaf_rn(d, dx, __fmul_rn(c, __fsub_rn(1.f, dx)));
    return __fmaf_rn(val2, dy, __fmul_rn(val1, __fsub_rn(1.f, dy)));
}

__device__ __forceinline__ float3 input_color(const DevView& V, int x, int y) {
    const float cs = V.color_scale;
    float3 c;
    c.x = __fmul_rn((float)V.py[(size_t)y * V.w + x], cs);
    c.y = __fmul_rn(chroma_at(V.pu, V.cw, V.chroma_sx, V.chroma_sy, V.ch, x, y), cs);
    c.z = __fmul_rn(chroma_at(V.pv, V.cw, V.chroma_sx, V.chroma_sy, V.ch, x, y), cs);
    return c;
}

// Vertex pixel coordinates of triangle `t` of quad (i, j) (transform.cpp:162-174).
__device__ __forceinline__ void tri_vertices(int w, int i, int j, int t, int& ax, int& ay, int& bx,
                                             int& by, int& cx, int& cy) {
    switch (t) {
        case 0: ax = j; ay = i; bx = j + 1; by = i; cx = j; cy = i + 1; break;
        case 1: ax = j + 1; ay = i + 1; bx = j; by = i + 1; cx = j + 1; cy = i; break;
        case 2: ax = w - 1; ay = i; bx = 0; by = i; cx = w - 1; cy = i + 1; break;
        default: ax = 0; ay = i + 1; bx = w - 1; by = i + 1; cx = 0; cy = i; break;
    }
}

struct Fragment {
    float3 col;
    float depth;      // +inf when uncovered
    float validity;   // triangle quality, 0 when uncovered
};

// Re-evaluates the winning triangle at pixel (x, y) exactly as the CPU's
// colorize_triangle does for the fragment it keeps.
__device__ Fragment resolve(const DevView& V, int wo, int ho, unsigned long long key, int x, int y) {
    Fragment f;
    f.col = make_float3(0.f, 0.f, 0.f);
    f.depth = INFINITY;
    f.validity = 0.f;
    if (key == kEmptyKey) return f;
    const uint32_t tri = (uint32_t)(key & 0xffffffffull);
    const uint32_t quad = tri >> 2;
    const int t = (int)(tri & 3u);
    const int i = (int)(quad / (uint32_t)(V.w - 1)), j = (int)(quad % (uint32_t)(V.w - 1));
    int ax, ay, bx, by, cx, cy;
    tri_vertices(V.w, i, j, t, ax, ay, bx, by, cx, cy);
    const float4 A = V.vert[(size_t)ay * V.w + ax];
    const float4 B = V.vert[(size_t)by * V.w + bx];
    const float4 C = V.vert[(size_t)cy * V.w + cx];
    TriSetup s;
    tri_setup(A, B, C, wo, ho, s);
    float l1, l2, l3;
    barycentric(s, C, x, y, l1, l2, l3);
    const float3 ca = input_color(V, ax, ay), cb = input_color(V, bx, by), cc = input_color(V, cx, cy);
    f.col.x = interp(ca.x, cb.x, cc.x, l1, l2, l3);
    f.col.y = interp(ca.y, cb.y, cc.y, l1, l2, l3);
    f.col.z = interp(ca.z, cb.z, cc.z, l1, l2, l3);
    f.depth = interp(A.z, B.z, C.z, l1, l2, l3);
    f.validity = tri_quality(A, B, C);
    return f;
}

__device__ __forceinline__ float blend_pow(float x, float e) {
    return e == 1.f ? x : powf(x, e);
}

__device__ __forceinline__ uint32_t quantize(float c, unsigned max_val) {
    // static_cast<ushort>(v * max_level) (image_writing.cpp:165-172).
    const uint32_t q = __float2uint_rz(__fmul_rn(c, (float)max_val));
    return q > 65535u ? 65535u : q;
}

// Grid: one CTA per 32x32 output tile.  For each input view in blend order:
// clear the shared z-buffer, rasterise the binned blocks with 64-bit
// atomicMin, resolve each pixel's winner and fold it into the running blend
// (BlendedViewSimple::blendBasicMode + blend_img, BlendedView.cpp:180-212,
// blending.cpp:310-369).  Then quantise, write the 2x2 blocks without holes
// directly and leave packed codes for the inpainting passes.
__global__ void __launch_bounds__(TILE_THREADS) tile_kernel(
    const DevView* __restrict__ views, const DevTarget* __restrict__ tgt, const int* __restrict__ counts,
    const int* __restrict__ offsets, const int* __restrict__ list, DevStatus* __restrict__ st,
    uint64_t* __restrict__ codes, uint16_t* __restrict__ out_y, uint16_t* __restrict__ out_u,
    uint16_t* __restrict__ out_v, DebugPtrs dbg) {
    __shared__ unsigned long long zb[TILE * TILE];
    __shared__ int s_hole_box[4];
    const DevTarget T = *tgt;
    const int tile = blockIdx.x;
    const int tx0 = (tile % T.ntx) * TILE, ty0 = (tile / T.ntx) * TILE;
    const int tid = threadIdx.x;
    const bool overflow = st->bin_overflow != 0;
    const bool wrap = T.wrap != 0;
    constexpr int PPT = TILE * TILE / TILE_THREADS;  // pixels per thread
    float acc_c[PPT][3];
    float acc_q[PPT];
    const size_t npo = (size_t)T.wo * T.ho;

    for (int v = 0; v < T.n_views; ++v) {
        const DevView& V = views[v];
        for (int k = tid; k < TILE * TILE; k += TILE_THREADS) zb[k] = kEmptyKey;
        __syncthreads();
        const int items_per_block = BLOCK_W * BLOCK_H;
        if (!overflow) {
            const int bin = tile * T.n_views + v;
            const int cnt = counts[bin], off = offsets[bin];
            for (int it = tid; it < cnt * items_per_block; it += TILE_THREADS) {
                const int e = it / items_per_block, qd = it % items_per_block;
                const int b = list[off + e];
                const int i = (b / V.nbx) * BLOCK_H + qd / BLOCK_W;
                const int j = (b % V.nbx) * BLOCK_W + qd % BLOCK_W;
                if (i < V.h - 1 && j < V.w - 1) raster_quad(V, T.wo, T.ho, wrap, i, j, tx0, ty0, zb);
            }
        } else {
            // Bin list overflowed: test every block's box against this tile.
            const int nb = V.nbx * V.nby;
            for (int it = tid; it < nb * items_per_block; it += TILE_THREADS) {
                const int b = it / items_per_block, qd = it % items_per_block;
                const int4 bb = V.bbox[b];
                if (bb.x > bb.z || bb.z < tx0 || bb.x > tx0 + TILE - 1 || bb.w < ty0 || bb.y > ty0 + TILE - 1)
                    continue;
                const int i = (b / V.nbx) * BLOCK_H + qd / BLOCK_W;
                const int j = (b % V.nbx) * BLOCK_W + qd % BLOCK_W;
                if (i < V.h - 1 && j < V.w - 1) raster_quad(V, T.wo, T.ho, wrap, i, j, tx0, ty0, zb);
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            const int p = tid + k * TILE_THREADS;
            const int x = tx0 + (p & (TILE - 1)), y = ty0 + p / TILE;
            if (x >= T.wo || y >= T.ho) continue;
            const Fragment f = resolve(V, T.wo, T.ho, zb[p], x, y);
            // SynthetisedViewTriangle::transform: quality = validity / depth.
            const float qv = __fdiv_rn(f.validity, f.depth);
            const size_t o = (size_t)y * T.wo + x;
            if (dbg.view_color) {
                float* c = dbg.view_color + ((size_t)v * npo + o) * 3;
                c[0] = f.col.x; c[1] = f.col.y; c[2] = f.col.z;
            }
            if (dbg.view_depth) dbg.view_depth[(size_t)v * npo + o] = f.depth;
            if (dbg.view_validity) dbg.view_validity[(size_t)v * npo + o] = f.validity;
            if (v == 0) {
                acc_c[k][0] = f.col.x; acc_c[k][1] = f.col.y; acc_c[k][2] = f.col.z;
                acc_q[k] = qv;
            } else {
                // blend_img over {accumulator, new view}: weights quality^exp
                // for quality > 0, colour * (1 / sum), quality = sum^(1/exp).
                float sum = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
                if (acc_q[k] > 0.f) {
                    const float w = blend_pow(acc_q[k], T.blend_exp);
                    sum = __fadd_rn(sum, w);
                    c0 = __fadd_rn(c0, __fmul_rn(w, acc_c[k][0]));
                    c1 = __fadd_rn(c1, __fmul_rn(w, acc_c[k][1]));
                    c2 = __fadd_rn(c2, __fmul_rn(w, acc_c[k][2]));
                }
                if (qv > 0.f) {
                    const float w = blend_pow(qv, T.blend_exp);
                    sum = __fadd_rn(sum, w);
                    c0 = __fadd_rn(c0, __fmul_rn(w, f.col.x));
                    c1 = __fadd_rn(c1, __fmul_rn(w, f.col.y));
                    c2 = __fadd_rn(c2, __fmul_rn(w, f.col.z));
                }
                if (sum == 0.f) {
                    acc_c[k][0] = 0.f; acc_c[k][1] = 1.f; acc_c[k][2] = 0.f;
                    acc_q[k] = 0.f;
                } else {
                    const float inv = __frcp_rn(sum);
                    acc_c[k][0] = __fmul_rn(c0, inv);
                    acc_c[k][1] = __fmul_rn(c1, inv);
                    acc_c[k][2] = __fmul_rn(c2, inv);
                    acc_q[k] = blend_pow(sum, T.inv_blend_exp);
                }
            }
        }
        __syncthreads();
    }

    // Quantise into packed codes (Y | U << 16 | V << 32 | hole << 48).
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = tid + k * TILE_THREADS;
        const int x = tx0 + (p & (TILE - 1)), y = ty0 + p / TILE;
        uint64_t code = 0;
        if (x < T.wo && y < T.ho) {
            const bool hole = !(acc_q[k] > 0.f);
            code = (uint64_t)quantize(acc_c[k][0], T.max_val) |
                   ((uint64_t)quantize(acc_c[k][1], T.max_val) << 16) |
                   ((uint64_t)quantize(acc_c[k][2], T.max_val) << 32) | (hole ? kHoleBit : 0ull);
            const size_t o = (size_t)y * T.wo + x;
            if (dbg.blend_color) {
                dbg.blend_color[o * 3 + 0] = acc_c[k][0];
                dbg.blend_color[o * 3 + 1] = acc_c[k][1];
                dbg.blend_color[o * 3 + 2] = acc_c[k][2];
            }
            if (dbg.blend_quality) dbg.blend_quality[o] = acc_q[k];
            if (dbg.inpaint_source) {
                dbg.inpaint_source[o * 2 + 0] = x;
                dbg.inpaint_source[o * 2 + 1] = y;
            }
        }
        zb[p] = code;
    }
    if (tid == 0) {
        s_hole_box[0] = INT_MAX; s_hole_box[1] = INT_MAX;
        s_hole_box[2] = INT_MIN; s_hole_box[3] = INT_MIN;
    }
    __syncthreads();
    // One 2x2 block per thread (16x16 blocks per tile).
    {
        const int bx = tid & 15, by = tid >> 4;
        const int x = tx0 + 2 * bx, y = ty0 + 2 * by;
        if (x < T.wo && y < T.ho) {
            const int l = (2 * by) * TILE + 2 * bx;
            const uint64_t c00 = zb[l], c01 = zb[l + 1], c10 = zb[l + TILE], c11 = zb[l + TILE + 1];
            const size_t o = (size_t)y * T.wo + x;
            codes[o] = c00;
            codes[o + 1] = c01;
            codes[o + T.wo] = c10;
            codes[o + T.wo + 1] = c11;
            const bool any_hole = ((c00 | c01 | c10 | c11) & kHoleBit) != 0;
            if (!any_hole) {
                out_y[o] = (uint16_t)(c00 & 0xffff);
                out_y[o + 1] = (uint16_t)(c01 & 0xffff);
                out_y[o + T.wo] = (uint16_t)(c10 & 0xffff);
                out_y[o + T.wo + 1] = (uint16_t)(c11 & 0xffff);
                const size_t co = (size_t)(y / 2) * (T.wo / 2) + x / 2;
                const uint32_t su = (uint32_t)((c00 >> 16) & 0xffff) + ((c01 >> 16) & 0xffff) +
                                    ((c10 >> 16) & 0xffff) + ((c11 >> 16) & 0xffff);
                const uint32_t sv = (uint32_t)((c00 >> 32) & 0xffff) + ((c01 >> 32) & 0xffff) +
                                    ((c10 >> 32) & 0xffff) + ((c11 >> 32) & 0xffff);
                out_u[co] = (uint16_t)((su + 2) >> 2);
                out_v[co] = (uint16_t)((sv + 2) >> 2);
            } else {
                const int hx0 = (c00 & kHoleBit) || (c10 & kHoleBit) ? x : x + 1;
                const int hx1 = (c01 & kHoleBit) || (c11 & kHoleBit) ? x + 1 : x;
                const int hy0 = (c00 & kHoleBit) || (c01 & kHoleBit) ? y : y + 1;
                const int hy1 = (c10 & kHoleBit) || (c11 & kHoleBit) ? y + 1 : y;
                atomicMin(&s_hole_box[0], hx0);
                atomicMin(&s_hole_box[1], hy0);
                atomicMax(&s_hole_box[2], hx1);
                atomicMax(&s_hole_box[3], hy1);
            }
        }
    }
    __syncthreads();
    if (tid == 0 && s_hole_box[0] != INT_MAX) {
        atomicMin(&st->hole_x0, s_hole_box[0]);
        atomicMin(&st->hole_y0, s_hole_box[1]);
        atomicMax(&st->hole_x1, s_hole_box[2]);
        atomicMax(&st->hole_y1, s_hole_box[3]);
        atomicAdd(&st->n_holes, 1);
    }
}

// ---------------------------------------------------------------------------
// Inpainting (compute_nearest, inpainting.cpp:104-136) as two sweeps of
// min-plus scans over the hole bounding box grown by one pixel.
// ---------------------------------------------------------------------------

struct Region {
    int x0, y0, x1, y1;
    bool empty;
};

__device__ __forceinline__ Region hole_region(const DevStatus* st, int wo, int ho) {
    Region r;
    r.empty = st->n_holes == 0;
    r.x0 = max(0, st->hole_x0 - 1);
    r.y0 = max(0, st->hole_y0 - 1);
    r.x1 = min(wo - 1, st->hole_x1 + 1);
    r.y1 = min(ho - 1, st->hole_y1 + 1);
    return r;
}

__device__ __forceinline__ bool is_hole(const uint64_t* codes, int wo, int x, int y) {
    return (codes[(size_t)y * wo + x] & kHoleBit) != 0;
}

__device__ __forceinline__ uint64_t pack_dxy(uint32_t d, int x, int y) {
    return ((uint64_t)d << 32) | ((uint64_t)(uint32_t)x << 16) | (uint64_t)(uint32_t)y;
}

__device__ __forceinline__ unsigned long long warp_incl_min(unsigned long long v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = y < v ? y : v;
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_incl_min_rev(unsigned long long v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o < 32) v = y < v ? y : v;
    }
    return v;
}

// Sweep 0, rows (forward): R(p) = lexmin over q.x <= p.x of
// (C(q).d + p.x - q.x, C(q).src).  One warp per row of the region.
__global__ void inpaint_row0_kernel(const DevTarget* __restrict__ tgt, const DevStatus* __restrict__ st,
                                    const uint64_t* __restrict__ codes, uint64_t* __restrict__ R) {
    const int wo = tgt->wo, ho = tgt->ho;
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int lane = threadIdx.x & 31;
    const int y = rg.y0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (y > rg.y1) return;
    unsigned long long carry = kEmptyKey;
    for (int base = rg.x0; base <= rg.x1; base += 32) {
        const int x = base + lane;
        unsigned long long key = kEmptyKey;
        if (x <= rg.x1) {
            uint32_t d = kInfD;
            int sx = x, sy = y;
            if (!is_hole(codes, wo, x, y)) {
                d = 0;
            } else if (y + 1 < ho && !is_hole(codes, wo, x, y + 1)) {
                d = 1; sy = y + 1;
            } else if (x + 1 < wo && !is_hole(codes, wo, x + 1, y)) {
                d = 1; sx = x + 1;
            }
            if (d != kInfD) key = pack_dxy((uint32_t)((int)d - x + kScanBias), sx, sy);
        }
        key = warp_incl_min(key, lane);
        key = key < carry ? key : carry;
        if (x <= rg.x1) {
            uint64_t out = ~0ull;
            if (key != kEmptyKey)
                out = pack_dxy((uint32_t)((int)(key >> 32) - kScanBias + x), (int)((key >> 16) & 0xffff),
                               (int)(key & 0xffff));
            R[(size_t)y * wo + x] = out;
        }
        carry = __shfl_sync(0xffffffffu, key, 31);
    }
}

// Column scans: CTA = 32 columns x 32 row segments (one warp per segment).
// Phase 1 reduces each segment, phase 2 rescans it with the carry of the
// segments before it (above for forward scans, below for backward scans).

// Sweep 0, columns (forward): D0, S0 (p) = lexmin over q.y <= p.y of
// (R(q).d + p.y - q.y, src).  Output packed (D0, S0) per pixel.
__device__ __forceinline__ unsigned long long col0_key(const uint64_t* R, int wo, int x, int y) {
    const uint64_t r = R[(size_t)y * wo + x];
    if (r == ~0ull) return kEmptyKey;
    const int d = (int)(r >> 32);
    return pack_dxy((uint32_t)(d - y + kScanBias), (int)((r >> 16) & 0xffff), (int)(r & 0xffff));
}

__global__ void __launch_bounds__(1024) inpaint_col0_kernel(const DevTarget* __restrict__ tgt,
                                                            const DevStatus* __restrict__ st,
                                                            const uint64_t* __restrict__ codes,
                                                            const uint64_t* __restrict__ R,
                                                            uint64_t* __restrict__ DS) {
    __shared__ unsigned long long seg[32][33];
    const int wo = tgt->wo, ho = tgt->ho;
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = rg.x0 + (int)blockIdx.x * 32 + lane;
    if (rg.x0 + (int)blockIdx.x * 32 > rg.x1) return;
    const int nrows = rg.y1 - rg.y0 + 1;
    const int L = (nrows + 31) / 32;
    const int yb = rg.y0 + w * L, ye = min(rg.y1, yb + L - 1);
    const bool col_ok = x <= rg.x1;
    unsigned long long m = kEmptyKey;
    if (col_ok)
        for (int y = yb; y <= ye; ++y) {
            const unsigned long long k = col0_key(R, wo, x, y);
            m = k < m ? k : m;
        }
    seg[w][lane] = m;
    __syncthreads();
    unsigned long long run = kEmptyKey;
    for (int s = 0; s < w; ++s) run = seg[s][lane] < run ? seg[s][lane] : run;
    if (!col_ok) return;
    const uint32_t big = (uint32_t)(wo + ho);
    for (int y = yb; y <= ye; ++y) {
        const unsigned long long k = col0_key(R, wo, x, y);
        run = k < run ? k : run;
        uint64_t out;
        if (!is_hole(codes, wo, x, y))
            out = pack_dxy(0, x, y);
        else if (run == kEmptyKey)
            out = pack_dxy(big, x, y);
        else
            out = pack_dxy((uint32_t)((int)(run >> 32) - kScanBias + y), (int)((run >> 16) & 0xffff),
                           (int)(run & 0xffff));
        DS[(size_t)y * wo + x] = out;
    }
}

// Packed (D0, S0) of pixel (x, y), or (0, itself) outside the region (a
// non-hole: every hole lies inside the region).
__device__ __forceinline__ uint64_t ds_at(const uint64_t* DS, const Region& rg, int wo, int x, int y) {
    if (x < rg.x0 || x > rg.x1 || y < rg.y0 || y > rg.y1) return pack_dxy(0, x, y);
    return DS[(size_t)y * wo + x];
}

// Sweep 1 seeds: T(q) = best of stay (D0(q), S0(q)), left (D0+1, S0 of left),
// up (D0+1, S0 of up) with priority stay > left > up; T'(q) the same without
// stay.  Non-holes: (0, q).
__global__ void inpaint_seed1_kernel(const DevTarget* __restrict__ tgt, const DevStatus* __restrict__ st,
                                     const uint64_t* __restrict__ codes, const uint64_t* __restrict__ DS,
                                     uint64_t* __restrict__ Tq, uint64_t* __restrict__ Tp) {
    const int wo = tgt->wo, ho = tgt->ho;
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int x = rg.x0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = rg.y0 + (int)blockIdx.y;
    if (x > rg.x1 || y > rg.y1) return;
    const size_t o = (size_t)y * wo + x;
    if (!is_hole(codes, wo, x, y)) {
        Tq[o] = pack_dxy(0, x, y);
        Tp[o] = pack_dxy(0, x, y);
        return;
    }
    const uint64_t self = DS[o];
    uint64_t best = self;
    uint64_t bp = ~0ull;
    if (x > 0) {
        const uint64_t l = ds_at(DS, rg, wo, x - 1, y);
        const uint64_t c = l + (1ull << 32);
        if ((c >> 32) < (best >> 32)) best = c;
        bp = c;
    }
    if (y > 0) {
        const uint64_t u = ds_at(DS, rg, wo, x, y - 1);
        const uint64_t c = u + (1ull << 32);
        if ((c >> 32) < (best >> 32)) best = c;
        if (bp == ~0ull || (c >> 32) < (bp >> 32)) bp = c;
    }
    Tq[o] = best;
    Tp[o] = bp;
}

// Sweep 1, rows (backward, exclusive): RR(x, y) = min over q.x > x of
// (T(q).d + q.x, q.x).  One warp per row.
__global__ void inpaint_row1_kernel(const DevTarget* __restrict__ tgt, const DevStatus* __restrict__ st,
                                    const uint64_t* __restrict__ Tq, uint64_t* __restrict__ RR) {
    const int wo = tgt->wo, ho = tgt->ho;
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int lane = threadIdx.x & 31;
    const int y = rg.y0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (y > rg.y1) return;
    unsigned long long carry = kEmptyKey;
    const int n = rg.x1 - rg.x0 + 1;
    for (int base = 0; base < n; base += 32) {
        // process x from the right end: x = x1 - (base + lane)
        const int x = rg.x1 - (base + (31 - lane));
        unsigned long long key = kEmptyKey;
        if (x >= rg.x0) {
            const uint64_t t = Tq[(size_t)y * wo + x];
            key = ((unsigned long long)((t >> 32) + (uint64_t)x) << 16) | (unsigned long long)x;
        }
        // lane 31 holds the rightmost x of this chunk; suffix min towards lane 0
        unsigned long long incl = warp_incl_min_rev(key, lane);
        incl = incl < carry ? incl : carry;
        // exclusive: the value of lane + 1, or the carry for lane 31
        unsigned long long excl = __shfl_down_sync(0xffffffffu, incl, 1);
        if (lane == 31) excl = carry;
        if (x >= rg.x0) RR[(size_t)y * wo + x] = excl;
        carry = __shfl_sync(0xffffffffu, incl, 0);
    }
}

// Sweep 1, columns (backward): for each hole p choose its sweep-1 source
// and copy that pixel's codes (the fill of inpaint_color,
// inpainting.cpp:191-198).
__global__ void __launch_bounds__(1024) inpaint_col1_kernel(
    const DevTarget* __restrict__ tgt, const DevStatus* __restrict__ st, uint64_t* __restrict__ codes,
    const uint64_t* __restrict__ DS, const uint64_t* __restrict__ Tq, const uint64_t* __restrict__ Tp,
    const uint64_t* __restrict__ RR, int32_t* __restrict__ dbg_source) {
    __shared__ unsigned long long seg_col[32][33];
    __shared__ unsigned long long seg_off[32][33];
    const int wo = tgt->wo, ho = tgt->ho;
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = rg.x0 + (int)blockIdx.x * 32 + lane;
    if (rg.x0 + (int)blockIdx.x * 32 > rg.x1) return;
    const bool col_ok = x <= rg.x1;
    const int nrows = rg.y1 - rg.y0 + 1;
    const int L = (nrows + 31) / 32;
    const int yb = rg.y0 + w * L, ye = min(rg.y1, yb + L - 1);
    // Keys: column part (T.d + y) << 16 | y (minimum y on ties);
    //       off-column (RR.d - x + y) << 32 | (0xffff - y) << 16 | qx
    //       (largest y, then smallest x on ties).
    auto col_key = [&](int y) -> unsigned long long {
        const uint64_t t = Tq[(size_t)y * wo + x];
        return ((unsigned long long)((t >> 32) + (uint64_t)y) << 16) | (unsigned long long)y;
    };
    auto off_key = [&](int y) -> unsigned long long {
        const uint64_t r = RR[(size_t)y * wo + x];
        if (r == kEmptyKey) return kEmptyKey;
        const uint64_t v = (r >> 16) - (uint64_t)x + (uint64_t)y;
        return (v << 32) | ((uint64_t)(0xffff - y) << 16) | (r & 0xffff);
    };
    unsigned long long mc = kEmptyKey, mo = kEmptyKey;
    if (col_ok)
        for (int y = yb; y <= ye; ++y) {
            const unsigned long long a = col_key(y), b = off_key(y);
            mc = a < mc ? a : mc;
            mo = b < mo ? b : mo;
        }
    seg_col[w][lane] = mc;
    seg_off[w][lane] = mo;
    __syncthreads();
    unsigned long long run_c = kEmptyKey, run_o = kEmptyKey;
    for (int s = w + 1; s < 32; ++s) {
        run_c = seg_col[s][lane] < run_c ? seg_col[s][lane] : run_c;
        run_o = seg_off[s][lane] < run_o ? seg_off[s][lane] : run_o;
    }
    if (!col_ok) return;
    for (int y = ye; y >= yb; --y) {
        // run_c holds the exclusive (rows below) column minimum here.
        const unsigned long long ok = off_key(y);
        run_o = ok < run_o ? ok : run_o;
        const size_t o = (size_t)y * wo + x;
        const uint64_t code = codes[o];
        if (code & kHoleBit) {
            const uint64_t tp = Tp[o];
            // column candidate (cost, y)
            uint64_t c_cost = tp == ~0ull ? (uint64_t)1 << 40 : (tp >> 32);
            int c_y = y;
            if (run_c != kEmptyKey) {
                const uint64_t cost = (run_c >> 16) - (uint64_t)y;
                if (cost < c_cost) {
                    c_cost = cost;
                    c_y = (int)(run_c & 0xffff);
                }
            }
            uint64_t o_cost = (uint64_t)1 << 40;
            int o_x = 0, o_y = 0;
            if (run_o != kEmptyKey) {
                o_cost = (run_o >> 32) - (uint64_t)y;
                o_y = 0xffff - (int)((run_o >> 16) & 0xffff);
                o_x = (int)(run_o & 0xffff);
            }
            const uint64_t ds = DS[o];
            const uint64_t d0 = ds >> 32;
            uint64_t src = ds;
            if (c_cost <= o_cost) {
                if (c_cost < d0) src = (c_y == y) ? tp : Tq[(size_t)c_y * wo + x];
            } else {
                if (o_cost < d0) src = Tq[(size_t)o_y * wo + o_x];
            }
            const int sx = (int)((src >> 16) & 0xffff), sy = (int)(src & 0xffff);
            codes[o] = (codes[(size_t)sy * wo + sx] & kCodeMask) | kHoleBit;
            if (dbg_source) {
                dbg_source[o * 2 + 0] = sx;
                dbg_source[o * 2 + 1] = sy;
            }
        }
        const unsigned long long ck = col_key(y);
        run_c = ck < run_c ? ck : run_c;
    }
}

// Writes the 2x2 output blocks of the region that hold at least one hole.
__global__ void inpaint_write_kernel(const DevTarget* __restrict__ tgt, const DevStatus* __restrict__ st,
                                     const uint64_t* __restrict__ codes, uint16_t* __restrict__ out_y,
                                     uint16_t* __restrict__ out_u, uint16_t* __restrict__ out_v) {
    const int wo = tgt->wo, ho = tgt->ho;
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int bx0 = rg.x0 / 2, by0 = rg.y0 / 2;
    const int x = 2 * (bx0 + (int)(blockIdx.x * blockDim.x + threadIdx.x));
    const int y = 2 * (by0 + (int)blockIdx.y);
    if (x > rg.x1 || y > rg.y1 || x >= wo || y >= ho) return;
    const size_t o = (size_t)y * wo + x;
    const uint64_t c00 = codes[o], c01 = codes[o + 1], c10 = codes[o + wo], c11 = codes[o + wo + 1];
    if (!((c00 | c01 | c10 | c11) & kHoleBit)) return;
    out_y[o] = (uint16_t)(c00 & 0xffff);
    out_y[o + 1] = (uint16_t)(c01 & 0xffff);
    out_y[o + wo] = (uint16_t)(c10 & 0xffff);
    out_y[o + wo + 1] = (uint16_t)(c11 & 0xffff);
    const size_t co = (size_t)(y / 2) * (wo / 2) + x / 2;
    const uint32_t su = (uint32_t)((c00 >> 16) & 0xffff) + ((c01 >> 16) & 0xffff) + ((c10 >> 16) & 0xffff) +
                        ((c11 >> 16) & 0xffff);
    const uint32_t sv = (uint32_t)((c00 >> 32) & 0xffff) + ((c01 >> 32) & 0xffff) + ((c10 >> 32) & 0xffff) +
                        ((c11 >> 32) & 0xffff);
    out_u[co] = (uint16_t)((su + 2) >> 2);
    out_v[co] = (uint16_t)((sv + 2) >> 2);
}

__global__ void status_init_kernel(DevStatus* st) {
    st->bin_total = 0;
    st->bin_overflow = 0;
    st->hole_x0 = INT_MAX;
    st->hole_y0 = INT_MAX;
    st->hole_x1 = INT_MIN;
    st->hole_y1 = INT_MIN;
    st->n_holes = 0;
}

}  // namespace

int launch_synthesis(const SynthBuffers& b, const LaunchShape& sh, const DebugPtrs& dbg, uint16_t* out_y,
                     uint16_t* out_u, uint16_t* out_v, cudaStream_t s) {
    int launches = 0;
    const int n = sh.n_views;
    const int ntiles = sh.ntx * sh.nty;
    status_init_kernel<<<1, 1, 0, s>>>(b.status);
    ++launches;
    cudaMemsetAsync(b.counts, 0, sizeof(int) * (size_t)ntiles * n, s);
    {
        dim3 grid((sh.max_w + 15) / 16, (sh.max_h + 15) / 16, n);
        warp_kernel<<<grid, dim3(16, 16), 0, s>>>(b.views, b.target);
        ++launches;
    }
    {
        dim3 grid((sh.max_blocks + 255) / 256, n);
        bin_count_kernel<<<grid, 256, 0, s>>>(b.views, b.target, b.counts, b.status);
        bin_scan_kernel<<<1, 1024, 0, s>>>(b.counts, b.offsets, b.cursor, ntiles * n, b.target, b.status);
        bin_fill_kernel<<<grid, 256, 0, s>>>(b.views, b.target, b.cursor, b.list, b.status);
        launches += 3;
    }
    tile_kernel<<<ntiles, TILE_THREADS, 0, s>>>(b.views, b.target, b.counts, b.offsets, b.list, b.status,
                                                b.codes, out_y, out_u, out_v, dbg);
    ++launches;
    {
        const int rows_per_cta = 8;  // 8 warps of 32
        inpaint_row0_kernel<<<(sh.ho + rows_per_cta - 1) / rows_per_cta, 256, 0, s>>>(b.target, b.status,
                                                                                      b.codes, b.scan_a);
        inpaint_col0_kernel<<<(sh.wo + 31) / 32, 1024, 0, s>>>(b.target, b.status, b.codes, b.scan_a,
                                                              b.scan_b);
        inpaint_seed1_kernel<<<dim3((sh.wo + 255) / 256, sh.ho), 256, 0, s>>>(b.target, b.status, b.codes,
                                                                            b.scan_b, b.scan_c, b.scan_d);
        inpaint_row1_kernel<<<(sh.ho + rows_per_cta - 1) / rows_per_cta, 256, 0, s>>>(b.target, b.status,
                                                                                      b.scan_c, b.scan_a);
        inpaint_col1_kernel<<<(sh.wo + 31) / 32, 1024, 0, s>>>(b.target, b.status, b.codes, b.scan_b,
                                                              b.scan_c, b.scan_d, b.scan_a,
                                                              dbg.inpaint_source);
        inpaint_write_kernel<<<dim3((sh.wo / 2 + 127) / 128, (sh.ho + 1) / 2), 128, 0, s>>>(
            b.target, b.status, b.codes, out_y, out_u, out_v);
        launches += 6;
    }
    if (cudaPeekAtLastError() != cudaSuccess) return -1;
    return launches;
}

}  // namespace rvsb
