// Raster stage (templates): one CTA per output tile rasterises every binned
// input block into 64-bit z-buffers in shared memory (a group of views at a
// time), resolves each view's winning fragment per pixel and blends it into
// the tile's accumulators, then quantises and writes the tile.  The tile
// size, the views per z-buffer group, the small-triangle threshold and the
// bin entries staged per round are template parameters; each raster_v*.cu
// instantiates one combination, and the autotuner picks among them.
#pragma once

#include "device_common.cuh"
#include "kernels.hpp"
#include "resolve.cuh"

namespace rvsb {
namespace raster {

using namespace dev;

constexpr int QUADS = BLOCK_W * BLOCK_H;
static_assert(QUADS == 32, "one warp per binning block");
// A binning block whose pixel box exceeds four times its (BLOCK_W + 1) x
// (BLOCK_H + 1) vertices holds stretched triangles (a depth discontinuity)
// and is rasterised before the others of its tile, the longest work first:
// on the plain 1080p view the median box is 60 pixels and 2.5% of the
// blocks exceed this.
constexpr int kBigBlockArea = 4 * (BLOCK_W + 1) * (BLOCK_H + 1);

// TW x TH output pixels per tile (TH <= 32: the stretched-triangle path
// gives one lane per row), VG views per shared z-buffer group, triangles
// with more than SMALL candidate pixels go warp-cooperative, ENT bin
// entries staged per round.
template <int TW_, int TH_, int VG_, int SMALL_, int ENT_, int MED_, int THREADS_ = TILE_THREADS>
struct Cfg {
    static constexpr int TW = TW_, TH = TH_, VG = VG_, SMALL = SMALL_, ENT = ENT_;
    // Threads per CTA (one CTA per tile); CTAs resident per SM with 64
    // registers per thread (1024 threads fill the 65536 registers).
    static constexpr int THREADS = THREADS_, NWARPS = THREADS_ / 32, MIN_CTAS = 1024 / THREADS_;
    // Triangles with more than SMALL and at most MED candidate pixels are
    // rasterised with their candidates flattened across the warp (MED <=
    // SMALL: none); larger ones one at a time, row span by row span.
    static constexpr int MED = MED_;
    static constexpr int BIG = MED_ > SMALL_ ? MED_ : SMALL_;
    static constexpr int NPIX = TW * TH;
    static constexpr size_t kZbBytes = sizeof(unsigned long long) * VG * NPIX;
    static constexpr size_t kEntBytes = sizeof(int) * ENT;
    static constexpr size_t kAccBytes = sizeof(float) * 4 * NPIX;
    static constexpr size_t kSmemBytes = kZbBytes + kEntBytes + kAccBytes;
    static_assert(TH <= 32 && TW % 2 == 0 && TH % 2 == 0, "tile shape");
    static_assert(MED <= 32, "a medium triangle's candidate index stays below 32");
    static_assert(kZbBytes % 16 == 0 && kEntBytes % 16 == 0, "shared-memory carve alignment");
    static_assert(THREADS % 32 == 0 && 1024 % THREADS == 0, "whole warps, whole CTAs per SM");
};

// Candidate pixel (x, y) of a set-up triangle: the coverage test of
// transform.cpp:105-114; on success the fragment key goes to the z-buffer.
// The CPU keeps, per output pixel, the fragment with the largest
// quality / depth^3 (a later fragment replaces the stored one iff
// (d/D)^3 * Q < q, transform.cpp:119-142), the earliest in scan order on
// ties.  The key holds the bits of depth^3 / quality (smaller is better)
// above the triangle's scan index, so 64-bit atomicMin keeps that winner
// whatever the scheduling order.
//
// The coordinates come from rinv, an approximate reciprocal of den (at most
// 1 ulp off).  Then l1 and l2 are within 4u|l| of the CPU's n / den
// (u = 2^-24: 2u from the reciprocal, one rounding here and one in the
// CPU's division), and l3 = (1 - l1) - l2 within
// u * (4|l1| + 2|1 - l1| + 4|l2| + 2|l3|) of the CPU's, which is below
// 21u * M with M = max(|l1|, |l2|, |l3|, 1).  One bound, 24u * M, therefore
// covers every coordinate: the test is decided when the smallest coordinate
// is farther than the bound from -1e-6; otherwise the coordinates are
// recomputed with the reference's divisions.  The depth in the key uses the
// fast coordinates; the resolve recomputes the winning fragment exactly.
__device__ __forceinline__ bool test_pixel(const TriSetup& s, float cx, float cy, float za, float zb_, float zc,
                                           int x, int y, float& d) {
    const float u = 5.9604645e-8f, eps = 1e-6f;
    const float tx = __fsub_rn(__fadd_rn((float)x, 0.5f), cx);
    const float ty = __fsub_rn(__fadd_rn((float)y, 0.5f), cy);
    const float n1 = __fadd_rn(__fmul_rn(s.b1c1, tx), __fmul_rn(s.c0b0, ty));
    const float n2 = __fadd_rn(__fmul_rn(s.c1a1, tx), __fmul_rn(s.a0c0, ty));
    float l1 = __fmul_rn(n1, s.rinv), l2 = __fmul_rn(n2, s.rinv);
    float l3 = __fsub_rn(__fsub_rn(1.f, l1), l2);
    const float mn = fminf(fminf(l1, l2), l3);
    const float M = fmaxf(fmaxf(fabsf(l1), fabsf(l2)), fmaxf(fabsf(l3), 1.f));
    const float bound = __fmul_rn(24.f * u, M);
    if (__fadd_rn(mn, bound) < -eps) return false;
    if (!(__fsub_rn(mn, bound) >= -eps)) {
        l1 = __fdiv_rn(n1, s.den);
        l2 = __fdiv_rn(n2, s.den);
        l3 = __fsub_rn(__fsub_rn(1.f, l1), l2);
        if (!covered(l1, l2, l3)) return false;
    }
    d = interp(za, zb_, zc, l1, l2, l3);
    return !isnan(d);
}

// Quality of the key only (the resolve recomputes it exactly): the longest
// edge in float, a few ulp from the reference's double evaluation.  The
// squared lengths of an edge shared by two triangles are identical, so
// equal reference qualities stay equal here.
__device__ __forceinline__ float key_invq(float4 A, float4 B, float4 C, float precision) {
    auto sq = [](float ax, float ay, float bx, float by) {
        const float dx = __fsub_rn(ax, bx), dy = __fsub_rn(ay, by);
        return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    };
    const float m = fmaxf(sq(B.x, B.y, C.x, C.y), fmaxf(sq(A.x, A.y, B.x, B.y), sq(A.x, A.y, C.x, C.y)));
    float stretch = __fsqrt_rn(m);
    if (precision != 1.f) stretch = __fdiv_rn(stretch, precision);
    const float q = fminf(10000.f, fmaxf(1.f, __fsub_rn(10000.f, __fmul_rn(1000.f, stretch))));
    return rcp_approx(q);
}

__device__ __forceinline__ unsigned long long frag_key(float d, float invq, uint32_t tri) {
    uint32_t hi = 0u;
    if (d > 0.f) hi = __float_as_uint(__fmul_rn(__fmul_rn(__fmul_rn(d, d), d), invq));
    return ((unsigned long long)hi << 32) | tri;
}

// Rasterises the triangles of the 32 quads of binning block `b` of view V
// (one quad per lane) into the tile's z-buffer `zb`: transform.cpp:159-176.
template <class C>
__device__ __forceinline__ void raster_block(const DevView& V, int wo, int ho, bool wrap, int bx, int by,
                                             int tx0, int ty0, unsigned long long* zb, int lane, float precision) {
    const int i = by * BLOCK_H + lane / BLOCK_W, j = bx * BLOCK_W + lane % BLOCK_W;
    const bool quad_ok = i < V.h - 1 && j < V.w - 1;
    float4 v00, v01, v10, v11;
    bool cond0 = false;
    const size_t r0 = (size_t)i * V.w, r1 = r0 + V.w;
    if (quad_ok) {
        // All four corners at once (one memory round trip), then the
        // emission test of transform.cpp:161.
        v00 = __ldg(V.vert + r0 + j);
        v01 = __ldg(V.vert + r0 + j + 1);
        v10 = __ldg(V.vert + r1 + j);
        v11 = __ldg(V.vert + r1 + j + 1);
        cond0 = v01.z > 0.f && v10.z > 0.f && v01.x > 0.f && v10.x > 0.f;
    }
    // Scan order of transform.cpp:159-176: row i, column j, then triangle
    // 1, triangle 2, and the two seam triangles at j = 0.
    const uint32_t quad = ((uint32_t)i << (V.tri_shift - 2)) | (uint32_t)j;
    const int n_slots = wrap ? 4 : 2;
    for (int slot = 0; slot < n_slots; ++slot) {
        float4 A, B, C;
        bool active = cond0;
        switch (slot) {
            case 0: A = v00; B = v01; C = v10; active = active && v00.z > 0.f && v00.x > 0.f; break;
            case 1: A = v11; B = v10; C = v01; active = active && v11.z > 0.f && v11.x > 0.f; break;
            // Seam triangles (wrapping outputs only): their column W-1
            // vertices are loaded here, so that they hold no registers
            // across the common case.
            case 2:
                active = active && j == 0;
                A = B = C = v00;
                if (active) {
                    A = __ldg(V.vert + r0 + V.w - 1);
                    C = __ldg(V.vert + r1 + V.w - 1);
                }
                break;
            default:
                active = active && j == 0;
                A = v10; B = v10; C = v00;
                if (active) B = __ldg(V.vert + r1 + V.w - 1);
                break;
        }
        TriSetup s;
        int count = 0;
        if (active && tri_coef(A, B, C, s) &&
            tri_range(A, B, C, wo, ho, tx0, tx0 + C::TW - 1, ty0, ty0 + C::TH - 1, s)) {
            count = (s.x1 - s.x0 + 1) * (s.y1 - s.y0 + 1);
            s.rinv = rcp_approx(s.den);
        }
        const uint32_t tri = quad * 4u + (uint32_t)slot;
        const bool medium = count > C::SMALL && count <= C::MED;
        const bool big = count > C::BIG;
        if (count > 0 && count <= C::SMALL) {
            // One flat loop over the candidate box (at most SMALL pixels),
            // with the quality key computed once up front.
            const float invq = key_invq(A, B, C, precision);
            int x = s.x0, y = s.y0;
            for (int k = 0; k < count; ++k) {
                float d;
                if (test_pixel(s, C.x, C.y, A.z, B.z, C.z, x, y, d))
                    atomicMin(&zb[(y - ty0) * C::TW + (x - tx0)], frag_key(d, invq, tri));
                if (++x > s.x1) {
                    x = s.x0;
                    ++y;
                }
            }
        }
        // Medium triangles (at most MED candidates in their box): the
        // candidates of all of the warp's medium triangles flattened into
        // one sequence, 32 per round; each lane fetches its candidate's
        // triangle from the lane that set it up.
        if constexpr (C::MED > C::SMALL) {
            if (__ballot_sync(0xffffffffu, medium)) {
                const int mc = medium ? count : 0;
                int incl = mc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const int excl = incl - mc;
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                const float invq_m = medium ? key_invq(A, B, C, precision) : 0.f;
                const int bw = s.x1 - s.x0 + 1;
                for (int base = 0; base < total; base += 32) {
                    const int c = base + lane;
                    int own = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        const int probe = __shfl_sync(0xffffffffu, incl, own + step - 1);
                        if (probe <= c) own += step;
                    }
                    TriSetup t;
                    t.b1c1 = __shfl_sync(0xffffffffu, s.b1c1, own);
                    t.c0b0 = __shfl_sync(0xffffffffu, s.c0b0, own);
                    t.c1a1 = __shfl_sync(0xffffffffu, s.c1a1, own);
                    t.a0c0 = __shfl_sync(0xffffffffu, s.a0c0, own);
                    t.den = __shfl_sync(0xffffffffu, s.den, own);
                    t.rinv = __shfl_sync(0xffffffffu, s.rinv, own);
                    const float cx = __shfl_sync(0xffffffffu, C.x, own), cy = __shfl_sync(0xffffffffu, C.y, own);
                    const float za = __shfl_sync(0xffffffffu, A.z, own), zb_ = __shfl_sync(0xffffffffu, B.z, own);
                    const float zc = __shfl_sync(0xffffffffu, C.z, own);
                    const float invq = __shfl_sync(0xffffffffu, invq_m, own);
                    const uint32_t ttri = __shfl_sync(0xffffffffu, tri, own);
                    const int ox0 = __shfl_sync(0xffffffffu, s.x0, own), oy0 = __shfl_sync(0xffffffffu, s.y0, own);
                    const int obw = __shfl_sync(0xffffffffu, bw, own), oex = __shfl_sync(0xffffffffu, excl, own);
                    if (c >= total) continue;
                    // k < MED <= 32 and the box width <= 32: (k + 0.5) / width is
                    // at least 1/64 from an integer, so the fast quotient
                    // truncates to the exact row.
                    const int k = c - oex;
                    const int dy = (int)__fdividef((float)k + 0.5f, (float)obw);
                    const int x = ox0 + (k - dy * obw), y = oy0 + dy;
                    float d;
                    if (test_pixel(t, cx, cy, za, zb_, zc, x, y, d))
                        atomicMin(&zb[(y - ty0) * C::TW + (x - tx0)], frag_key(d, invq, ttri));
                }
            }
        }
        unsigned mask = __ballot_sync(0xffffffffu, big);
        if (!mask) continue;
        float invq_own = 0.f;
        if (big) invq_own = key_invq(A, B, C, precision);
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            TriSetup t;
            t.b1c1 = __shfl_sync(0xffffffffu, s.b1c1, src);
            t.c0b0 = __shfl_sync(0xffffffffu, s.c0b0, src);
            t.c1a1 = __shfl_sync(0xffffffffu, s.c1a1, src);
            t.a0c0 = __shfl_sync(0xffffffffu, s.a0c0, src);
            t.den = __shfl_sync(0xffffffffu, s.den, src);
            t.rinv = __shfl_sync(0xffffffffu, s.rinv, src);
            const float cx = __shfl_sync(0xffffffffu, C.x, src), cy = __shfl_sync(0xffffffffu, C.y, src);
            const float za = __shfl_sync(0xffffffffu, A.z, src), zb_ = __shfl_sync(0xffffffffu, B.z, src);
            const float zc = __shfl_sync(0xffffffffu, C.z, src);
            const float invq = __shfl_sync(0xffffffffu, invq_own, src);
            const uint32_t ttri = __shfl_sync(0xffffffffu, tri, src);
            t.x0 = __shfl_sync(0xffffffffu, s.x0, src);
            t.x1 = __shfl_sync(0xffffffffu, s.x1, src);
            t.y0 = __shfl_sync(0xffffffffu, s.y0, src);
            t.y1 = __shfl_sync(0xffffffffu, s.y1, src);
            // Candidate span of each row of the (tile-clipped) range, one lane
            // per row (at most TH rows), then the spans' pixels flattened
            // over the warp: 32 candidates per round whatever the shape.
            const int y = t.y0 + lane;
            int xl = 0, xr = -1;
            if (y <= t.y1) row_span(t, cx, cy, y, xl, xr);
            const int len = max(0, xr - xl + 1);
            int incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int excl = incl - len;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int base = 0; base < total; base += 32) {
                const int c = base + lane;
                // Row of candidate c: the number of rows whose spans end at
                // or before c (binary search over the inclusive prefix).
                int row = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int probe = __shfl_sync(0xffffffffu, incl, row + step - 1);
                    if (probe <= c) row += step;
                }
                const int rxl = __shfl_sync(0xffffffffu, xl, row);
                const int rex = __shfl_sync(0xffffffffu, excl, row);
                if (c >= total) continue;
                const int x = rxl + (c - rex), yy = t.y0 + row;
                float d;
                if (!test_pixel(t, cx, cy, za, zb_, zc, x, yy, d)) continue;
                atomicMin(&zb[(yy - ty0) * C::TW + (x - tx0)], frag_key(d, invq, ttri));
            }
        }
    }
}


// Resolves and blends the views g0 .. g0 + gn - 1 of the tile, one pixel per
// thread and step, into the accumulators (c0, c1, c2, q per pixel).
// Extras: the per-view multispectral, auxiliary and debug outputs are
// written (without them the view loop holds no global store, so a view's
// loads may be issued while the previous view is blended).
template <class C, bool Extras>
__device__ __forceinline__ void resolve_group(const SlotTable& tab, int g0, int gn, int tx0, int ty0,
                                              const unsigned long long (*zb)[C::NPIX], float (*acc)[C::NPIX],
                                              const DebugPtrs& dbg) {
    const DevTarget& T = tab.t;
    const size_t npo = (size_t)T.wo * T.ho;
    for (int p = threadIdx.x; p < C::NPIX; p += C::THREADS) {
        const int x = tx0 + p % C::TW, y = ty0 + p / C::TW;
        if (x >= T.wo || y >= T.ho) continue;
        BlendAcc a = {0.f, 0.f, 0.f, 0.f};
        if (g0 > 0) {
            a.c0 = acc[0][p]; a.c1 = acc[1][p]; a.c2 = acc[2][p]; a.q = acc[3][p];
        }
        const bool aux = Extras && tab.aux.on != 0;
        const size_t po = (size_t)y * T.wo + x;
        float adepth = 0.f, avalid = 0.f;
        if (aux && g0 > 0) {
            adepth = tab.aux.acc_depth[po];
            avalid = tab.aux.acc_valid[po];
        }
        for (int k = 0; k < gn; ++k) {
            const int v = g0 + k;
            const Fragment f = resolve_fragment(tab.v[v], zb[k][p], x, y, T.precision);
            const float qv = __fdiv_rn(f.validity, f.depth);
            if (Extras && tab.ms.on) tab.ms.view[(size_t)v * npo + po] = make_float4(f.col.x, f.col.y, f.col.z, qv);
            if (aux) {
                // BlendedView.cpp:205-208: the view's depth where its quality
                // beats the accumulator's before this blend (view 0: its
                // quality; later: (weight sum)^(1/exp)); validity = max.
                if (v == 0) {
                    adepth = f.depth;
                    avalid = f.validity;
                } else {
                    const float qacc =
                        (v == 1 || T.blend_max) ? a.q : (a.q > 0.f ? powf(a.q, T.inv_blend_exp) : a.q);
                    if (qv > qacc) adepth = f.depth;
                    avalid = smax(avalid, f.validity);
                }
            }
            if (Extras && (dbg.view_color || dbg.view_depth || dbg.view_validity)) {
                const size_t o = (size_t)y * T.wo + x;
                if (dbg.view_color) {
                    float* c = dbg.view_color + ((size_t)v * npo + o) * 3;
                    c[0] = f.col.x; c[1] = f.col.y; c[2] = f.col.z;
                }
                if (dbg.view_depth) dbg.view_depth[(size_t)v * npo + o] = f.depth;
                if (dbg.view_validity) dbg.view_validity[(size_t)v * npo + o] = f.validity;
            }
            blend_view(a, v, f, qv, T);
        }
        acc[0][p] = a.c0; acc[1][p] = a.c1; acc[2][p] = a.c2; acc[3][p] = a.q;
        if (aux) {
            tab.aux.acc_depth[po] = adepth;
            tab.aux.acc_valid[po] = avalid;
        }
    }
}

// Quantises the tile (image_writing.cpp:142-180), one 2x2 block per thread
// and round: packed codes and the hole mask for the inpainting passes, the
// 4:2:0 samples of blocks without holes, and the bounding box of the holes.
template <class C>
__device__ __forceinline__ void write_tile(const DevTarget& T, int tx0, int ty0, const float (*acc)[C::NPIX],
                                          DevStatus* st, uint64_t* codes, uint8_t* holes, uint16_t* out_y,
                                          uint16_t* out_u, uint16_t* out_v, const DebugPtrs& dbg, float4* pcolor) {
    constexpr int BW = C::TW / 2, NB = (C::TW / 2) * (C::TH / 2);
    int hx0 = INT_MAX, hy0 = INT_MAX, hx1 = INT_MIN, hy1 = INT_MIN;
    bool warp_hole = false;
    for (int base = 0; base < NB; base += C::THREADS) {
        const int t = base + (int)threadIdx.x;
        const int lx = 2 * (t % BW), ly = 2 * (t / BW);
        const int x0 = tx0 + lx, y0 = ty0 + ly;
        const bool inside = t < NB && x0 < T.wo && y0 < T.ho;
        uint64_t code[4] = {0, 0, 0, 0};
        bool any_hole = false;
        // A raster of odd width or height (Precision != 1 only: the output
        // itself has even sides) ends in partial blocks.
        const bool full = x0 + 1 < T.wo && y0 + 1 < T.ho;
        if (inside) {
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                if (!full && (x0 + (p & 1) >= T.wo || y0 + (p >> 1) >= T.ho)) continue;
                const int sp = (ly + (p >> 1)) * C::TW + lx + (p & 1);
                const float c0 = acc[0][sp], c1 = acc[1][sp], c2 = acc[2][sp], q = acc[3][sp];
                const bool hole = !(q > 0.f);
                any_hole |= hole;
                code[p] = (uint64_t)quantize(c0, T.max_val) | ((uint64_t)quantize(c1, T.max_val) << 16) |
                          ((uint64_t)quantize(c2, T.max_val) << 32) | (hole ? kHoleBit : 0ull);
                const int x = x0 + (p & 1), y = y0 + (p >> 1);
                const size_t o = (size_t)y * T.wo + x;
                if (dbg.blend_color) {
                    dbg.blend_color[o * 3 + 0] = c0;
                    dbg.blend_color[o * 3 + 1] = c1;
                    dbg.blend_color[o * 3 + 2] = c2;
                }
                if (dbg.blend_quality)
                    dbg.blend_quality[o] =
                        (T.n_views == 1 || T.blend_max || !(q > 0.f)) ? q : powf(q, T.inv_blend_exp);
                if (dbg.inpaint_source) {
                    dbg.inpaint_source[o * 2 + 0] = x;
                    dbg.inpaint_source[o * 2 + 1] = y;
                }
                if (T.rescale) pcolor[o] = make_float4(c0, c1, c2, 0.f);
            }
            const size_t o = (size_t)y0 * T.wo + x0;
            auto hole_of = [](uint64_t c) -> uint16_t { return (c & kHoleBit) ? 1 : 0; };
            if (!(T.wo & 1)) {
                reinterpret_cast<ulonglong2*>(codes + o)[0] = make_ulonglong2(code[0], code[1]);
                reinterpret_cast<uint16_t*>(holes + o)[0] = (uint16_t)(hole_of(code[0]) | (hole_of(code[1]) << 8));
                if (full) {
                    reinterpret_cast<ulonglong2*>(codes + o + T.wo)[0] = make_ulonglong2(code[2], code[3]);
                    reinterpret_cast<uint16_t*>(holes + o + T.wo)[0] =
                        (uint16_t)(hole_of(code[2]) | (hole_of(code[3]) << 8));
                }
            } else {
                // odd width: the second row of a block is not 16-byte aligned
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const int x = x0 + (p & 1), y = y0 + (p >> 1);
                    if (x >= T.wo || y >= T.ho) continue;
                    codes[(size_t)y * T.wo + x] = code[p];
                    holes[(size_t)y * T.wo + x] = (uint8_t)hole_of(code[p]);
                }
            }
            if (!any_hole && !T.rescale) {
                reinterpret_cast<uint32_t*>(out_y + o)[0] =
                    (uint32_t)(code[0] & 0xffff) | ((uint32_t)(code[1] & 0xffff) << 16);
                reinterpret_cast<uint32_t*>(out_y + o + T.wo)[0] =
                    (uint32_t)(code[2] & 0xffff) | ((uint32_t)(code[3] & 0xffff) << 16);
                uint32_t su = 0, sv = 0;
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    su += (uint32_t)((code[p] >> 16) & 0xffff);
                    sv += (uint32_t)((code[p] >> 32) & 0xffff);
                }
                const size_t co = (size_t)(y0 / 2) * (T.wo / 2) + x0 / 2;
                out_u[co] = quarter_round(su, T.chroma_ties_up);
                out_v[co] = quarter_round(sv, T.chroma_ties_up);
            }
        }
        if (any_hole) {
            const bool left = (code[0] & kHoleBit) || (code[2] & kHoleBit);
            const bool right = (code[1] & kHoleBit) || (code[3] & kHoleBit);
            const bool top = (code[0] & kHoleBit) || (code[1] & kHoleBit);
            const bool bottom = (code[2] & kHoleBit) || (code[3] & kHoleBit);
            hx0 = min(hx0, left ? x0 : x0 + 1);
            hx1 = max(hx1, right ? x0 + 1 : x0);
            hy0 = min(hy0, top ? y0 : y0 + 1);
            hy1 = max(hy1, bottom ? y0 + 1 : y0);
            warp_hole = true;
        }
    }
    // Bounding box of the holes: warp reduction, one atomic per warp.
    const unsigned m = __ballot_sync(0xffffffffu, warp_hole);
    if (m) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            hx0 = min(hx0, __shfl_xor_sync(0xffffffffu, hx0, o));
            hy0 = min(hy0, __shfl_xor_sync(0xffffffffu, hy0, o));
            hx1 = max(hx1, __shfl_xor_sync(0xffffffffu, hx1, o));
            hy1 = max(hy1, __shfl_xor_sync(0xffffffffu, hy1, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&st->hole_x0, hx0);
            atomicMin(&st->hole_y0, hy0);
            atomicMax(&st->hole_x1, hx1);
            atomicMax(&st->hole_y1, hy1);
            atomicAdd(&st->n_holes, 1);
        }
    }
}

// Grid (max tiles, slots): one CTA per TW x TH output tile of a slot.
// Views are processed in groups of VG: clear the group's shared z-buffers,
// stage the group's bin entries (view, block) in shared memory, rasterise
// them (one warp per block), then resolve and blend the group's views into
// the tile's accumulators.  After the last group the tile is quantised and
// written.
template <class C, class Tabs>
__global__ void __launch_bounds__(C::THREADS, C::MIN_CTAS) raster_kernel(const __grid_constant__ Tabs tabs) {
    grid_dep_wait();
    // Dynamic shared memory: the group's z-buffers, the staged bin entries
    // and the tile's blend accumulators.
    extern __shared__ __align__(16) unsigned char s_raw[];
    auto zb = reinterpret_cast<unsigned long long(*)[C::NPIX]>(s_raw);
    int* s_ent = reinterpret_cast<int*>(s_raw + C::kZbBytes);
    auto acc = reinterpret_cast<float(*)[C::NPIX]>(s_raw + C::kZbBytes + C::kEntBytes);
    __shared__ int s_pref[C::VG + 1];
    __shared__ int s_off[C::VG];
    __shared__ int s_next, s_front, s_back;
    const SlotTable& tab = tabs.at(blockIdx.y);
    const DevTarget& T = tab.t;
    if ((int)blockIdx.x >= T.ntx * T.nty) return;
    const int tile = tab.b.tile_order[blockIdx.x];
    const int* __restrict__ counts = tab.b.counts;
    const int* __restrict__ offsets = tab.b.offsets;
    const int* __restrict__ list = tab.b.list;
    const int tx0 = (tile % T.ntx) * C::TW, ty0 = (tile / T.ntx) * C::TH;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool overflow = tab.b.status->bin_overflow != 0;
    const bool wrap = T.wrap != 0;

    for (int g0 = 0; g0 < T.n_views; g0 += C::VG) {
        const int gn = min(C::VG, T.n_views - g0);
        for (int k = tid; k < gn * C::NPIX; k += C::THREADS) zb[k / C::NPIX][k % C::NPIX] = kEmptyKey;
        if (tid == 0) {
            int run = 0;
            for (int k = 0; k < gn; ++k) {
                s_pref[k] = run;
                const DevView& V = tab.v[g0 + k];
                const int bin = tile * T.n_views + g0 + k;
                s_off[k] = overflow ? 0 : offsets[bin];
                run += overflow ? V.nbx * V.nby : counts[bin];
            }
            s_pref[gn] = run;
        }
        __syncthreads();
        const int E = s_pref[gn];
        for (int base = 0; base < E; base += C::ENT) {
            const int n = min(C::ENT, E - base);
            if (tid == 0) {
                s_next = C::NWARPS;
                s_front = 0;
                s_back = 0;
            }
            __syncthreads();
            // Staged big blocks first (from the front), the others from the
            // back; the order within each part does not matter (the keys
            // are order independent).
            for (int q = tid; q < n; q += C::THREADS) {
                const int e = base + q;
                int k = 0;
                while (k + 1 < gn && e >= s_pref[k + 1]) ++k;
                int b;
                if (overflow) {
                    const DevView& V = tab.v[g0 + k];
                    b = e - s_pref[k];
                    const int4 bb = V.bbox[b];
                    if (bb.x > bb.z || bb.z < tx0 || bb.x > tx0 + C::TW - 1 || bb.w < ty0 ||
                        bb.y > ty0 + C::TH - 1)
                        b = -1;
                    else
                        b = ((b / V.nbx) << 11) | (b % V.nbx);
                } else {
                    b = list[s_off[k] + (e - s_pref[k])];
                }
                int code = -1;
                bool big_block = false;
                if (b >= 0) {
                    code = (k << 26) | b;
                    const DevView& V = tab.v[g0 + k];
                    const int4 bb = V.bbox[(b >> 11) * V.nbx + (b & 2047)];
                    big_block = (bb.z - bb.x + 1) * (bb.w - bb.y + 1) > kBigBlockArea;
                }
                s_ent[big_block ? atomicAdd(&s_front, 1) : n - 1 - atomicAdd(&s_back, 1)] = code;
            }
            __syncthreads();
            // Entries are taken dynamically: a warp claims its next entry
            // before rasterising the current one, so that warps which meet
            // stretched triangles do not hold the others at the barrier.
            for (int q = warp; q < n;) {
                const int ent = s_ent[q];
                int next = 0;
                if (lane == 0) next = atomicAdd(&s_next, 1);
                if (ent >= 0) {
                    const int k = ent >> 26, bx = ent & 2047, by = (ent >> 11) & 32767;
                    raster_block<C>(tab.v[g0 + k], T.wo, T.ho, wrap, bx, by, tx0, ty0, zb[k], lane, T.precision);
                }
                q = __shfl_sync(0xffffffffu, next, 0);
            }
            __syncthreads();
        }
        if (tab.ms.on || tab.aux.on || tab.dbg.view_color || tab.dbg.view_depth || tab.dbg.view_validity)
            resolve_group<C, true>(tab, g0, gn, tx0, ty0, zb, acc, tab.dbg);
        else
            resolve_group<C, false>(tab, g0, gn, tx0, ty0, zb, acc, tab.dbg);
        __syncthreads();
    }
    write_tile<C>(T, tx0, ty0, acc, tab.b.status, tab.b.codes, tab.b.holes, tab.out_y, tab.out_u, tab.out_v,
                  tab.dbg, tab.b.pcolor);
}

template <class C, class Tabs>
void launch(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    launch_dependent(raster_kernel<C, Tabs>, dim3(sh.max_tiles, sh.slots), dim3(C::THREADS), C::kSmemBytes, s, tabs);
}

template <class C>
void prepare() {
    cudaFuncSetAttribute(raster_kernel<C, TableParam>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)C::kSmemBytes);
    cudaFuncSetAttribute(raster_kernel<C, TablePtr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)C::kSmemBytes);
}

}  // namespace raster
}  // namespace rvsb

// Defines the host entry points of raster variant N (one per .cu file, so
// the variants compile in parallel).
#define RVSB_RASTER_VARIANT(N, TW, TH, VG, SMALL, ENT, MED, THREADS)                                      \
    namespace rvsb {                                                                                     \
    using RasterCfg##N = raster::Cfg<TW, TH, VG, SMALL, ENT, MED, THREADS>;                              \
    static_assert(kRasterVariants[N].tw == TW && kRasterVariants[N].th == TH &&                          \
                      kRasterVariants[N].vg == VG && kRasterVariants[N].small == SMALL &&                \
                      kRasterVariants[N].ent == ENT && kRasterVariants[N].med == MED &&                  \
                      kRasterVariants[N].threads == THREADS,                                             \
                  "variant table");                                                                      \
    void launch_raster_v##N(const TableParam& t, const BatchShape& sh, cudaStream_t s) {                 \
        raster::launch<RasterCfg##N>(t, sh, s);                                                          \
    }                                                                                                    \
    void launch_raster_v##N(const TablePtr& t, const BatchShape& sh, cudaStream_t s) {                   \
        raster::launch<RasterCfg##N>(t, sh, s);                                                          \
    }                                                                                                    \
    void prepare_raster_v##N() { raster::prepare<RasterCfg##N>(); }                                      \
    }
