// Inpainting stage: compute_nearest (rvs/src/inpainting.cpp:104-136) as two
// sweeps of min-plus scans over the hole bounding box grown by one pixel,
// then the fill of inpaint_color (inpainting.cpp:191-198) and the write of
// the 2x2 output blocks that held holes.
//
// Why two sweeps of scans are exact: the reference alternates column-major
// Gauss-Seidel sweeps (forward, then reverse) until one changes nothing.
// After the forward sweep 0 and the reverse sweep 1 every distance equals
// the L1 distance transform, so sweep 2 never changes anything and the
// result is the state after sweep 1.  Each sweep is a min-plus recurrence
// over left/up (or right/down) neighbours with a fixed neighbour priority:
//  sweep 0: (D0, S0)(p) = lexmin over q with q.x <= p.x, q.y <= p.y of
//           (C(q).d + |p - q|, C(q).source), C(q) = (0, q) for a non-hole,
//           (1, down(q)) or else (1, right(q)) for a hole whose down/right
//           neighbour is a non-hole;
//  sweep 1: seeds T(q) = best of stay (D0, S0), left (D0 + 1, S0 of left),
//           up (D0 + 1, S0 of up), in that priority (T'(q) without stay);
//           a hole p takes the best seed of its lower-right quadrant, from
//           its own column (smallest y) when the column holds a minimum,
//           otherwise the minimum with the largest y, then smallest x, and
//           changes only on strict improvement.
// Every hole lies inside the region and every source lies within one pixel
// of a hole, so restricting the scans to the grown bounding box changes
// nothing.  Loads are issued in batches (RB rows, CB chunks) so each thread
// keeps several in flight.  The last column scan only records each hole's
// choice (its source, or the seed it takes the source from); the gathers
// that follow a choice (the seed, then the source pixel's codes) run in the
// write pass, one thread per 2x2 block, off the scans' serial chains.
#include <algorithm>

#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

constexpr int kScanBias = 1 << 20;
constexpr uint32_t kInfD = 0xFFFFFFFFu;
constexpr int CB = 4;  // row scans: 32-pixel chunks loaded per batch
constexpr int RB = 8;  // column scans: rows loaded per batch
constexpr int RB1 = 4; // last column scan: rows per batch (five words a row)
// A hole's sweep-1 choice stored in its D0/S0 word by the last column
// scan: with this bit, (x << 16 | y) of the seed T(q) whose source it
// takes; without, its source itself (x << 16 | y in the low 32 bits).
constexpr uint64_t kSeedRef = 1ull << 63;

struct Region {
    int x0, y0, x1, y1;
    bool empty;
};

// The buffers of one image the passes work on.
struct InpaintImage {
    int wo, ho;
    const DevStatus* st;       // hole count and bounding box
    const uint8_t* holes;      // wo*ho, nonzero = hole
    uint64_t* codes;           // wo*ho packed codes (the fill copies them)
    uint64_t* scan[4];         // wo*ho words each
    int32_t* sources;          // optional: (x, y) source of every hole
    uint64_t* seg;             // column-group minima (2 words per group, strip and lane), G > 1 only
    uint16_t* out_y;
    uint16_t* out_u;
    uint16_t* out_v;
    int ties_up;               // output chroma rounding
    int no_write;              // Precision != 1: the resize writes the output
};

// Image of slot blockIdx.z of a batch.
template <class Tabs>
struct FromTables {
    Tabs tabs;
    __device__ InpaintImage operator()() const {
        const SlotTable& t = tabs.at(blockIdx.z);
        InpaintImage im;
        im.wo = t.t.wo;
        im.ho = t.t.ho;
        im.st = t.b.status;
        im.holes = t.b.holes;
        im.codes = t.b.codes;
#pragma unroll
        for (int k = 0; k < 4; ++k) im.scan[k] = t.b.scan[k];
        im.sources = t.t.rescale ? t.b.psrc : t.dbg.inpaint_source;
        im.seg = t.b.inpaint_seg;
        im.no_write = t.t.rescale;
        im.out_y = t.out_y;
        im.out_u = t.out_u;
        im.out_v = t.out_v;
        im.ties_up = t.t.chroma_ties_up;
        return im;
    }
};

// One image given directly (kernel parameter).
struct Direct {
    InpaintImage im;
    __device__ InpaintImage operator()() const { return im; }
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

__device__ __forceinline__ uint64_t pack_dxy(uint32_t d, int x, int y) {
    return ((uint64_t)d << 32) | ((uint64_t)(uint32_t)x << 16) | (uint64_t)(uint32_t)y;
}

__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) {
    return b < a ? b : a;
}

__device__ __forceinline__ unsigned long long warp_incl_min(unsigned long long v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = umin64(v, y);
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_incl_min_rev(unsigned long long v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o < 32) v = umin64(v, y);
    }
    return v;
}

// Sweep 0, rows (forward): R(p) = lexmin over q.x <= p.x of
// (C(q).d + p.x - q.x, C(q).src).  One warp per row of the region.
// Rows are scanned by one CTA each: 8 warps take 128-pixel segments in
// rounds of 8, exchange their segment minima through shared memory and scan
// with the minimum of every segment before them.  The keys carry the column
// bias, so a segment's minimum does not depend on where it is applied.
constexpr int ROW_WARPS = 8;
constexpr int SEG = 32 * CB;

template <class Src>
__global__ void __launch_bounds__(32 * ROW_WARPS) inpaint_row0_kernel(const __grid_constant__ Src src) {
    grid_dep_wait();
    const InpaintImage im = src();
    const int wo = im.wo, ho = im.ho;
    const DevStatus* __restrict__ st = im.st;
    const uint8_t* __restrict__ holes = im.holes;
    uint64_t* __restrict__ R = im.scan[0];
    __shared__ unsigned long long s_min[ROW_WARPS];
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int y = rg.y0 + (int)blockIdx.x;
    if (y > rg.y1) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint8_t* hr = holes + (size_t)y * wo;
    const uint8_t* hd = y + 1 < ho ? hr + wo : nullptr;
    const int nseg = (rg.x1 - rg.x0 + SEG) / SEG;
    unsigned long long round_carry = kEmptyKey;
    for (int seg0 = 0; seg0 < nseg; seg0 += ROW_WARPS) {
        const int base = rg.x0 + (seg0 + warp) * SEG;
        unsigned long long incl[CB];
        unsigned long long local = kEmptyKey;
#pragma unroll
        for (int c = 0; c < CB; ++c) {
            const int x = base + 32 * c + lane;
            unsigned long long key = kEmptyKey;
            if (x <= rg.x1) {
                uint32_t d = kInfD;
                int sx = x, sy = y;
                if (!hr[x]) {
                    d = 0;
                } else if (hd && !hd[x]) {
                    d = 1; sy = y + 1;
                } else if (x + 1 < wo && !hr[x + 1]) {
                    d = 1; sx = x + 1;
                }
                if (d != kInfD) key = pack_dxy((uint32_t)((int)d - x + kScanBias), sx, sy);
            }
            incl[c] = umin64(warp_incl_min(key, lane), local);
            local = __shfl_sync(0xffffffffu, incl[c], 31);
        }
        if (lane == 0) s_min[warp] = local;
        __syncthreads();
        unsigned long long carry = round_carry;
        for (int w2 = 0; w2 < warp; ++w2) carry = umin64(carry, s_min[w2]);
#pragma unroll
        for (int c = 0; c < CB; ++c) {
            const int x = base + 32 * c + lane;
            if (x > rg.x1) continue;
            const unsigned long long k = umin64(incl[c], carry);
            uint64_t out = ~0ull;
            if (k != kEmptyKey)
                out = pack_dxy((uint32_t)((int)(k >> 32) - kScanBias + x), (int)((k >> 16) & 0xffff),
                               (int)(k & 0xffff));
            R[(size_t)y * wo + x] = out;
        }
        for (int w2 = 0; w2 < ROW_WARPS; ++w2) round_carry = umin64(round_carry, s_min[w2]);
        __syncthreads();
    }
}

// Column scans: CTA = 32 columns x 32 row segments (one warp per segment).
// Phase 1 reduces each segment, phase 2 rescans it with the carry of the
// segments before it (above for forward scans, below for backward scans).

__device__ __forceinline__ unsigned long long col0_key(uint64_t r, int y) {
    if (r == ~0ull) return kEmptyKey;
    const int d = (int)(r >> 32);
    return pack_dxy((uint32_t)(d - y + kScanBias), (int)((r >> 16) & 0xffff), (int)(r & 0xffff));
}

// Sweep 0, columns (forward): D0, S0 (p) = lexmin over q.y <= p.y of
// (R(q).d + p.y - q.y, src).  Output packed (D0, S0) per pixel.
// Rows [gy0, gy1] of column group blockIdx.y of G, and the rows of warp w
// within them.
struct GroupRows {
    int yb, ye;
};
__device__ __forceinline__ GroupRows group_rows(const Region& rg, int G, int w) {
    const int nrows = rg.y1 - rg.y0 + 1;
    const int RG = (nrows + G - 1) / G;
    const int gy0 = rg.y0 + (int)blockIdx.y * RG, gy1 = min(rg.y1, gy0 + RG - 1);
    const int L = (max(0, gy1 - gy0 + 1) + 31) / 32;
    GroupRows r;
    r.yb = gy0 + w * L;
    r.ye = min(gy1, r.yb + L - 1);
    return r;
}

// The column-minima table of the pre-passes (G > 1): first every group's
// minima per strip (64 words: 32 lanes, and 32 more for the second key of
// the backward scan), then every warp segment's minima, 32 segments per
// group and strip, so that the scan passes need not re-read their own
// rows to find the carry from the segments before them.
__device__ __forceinline__ size_t seg_total(int g, int nstrips, int strip) {
    return ((size_t)g * nstrips + strip) * 64;
}
__device__ __forceinline__ size_t seg_warp(int G, int g, int nstrips, int strip, int w) {
    return (size_t)G * nstrips * 64 + (((size_t)g * nstrips + strip) * 32 + w) * 64;
}

// Grid (strips of 32 columns, G row groups, images).  With PRE the CTA only
// stores its group's and its warp segments' column minima; otherwise it
// scans its group starting from the minima of the groups and segments
// above it (recomputed from its own rows when G = 1).
template <class Src, bool PRE>
__global__ void __launch_bounds__(1024) inpaint_col0_kernel(const __grid_constant__ Src src, int G) {
    grid_dep_wait();
    const InpaintImage im = src();
    const int wo = im.wo, ho = im.ho;
    const DevStatus* __restrict__ st = im.st;
    const uint8_t* __restrict__ holes = im.holes;
    const uint64_t* __restrict__ R = im.scan[0];
    uint64_t* __restrict__ DS = im.scan[1];
    __shared__ unsigned long long seg[32][33];
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = rg.x0 + (int)blockIdx.x * 32 + lane;
    if (rg.x0 + (int)blockIdx.x * 32 > rg.x1) return;
    const int nstrips = (rg.x1 - rg.x0 + 32) / 32;
    const GroupRows gr = group_rows(rg, G, w);
    const int yb = gr.yb, ye = gr.ye;
    const bool col_ok = x <= rg.x1;
    unsigned long long run = kEmptyKey;
    if (PRE || G == 1) {
        unsigned long long m = kEmptyKey;
        if (col_ok)
            for (int y0 = yb; y0 <= ye; y0 += RB) {
                uint64_t r[RB];
#pragma unroll
                for (int k = 0; k < RB; ++k) r[k] = y0 + k <= ye ? R[(size_t)(y0 + k) * wo + x] : ~0ull;
#pragma unroll
                for (int k = 0; k < RB; ++k) m = umin64(m, col0_key(r[k], y0 + k));
            }
        seg[w][lane] = m;
        __syncthreads();
        if (PRE) {
            im.seg[seg_warp(G, blockIdx.y, nstrips, blockIdx.x, w) + lane] = m;
            if (w == 0) {
                unsigned long long t = kEmptyKey;
                for (int s = 0; s < 32; ++s) t = umin64(t, seg[s][lane]);
                im.seg[seg_total(blockIdx.y, nstrips, blockIdx.x) + lane] = t;
            }
            return;
        }
        for (int s = 0; s < w; ++s) run = umin64(run, seg[s][lane]);
    } else {
        const uint64_t* sw = im.seg + seg_warp(G, blockIdx.y, nstrips, blockIdx.x, 0);
        for (int s = 0; s < w; ++s) run = umin64(run, sw[s * 64 + lane]);
    }
    for (int g = 0; g < (int)blockIdx.y; ++g) run = umin64(run, im.seg[seg_total(g, nstrips, blockIdx.x) + lane]);
    if (!col_ok) return;
    const uint32_t big = (uint32_t)(wo + ho);
    for (int y0 = yb; y0 <= ye; y0 += RB) {
        uint64_t r[RB];
        uint8_t h[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) {
            const bool ok = y0 + k <= ye;
            r[k] = ok ? R[(size_t)(y0 + k) * wo + x] : ~0ull;
            h[k] = ok ? holes[(size_t)(y0 + k) * wo + x] : 0;
        }
#pragma unroll
        for (int k = 0; k < RB; ++k) {
            const int y = y0 + k;
            if (y > ye) break;
            run = umin64(run, col0_key(r[k], y));
            uint64_t out;
            if (!h[k])
                out = pack_dxy(0, x, y);
            else if (run == kEmptyKey)
                out = pack_dxy(big, x, y);
            else
                out = pack_dxy((uint32_t)((int)(run >> 32) - kScanBias + y), (int)((run >> 16) & 0xffff),
                               (int)(run & 0xffff));
            DS[(size_t)y * wo + x] = out;
        }
    }
}

// Packed (D0, S0) of pixel (x, y), or (0, itself) outside the region (a
// non-hole: every hole lies inside the region).
__device__ __forceinline__ uint64_t ds_at(const uint64_t* DS, const Region& rg, int wo, int x, int y) {
    if (x < rg.x0 || x > rg.x1 || y < rg.y0 || y > rg.y1) return pack_dxy(0, x, y);
    return DS[(size_t)y * wo + x];
}

// Sweep 1 seeds of region pixel (x, y): T(q) = best of stay (D0(q), S0(q)),
// left (D0+1, S0 of left), up (D0+1, S0 of up) with priority stay > left >
// up; T'(q) the same without stay.  Non-holes: (0, q).  Stores both and
// returns T(q).  `self`, `left` and `up` are the (D0, S0) words of the
// pixel and its neighbours (ds_at), read by the caller for a hole only.
__device__ __forceinline__ uint64_t seed1_from(bool hole, uint64_t self, uint64_t left, uint64_t up,
                                               uint64_t* __restrict__ Tq, uint64_t* __restrict__ Tp, int x, int y,
                                               size_t o) {
    if (!hole) {
        const uint64_t own = pack_dxy(0, x, y);
        Tq[o] = own;
        Tp[o] = own;
        return own;
    }
    uint64_t best = self;
    uint64_t bp = ~0ull;
    if (x > 0) {
        const uint64_t c = left + (1ull << 32);
        if ((c >> 32) < (best >> 32)) best = c;
        bp = c;
    }
    if (y > 0) {
        const uint64_t c = up + (1ull << 32);
        if ((c >> 32) < (best >> 32)) best = c;
        if (bp == ~0ull || (c >> 32) < (bp >> 32)) bp = c;
    }
    Tq[o] = best;
    Tp[o] = bp;
    return best;
}

// Sweep 1, rows (backward, exclusive): RR(x, y) = min over q.x > x of
// (T(q).d + q.x, q.x), with the seeds T, T' computed (and stored for the
// column pass and the fill) as the row reads them.  One CTA per row.
template <class Src>
__global__ void __launch_bounds__(32 * ROW_WARPS) inpaint_row1_kernel(const __grid_constant__ Src src) {
    grid_dep_wait();
    const InpaintImage im = src();
    const int wo = im.wo, ho = im.ho;
    const DevStatus* __restrict__ st = im.st;
    const uint8_t* __restrict__ holes = im.holes;
    const uint64_t* __restrict__ DS = im.scan[1];
    uint64_t* __restrict__ Tq = im.scan[2];
    uint64_t* __restrict__ Tp = im.scan[3];
    uint64_t* __restrict__ RR = im.scan[0];
    __shared__ unsigned long long s_min[ROW_WARPS];
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int y = rg.y0 + (int)blockIdx.x;
    if (y > rg.y1) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nseg = (rg.x1 - rg.x0 + SEG) / SEG;
    unsigned long long round_carry = kEmptyKey;
    // Segments run from the right end; within a chunk lane 31 holds the
    // rightmost pixel.
    for (int seg0 = 0; seg0 < nseg; seg0 += ROW_WARPS) {
        const int base = (seg0 + warp) * SEG;
        unsigned long long excl[CB];
        unsigned long long local = kEmptyKey;
        // The chunks' hole flags, then the words their seeds read, before
        // any arithmetic: the dependent loads of the CB chunks overlap.
        bool hole[CB];
        uint64_t self[CB], left[CB], up[CB];
#pragma unroll
        for (int c = 0; c < CB; ++c) {
            const int x = rg.x1 - (base + 32 * c + (31 - lane));
            hole[c] = x >= rg.x0 && holes[(size_t)y * wo + x];
        }
#pragma unroll
        for (int c = 0; c < CB; ++c) {
            const int x = rg.x1 - (base + 32 * c + (31 - lane));
            self[c] = left[c] = up[c] = 0;
            if (hole[c]) {
                self[c] = DS[(size_t)y * wo + x];
                if (x > 0) left[c] = ds_at(DS, rg, wo, x - 1, y);
                if (y > 0) up[c] = ds_at(DS, rg, wo, x, y - 1);
            }
        }
#pragma unroll
        for (int c = 0; c < CB; ++c) {
            const int x = rg.x1 - (base + 32 * c + (31 - lane));
            unsigned long long key = kEmptyKey;
            if (x >= rg.x0) {
                const uint64_t t = seed1_from(hole[c], self[c], left[c], up[c], Tq, Tp, x, y, (size_t)y * wo + x);
                key = ((unsigned long long)((t >> 32) + (uint64_t)x) << 16) | (unsigned long long)x;
            }
            const unsigned long long incl = umin64(warp_incl_min_rev(key, lane), local);
            unsigned long long e = __shfl_down_sync(0xffffffffu, incl, 1);
            if (lane == 31) e = local;
            excl[c] = e;
            local = __shfl_sync(0xffffffffu, incl, 0);
        }
        if (lane == 0) s_min[warp] = local;
        __syncthreads();
        unsigned long long carry = round_carry;
        for (int w2 = 0; w2 < warp; ++w2) carry = umin64(carry, s_min[w2]);
#pragma unroll
        for (int c = 0; c < CB; ++c) {
            const int x = rg.x1 - (base + 32 * c + (31 - lane));
            if (x >= rg.x0) RR[(size_t)y * wo + x] = umin64(excl[c], carry);
        }
        for (int w2 = 0; w2 < ROW_WARPS; ++w2) round_carry = umin64(round_carry, s_min[w2]);
        __syncthreads();
    }
}

// Sweep 1, columns (backward): for each hole p choose its sweep-1 source
// and copy that pixel's codes (the fill of inpaint_color,
// inpainting.cpp:191-198).
template <class Src, bool PRE>
__global__ void __launch_bounds__(1024) inpaint_col1_kernel(const __grid_constant__ Src src, int G) {
    grid_dep_wait();
    const InpaintImage im = src();
    const int wo = im.wo, ho = im.ho;
    const DevStatus* __restrict__ st = im.st;
    uint64_t* __restrict__ codes = im.codes;
    const uint8_t* __restrict__ holes = im.holes;
    uint64_t* __restrict__ DS = im.scan[1];
    const uint64_t* __restrict__ Tq = im.scan[2];
    const uint64_t* __restrict__ Tp = im.scan[3];
    const uint64_t* __restrict__ RR = im.scan[0];
    __shared__ unsigned long long seg_col[32][33];
    __shared__ unsigned long long seg_off[32][33];
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = rg.x0 + (int)blockIdx.x * 32 + lane;
    if (rg.x0 + (int)blockIdx.x * 32 > rg.x1) return;
    const bool col_ok = x <= rg.x1;
    const int nstrips = (rg.x1 - rg.x0 + 32) / 32;
    const GroupRows gr = group_rows(rg, G, w);
    const int yb = gr.yb, ye = gr.ye;
    // Keys: column part (T.d + y) << 16 | y (minimum y on ties);
    //       off-column (RR.d - x + y) << 32 | (0xffff - y) << 16 | qx
    //       (largest y, then smallest x on ties).
    auto col_key = [&](uint64_t t, int y) -> unsigned long long {
        return ((unsigned long long)((t >> 32) + (uint64_t)y) << 16) | (unsigned long long)y;
    };
    auto off_key = [&](uint64_t r, int y) -> unsigned long long {
        if (r == kEmptyKey) return kEmptyKey;
        const uint64_t v = (r >> 16) - (uint64_t)x + (uint64_t)y;
        return (v << 32) | ((uint64_t)(0xffff - y) << 16) | (r & 0xffff);
    };
    unsigned long long run_c = kEmptyKey, run_o = kEmptyKey;
    if (PRE || G == 1) {
        unsigned long long mc = kEmptyKey, mo = kEmptyKey;
        if (col_ok)
            for (int y0 = yb; y0 <= ye; y0 += RB) {
                uint64_t t[RB], r[RB];
#pragma unroll
                for (int k = 0; k < RB; ++k) {
                    const bool ok = y0 + k <= ye;
                    t[k] = ok ? Tq[(size_t)(y0 + k) * wo + x] : ~0ull;
                    r[k] = ok ? RR[(size_t)(y0 + k) * wo + x] : ~0ull;
                }
#pragma unroll
                for (int k = 0; k < RB; ++k) {
                    if (y0 + k > ye) break;
                    mc = umin64(mc, col_key(t[k], y0 + k));
                    mo = umin64(mo, off_key(r[k], y0 + k));
                }
            }
        seg_col[w][lane] = mc;
        seg_off[w][lane] = mo;
        __syncthreads();
        if (PRE) {
            uint64_t* own = im.seg + seg_warp(G, blockIdx.y, nstrips, blockIdx.x, w);
            own[lane] = mc;
            own[32 + lane] = mo;
            if (w == 0) {
                unsigned long long tc = kEmptyKey, to = kEmptyKey;
                for (int s = 0; s < 32; ++s) {
                    tc = umin64(tc, seg_col[s][lane]);
                    to = umin64(to, seg_off[s][lane]);
                }
                uint64_t* dst = im.seg + seg_total(blockIdx.y, nstrips, blockIdx.x);
                dst[lane] = tc;
                dst[32 + lane] = to;
            }
            return;
        }
        for (int s = w + 1; s < 32; ++s) {
            run_c = umin64(run_c, seg_col[s][lane]);
            run_o = umin64(run_o, seg_off[s][lane]);
        }
    } else {
        const uint64_t* sw = im.seg + seg_warp(G, blockIdx.y, nstrips, blockIdx.x, 0);
        for (int s = w + 1; s < 32; ++s) {
            run_c = umin64(run_c, sw[s * 64 + lane]);
            run_o = umin64(run_o, sw[s * 64 + 32 + lane]);
        }
    }
    for (int g = (int)blockIdx.y + 1; g < G; ++g) {
        const uint64_t* src_seg = im.seg + seg_total(g, nstrips, blockIdx.x);
        run_c = umin64(run_c, src_seg[lane]);
        run_o = umin64(run_o, src_seg[32 + lane]);
    }
    if (!col_ok) return;
    // Bottom-up over the segment in batches of RB1 rows; every word a row
    // needs (the holes' own T' and D0/S0 too) is loaded with the batch, so
    // nothing on the serial chain below waits for memory.
    for (int y1 = ye; y1 >= yb; y1 -= RB1) {
        uint64_t t[RB1], r[RB1], tpk[RB1], dsk[RB1];
        uint8_t h[RB1];
#pragma unroll
        for (int k = 0; k < RB1; ++k) {
            const int y = y1 - k;
            const bool ok = y >= yb;
            const size_t o = (size_t)y * wo + x;
            t[k] = ok ? Tq[o] : ~0ull;
            r[k] = ok ? RR[o] : ~0ull;
            h[k] = ok ? holes[o] : 0;
            tpk[k] = ok ? Tp[o] : 0ull;
            dsk[k] = ok ? DS[o] : 0ull;
        }
#pragma unroll
        for (int k = 0; k < RB1; ++k) {
            const int y = y1 - k;
            if (y < yb) break;
            // run_c holds the exclusive (rows below) column minimum here.
            run_o = umin64(run_o, off_key(r[k], y));
            if (h[k]) {
                const size_t o = (size_t)y * wo + x;
                const uint64_t tp = tpk[k];
                const uint64_t ds = dsk[k];
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
                const uint64_t d0 = ds >> 32;
                // The choice: the source itself (stay: S0; own seed T'), or
                // the seed T(q) of the column or off-column minimum.
                uint64_t choice = ds & 0xffffffffull;
                if (c_cost <= o_cost) {
                    if (c_cost < d0)
                        choice = (c_y == y) ? (tp & 0xffffffffull)
                                            : kSeedRef | ((uint64_t)x << 16) | (uint64_t)c_y;
                } else {
                    if (o_cost < d0) choice = kSeedRef | ((uint64_t)o_x << 16) | (uint64_t)o_y;
                }
                DS[o] = choice;
            }
            run_c = umin64(run_c, col_key(t[k], y));
        }
    }
}

// The fill of inpaint_color (inpainting.cpp:191-198) for the 2x2 blocks of
// the region that hold at least one hole: each hole follows its recorded
// choice to its source and takes the source's codes (written back for the
// passes that read them later: the resize of Precision != 1, the auxiliary
// outputs, the source list); then, unless the resize writes the output,
// the block's Y/U/V samples are written.  Sources are never holes, so the
// codes read here are never the ones written.
template <class Src>
__global__ void inpaint_write_kernel(const __grid_constant__ Src src) {
    grid_dep_wait();
    const InpaintImage im = src();
    const int wo = im.wo, ho = im.ho;
    const DevStatus* __restrict__ st = im.st;
    uint64_t* __restrict__ codes = im.codes;
    const uint64_t* __restrict__ DS = im.scan[1];
    const uint64_t* __restrict__ Tq = im.scan[2];
    int32_t* __restrict__ sources = im.sources;
    uint16_t* __restrict__ out_y = im.out_y;
    uint16_t* __restrict__ out_u = im.out_u;
    uint16_t* __restrict__ out_v = im.out_v;
    const int ties_up = im.ties_up;
    const Region rg = hole_region(st, wo, ho);
    if (rg.empty) return;
    const int bx0 = rg.x0 / 2, by0 = rg.y0 / 2;
    const int x = 2 * (bx0 + (int)(blockIdx.x * blockDim.x + threadIdx.x));
    const int y = 2 * (by0 + (int)blockIdx.y);
    if (x > rg.x1 || y > rg.y1 || x >= wo || y >= ho) return;
    const size_t o = (size_t)y * wo + x;
    // A raster of odd width or height (Precision != 1) ends in partial
    // blocks: their missing pixels read as non-holes and are not written.
    const bool has_r = x + 1 < wo, has_b = y + 1 < ho;
    uint64_t c00 = codes[o], c01 = has_r ? codes[o + 1] : 0ull, c10 = has_b ? codes[o + wo] : 0ull,
             c11 = has_r && has_b ? codes[o + wo + 1] : 0ull;
    if (!((c00 | c01 | c10 | c11) & kHoleBit)) return;
    auto fill = [&](uint64_t& c, size_t q) {
        if (!(c & kHoleBit)) return;
        uint64_t w = DS[q];
        if (w & kSeedRef) w = Tq[(size_t)(w & 0xffff) * wo + ((w >> 16) & 0xffff)];
        const int sx = (int)((w >> 16) & 0xffff), sy = (int)(w & 0xffff);
        c = (codes[(size_t)sy * wo + sx] & kCodeMask) | kHoleBit;
        codes[q] = c;
        if (sources) {
            sources[q * 2 + 0] = sx;
            sources[q * 2 + 1] = sy;
        }
    };
    fill(c00, o);
    if (has_r) fill(c01, o + 1);
    if (has_b) fill(c10, o + wo);
    if (has_r && has_b) fill(c11, o + wo + 1);
    if (im.no_write) return;
    out_y[o] = (uint16_t)(c00 & 0xffff);
    out_y[o + 1] = (uint16_t)(c01 & 0xffff);
    out_y[o + wo] = (uint16_t)(c10 & 0xffff);
    out_y[o + wo + 1] = (uint16_t)(c11 & 0xffff);
    const size_t co = (size_t)(y / 2) * (wo / 2) + x / 2;
    const uint32_t su = (uint32_t)((c00 >> 16) & 0xffff) + ((c01 >> 16) & 0xffff) + ((c10 >> 16) & 0xffff) +
                        ((c11 >> 16) & 0xffff);
    const uint32_t sv = (uint32_t)((c00 >> 32) & 0xffff) + ((c01 >> 32) & 0xffff) + ((c10 >> 32) & 0xffff) +
                        ((c11 >> 32) & 0xffff);
    out_u[co] = quarter_round(su, ties_up);
    out_v[co] = quarter_round(sv, ties_up);
}

// The scan passes of `src` (grid z = images), sized for max_w x max_h.
// The column passes split each 32-column strip into G row groups (one CTA
// each) when the strips alone would not fill the device; a pre-pass then
// stores every group's column minima.
template <class Src>
int launch_scans(const Src& src, int max_w, int max_h, int images, int G, cudaStream_t s) {
    const int strips = (max_w + 31) / 32;
    int launches = 0;
    launch_dependent(inpaint_row0_kernel<Src>, dim3(max_h, 1, images), dim3(32 * ROW_WARPS), 0, s, src);
    if (G > 1) launch_dependent(inpaint_col0_kernel<Src, true>, dim3(strips, G, images), dim3(1024), 0, s, src, G);
    launch_dependent(inpaint_col0_kernel<Src, false>, dim3(strips, G, images), dim3(1024), 0, s, src, G);
    launch_dependent(inpaint_row1_kernel<Src>, dim3(max_h, 1, images), dim3(32 * ROW_WARPS), 0, s, src);
    if (G > 1) launch_dependent(inpaint_col1_kernel<Src, true>, dim3(strips, G, images), dim3(1024), 0, s, src, G);
    launch_dependent(inpaint_col1_kernel<Src, false>, dim3(strips, G, images), dim3(1024), 0, s, src, G);
    launches = 4 + (G > 1 ? 2 : 0);
    return launches;
}

// Row groups per strip for the column passes.
// The column kernels hold one 1024-thread CTA per SM (their registers), so
// the groups are sized for one wave: a second, partial wave would cost as
// much as the first.
int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 148;
    }
    return n;
}

int column_groups(int max_w, int images) {
    static const int sms = sm_count();
    const int strips = (max_w + 31) / 32;
    return std::max(1, std::min(INPAINT_MAX_GROUPS, sms / (strips * images)));
}

}  // namespace

size_t inpaint_seg_words(int wo) {
    // The most row groups any launch with an output this wide can use (one
    // image); the table is unused with one group.
    const int G = column_groups(wo, 1);
    return G > 1 ? (size_t)G * ((wo + 31) / 32) * 64 * 33 : 1;
}

template <class Tabs>
int launch_inpaint(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    const FromTables<Tabs> src{tabs};
    const int n = launch_scans(src, sh.max_wo, sh.max_ho, sh.slots, column_groups(sh.max_wo, sh.slots), s);
    launch_dependent(inpaint_write_kernel<FromTables<Tabs>>, dim3(((sh.max_wo + 1) / 2 + 127) / 128, (sh.max_ho + 1) / 2, sh.slots),
                     dim3(128), 0, s, src);
    return n + 1;
}

template int launch_inpaint<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template int launch_inpaint<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

void launch_inpaint_scans(DevStatus* st, const uint8_t* holes, uint64_t* codes, uint64_t* const scan[4], int w,
                          int h, int32_t* sources, cudaStream_t s) {
    Direct src;
    src.im.wo = w;
    src.im.ho = h;
    src.im.st = st;
    src.im.holes = holes;
    src.im.codes = codes;
    for (int k = 0; k < 4; ++k) src.im.scan[k] = scan[k];
    src.im.sources = sources;
    src.im.seg = nullptr;
    src.im.out_y = src.im.out_u = src.im.out_v = nullptr;
    src.im.ties_up = 0;
    src.im.no_write = 1;
    launch_scans(src, w, h, 1, 1, s);
    launch_dependent(inpaint_write_kernel<Direct>, dim3((w / 2 + 127) / 128, (h + 1) / 2, 1), dim3(128), 0, s, src);
}

}  // namespace rvsb
