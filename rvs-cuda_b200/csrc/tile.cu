// Tile stage: raster + resolve + blend + quantise, one CTA per output tile.
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

constexpr int VG = 4;          // views whose z-buffers are in shared memory at once
constexpr int SMALL = 4;       // triangles with more candidate pixels go warp-cooperative
constexpr int NWARPS = TILE_THREADS / 32;
constexpr int QUADS = BLOCK_W * BLOCK_H;
static_assert(QUADS == 32, "one warp per binning block");

// Candidate pixel (x, y) of a set-up triangle: the coverage test of
// transform.cpp:105-114; on success the fragment key goes to the z-buffer.
// The CPU keeps, per output pixel, the fragment with the largest
// quality / depth^3 (a later fragment replaces the stored one iff
// (d/D)^3 * Q < q, transform.cpp:119-142), the earliest in scan order on
// ties.  The key holds the bits of depth^3 / quality (smaller is better)
// above the triangle's scan index, so 64-bit atomicMin keeps that winner
// whatever the scheduling order.
//
// The first two tests use the exact numerator threshold (no division).  The
// third, l3 = (1 - l1) - l2 >= -1e-6, is evaluated with l1, l2 from the
// correctly rounded reciprocal of den; B bounds the difference to the
// CPU's l3 (relative errors: 3 ulp on l1 and l2, one rounding per
// subtraction), and only a value within B of the threshold is recomputed
// with the reference's divisions.  The depth in the key uses the
// reciprocal-based coordinates; the resolve recomputes the winner exactly.
__device__ __forceinline__ bool test_pixel(const TriSetup& s, float cx, float cy, float za, float zb_, float zc,
                                           int x, int y, float& d) {
    const float tx = __fsub_rn(__fadd_rn((float)x, 0.5f), cx);
    const float ty = __fsub_rn(__fadd_rn((float)y, 0.5f), cy);
    const float n1 = __fadd_rn(__fmul_rn(s.b1c1, tx), __fmul_rn(s.c0b0, ty));
    const float n2 = __fadd_rn(__fmul_rn(s.c1a1, tx), __fmul_rn(s.a0c0, ty));
    if (!(n1 >= s.tn && n2 >= s.tn)) return false;
    float l1 = __fmul_rn(n1, s.rinv), l2 = __fmul_rn(n2, s.rinv);
    const float a = __fsub_rn(1.f, l1);
    float l3 = __fsub_rn(a, l2);
    const float eps = 1e-6f;
    const float B = 5.9604645e-8f * (4.f * fabsf(l1) + 3.f * fabsf(a) + 4.f * fabsf(l2) + 3.f * fabsf(l3));
    if (!(l3 - B >= -eps)) {
        if (l3 + B < -eps) return false;
        l1 = __fdiv_rn(n1, s.den);
        l2 = __fdiv_rn(n2, s.den);
        l3 = __fsub_rn(__fsub_rn(1.f, l1), l2);
        if (!(l3 >= -eps)) return false;
    }
    d = interp(za, zb_, zc, l1, l2, l3);
    return !isnan(d);
}

__device__ __forceinline__ unsigned long long frag_key(float d, float invq, uint32_t tri) {
    uint32_t hi = 0u;
    if (d > 0.f) hi = __float_as_uint(__fmul_rn(__fmul_rn(__fmul_rn(d, d), d), invq));
    return ((unsigned long long)hi << 32) | tri;
}

// Rasterises the triangles of the 32 quads of binning block `b` of view V
// (one quad per lane) into the tile's z-buffer `zb`: transform.cpp:159-176.
__device__ __forceinline__ void raster_block(const DevView& V, int wo, int ho, bool wrap, double lambda_mid, int b,
                                             int tx0, int ty0, unsigned long long* zb, int lane) {
    const int bx = b % V.nbx, by = b / V.nbx;
    const int i = by * BLOCK_H + lane / BLOCK_W, j = bx * BLOCK_W + lane % BLOCK_W;
    const bool quad_ok = i < V.h - 1 && j < V.w - 1;
    float4 v00, v01, v10, v11, w0, w1;
    bool cond0 = false;
    if (quad_ok) {
        const size_t r0 = (size_t)i * V.w, r1 = r0 + V.w;
        v01 = V.vert[r0 + j + 1];
        v10 = V.vert[r1 + j];
        cond0 = v01.z > 0.f && v10.z > 0.f && v01.x > 0.f && v10.x > 0.f;
        if (cond0) {
            v00 = V.vert[r0 + j];
            v11 = V.vert[r1 + j + 1];
            if (wrap && j == 0) {
                w0 = V.vert[r0 + V.w - 1];
                w1 = V.vert[r1 + V.w - 1];
            }
        }
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
            case 2: A = w0; B = v00; C = w1; active = active && j == 0; break;
            default: A = v10; B = w1; C = v00; active = active && j == 0; break;
        }
        TriSetup s;
        int count = 0;
        if (active && tri_coef(A, B, C, s) &&
            tri_range(A, B, C, wo, ho, tx0, tx0 + TILE - 1, ty0, ty0 + TILE - 1, s)) {
            count = (s.x1 - s.x0 + 1) * (s.y1 - s.y0 + 1);
            s.tn = coverage_threshold(s.den, lambda_mid);
            s.rinv = __frcp_rn(s.den);
        }
        const uint32_t tri = quad * 4u + (uint32_t)slot;
        const bool big = count > SMALL;
        if (count > 0 && !big) {
            float invq = -1.f;
            for (int y = s.y0; y <= s.y1; ++y)
                for (int x = s.x0; x <= s.x1; ++x) {
                    float d;
                    if (!test_pixel(s, C.x, C.y, A.z, B.z, C.z, x, y, d)) continue;
                    if (invq < 0.f) invq = __frcp_rn(tri_quality(A.x, A.y, B.x, B.y, C.x, C.y));
                    atomicMin(&zb[(y - ty0) * TILE + (x - tx0)], frag_key(d, invq, tri));
                }
        }
        unsigned mask = __ballot_sync(0xffffffffu, big);
        if (!mask) continue;
        float invq_own = 0.f;
        if (big) invq_own = __frcp_rn(tri_quality(A.x, A.y, B.x, B.y, C.x, C.y));
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            TriSetup t;
            t.b1c1 = __shfl_sync(0xffffffffu, s.b1c1, src);
            t.c0b0 = __shfl_sync(0xffffffffu, s.c0b0, src);
            t.c1a1 = __shfl_sync(0xffffffffu, s.c1a1, src);
            t.a0c0 = __shfl_sync(0xffffffffu, s.a0c0, src);
            t.den = __shfl_sync(0xffffffffu, s.den, src);
            t.tn = __shfl_sync(0xffffffffu, s.tn, src);
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
            // One lane per row of the (tile-clipped) range: at most TILE rows.
            const int y = t.y0 + lane;
            if (y <= t.y1) {
                int xl, xr;
                row_span(t, cx, cy, y, xl, xr);
                for (int x = xl; x <= xr; ++x) {
                    float d;
                    if (!test_pixel(t, cx, cy, za, zb_, zc, x, y, d)) continue;
                    atomicMin(&zb[(y - ty0) * TILE + (x - tx0)], frag_key(d, invq, ttri));
                }
            }
        }
    }
}

struct Fragment {
    float3 col;
    float depth;      // +inf when uncovered
    float validity;   // triangle quality, 0 when uncovered
};

// Re-evaluates the winning triangle at pixel (x, y) exactly as the CPU's
// colorize_triangle does for the fragment it keeps (transform.cpp:109-135).
__device__ Fragment resolve(const DevView& V, unsigned long long key, int x, int y) {
    Fragment f;
    f.col = make_float3(0.f, 0.f, 0.f);
    f.depth = INFINITY;
    f.validity = 0.f;
    if (key == kEmptyKey) return f;
    const uint32_t tri = (uint32_t)(key & 0xffffffffull);
    const int t = (int)(tri & 3u);
    const int i = (int)(tri >> V.tri_shift), j = (int)((tri >> 2) & ((1u << (V.tri_shift - 2)) - 1u));
    int ax, ay, bx, by, cx, cy;
    tri_vertices(V.w, i, j, t, ax, ay, bx, by, cx, cy);
    const float4 A = V.vert[(size_t)ay * V.w + ax];
    const float4 B = V.vert[(size_t)by * V.w + bx];
    const float4 C = V.vert[(size_t)cy * V.w + cx];
    TriSetup s;
    s.b1c1 = __fsub_rn(B.y, C.y);
    s.a0c0 = __fsub_rn(A.x, C.x);
    s.c0b0 = __fsub_rn(C.x, B.x);
    s.c1a1 = __fsub_rn(C.y, A.y);
    s.den = __fadd_rn(__fmul_rn(s.b1c1, s.a0c0), __fmul_rn(s.c0b0, __fsub_rn(A.y, C.y)));
    float l1, l2, l3;
    barycentric(s, C.x, C.y, x, y, l1, l2, l3);
    const float3 ca = input_color(V, ax, ay), cb = input_color(V, bx, by), cc = input_color(V, cx, cy);
    f.col.x = interp(ca.x, cb.x, cc.x, l1, l2, l3);
    f.col.y = interp(ca.y, cb.y, cc.y, l1, l2, l3);
    f.col.z = interp(ca.z, cb.z, cc.z, l1, l2, l3);
    f.depth = interp(A.z, B.z, C.z, l1, l2, l3);
    f.validity = tri_quality(A.x, A.y, B.x, B.y, C.x, C.y);
    return f;
}

// Grid: one CTA per TILE x TILE output tile.  Views are processed in groups
// of VG in blend order: clear the group's shared z-buffers, rasterise every
// binned block of the group (one warp per block), then resolve each pixel's
// winners view by view and fold them into the running blend
// (BlendedViewSimple::blendBasicMode + blend_img, BlendedView.cpp:180-212,
// blending.cpp:310-369).  Finally quantise, write the 2x2 blocks without
// holes and leave packed codes for the inpainting passes.
__global__ void __launch_bounds__(TILE_THREADS, 3) tile_kernel(
    const __grid_constant__ ViewTable tab, const int* __restrict__ counts,
    const int* __restrict__ offsets, const int* __restrict__ list, DevStatus* __restrict__ st,
    uint64_t* __restrict__ codes, uint16_t* __restrict__ out_y, uint16_t* __restrict__ out_u,
    uint16_t* __restrict__ out_v, DebugPtrs dbg) {
    __shared__ unsigned long long zb[VG][TILE * TILE];
    __shared__ int s_pref[VG + 1];
    __shared__ int s_hole_box[4];
    const DevTarget& T = tab.t;
    const int tile = blockIdx.x;
    const int tx0 = (tile % T.ntx) * TILE, ty0 = (tile / T.ntx) * TILE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool overflow = st->bin_overflow != 0;
    const bool wrap = T.wrap != 0;
    constexpr int PPT = TILE * TILE / TILE_THREADS;  // pixels per thread
    float acc_c[PPT][3];
    float acc_q[PPT];
    const size_t npo = (size_t)T.wo * T.ho;

    for (int g0 = 0; g0 < T.n_views; g0 += VG) {
        const int gn = min(VG, T.n_views - g0);
        for (int k = tid; k < gn * TILE * TILE; k += TILE_THREADS) zb[k / (TILE * TILE)][k % (TILE * TILE)] = kEmptyKey;
        if (tid == 0) {
            int run = 0;
            for (int k = 0; k < gn; ++k) {
                s_pref[k] = run;
                const DevView& V = tab.v[g0 + k];
                run += overflow ? V.nbx * V.nby : counts[tile * T.n_views + g0 + k];
            }
            s_pref[gn] = run;
        }
        __syncthreads();
        const int E = s_pref[gn];
        for (int e = warp; e < E; e += NWARPS) {
            int k = 0;
            while (k + 1 < gn && e >= s_pref[k + 1]) ++k;
            const int v = g0 + k;
            const DevView& V = tab.v[v];
            int b;
            if (!overflow) {
                b = list[offsets[tile * T.n_views + v] + (e - s_pref[k])];
            } else {
                b = e - s_pref[k];
                const int4 bb = V.bbox[b];
                if (bb.x > bb.z || bb.z < tx0 || bb.x > tx0 + TILE - 1 || bb.w < ty0 || bb.y > ty0 + TILE - 1)
                    continue;
            }
            raster_block(V, T.wo, T.ho, wrap, T.lambda_mid, b, tx0, ty0, zb[k], lane);
        }
        __syncthreads();
        for (int k = 0; k < gn; ++k) {
            const int v = g0 + k;
            const DevView& V = tab.v[v];
#pragma unroll
            for (int pp = 0; pp < PPT; ++pp) {
                const int p = tid + pp * TILE_THREADS;
                const int x = tx0 + (p & (TILE - 1)), y = ty0 + p / TILE;
                if (x >= T.wo || y >= T.ho) continue;
                const Fragment f = resolve(V, zb[k][p], x, y);
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
                    acc_c[pp][0] = f.col.x; acc_c[pp][1] = f.col.y; acc_c[pp][2] = f.col.z;
                    acc_q[pp] = qv;
                } else {
                    // blend_img over {accumulator, new view}: weights quality^exp
                    // for quality > 0, colour * (1 / sum), quality = sum^(1/exp).
                    // acc_q holds the first view's quality after view 0 and the
                    // weight sum afterwards: the reference re-powers its stored
                    // quality sum^(1/exp) by exp, which returns the sum up to a
                    // few ulp, and quality > 0 exactly when the sum is > 0.
                    float sum = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
                    if (acc_q[pp] > 0.f) {
                        const float w = v == 1 ? blend_pow(acc_q[pp], T.blend_exp, T.blend_exp_int) : acc_q[pp];
                        sum = __fadd_rn(sum, w);
                        c0 = __fadd_rn(c0, __fmul_rn(w, acc_c[pp][0]));
                        c1 = __fadd_rn(c1, __fmul_rn(w, acc_c[pp][1]));
                        c2 = __fadd_rn(c2, __fmul_rn(w, acc_c[pp][2]));
                    }
                    if (qv > 0.f) {
                        const float w = blend_pow(qv, T.blend_exp, T.blend_exp_int);
                        sum = __fadd_rn(sum, w);
                        c0 = __fadd_rn(c0, __fmul_rn(w, f.col.x));
                        c1 = __fadd_rn(c1, __fmul_rn(w, f.col.y));
                        c2 = __fadd_rn(c2, __fmul_rn(w, f.col.z));
                    }
                    if (sum == 0.f) {
                        acc_c[pp][0] = 0.f; acc_c[pp][1] = 1.f; acc_c[pp][2] = 0.f;
                        acc_q[pp] = 0.f;
                    } else {
                        const float inv = __frcp_rn(sum);
                        acc_c[pp][0] = __fmul_rn(c0, inv);
                        acc_c[pp][1] = __fmul_rn(c1, inv);
                        acc_c[pp][2] = __fmul_rn(c2, inv);
                        acc_q[pp] = sum;
                    }
                }
            }
        }
        __syncthreads();
    }

    // Quantise into packed codes (Y | U << 16 | V << 32 | hole << 48).
    unsigned long long* codes_s = zb[0];
#pragma unroll
    for (int pp = 0; pp < PPT; ++pp) {
        const int p = tid + pp * TILE_THREADS;
        const int x = tx0 + (p & (TILE - 1)), y = ty0 + p / TILE;
        uint64_t code = 0;
        if (x < T.wo && y < T.ho) {
            const bool hole = !(acc_q[pp] > 0.f);
            code = (uint64_t)quantize(acc_c[pp][0], T.max_val) | ((uint64_t)quantize(acc_c[pp][1], T.max_val) << 16) |
                   ((uint64_t)quantize(acc_c[pp][2], T.max_val) << 32) | (hole ? kHoleBit : 0ull);
            const size_t o = (size_t)y * T.wo + x;
            if (dbg.blend_color) {
                dbg.blend_color[o * 3 + 0] = acc_c[pp][0];
                dbg.blend_color[o * 3 + 1] = acc_c[pp][1];
                dbg.blend_color[o * 3 + 2] = acc_c[pp][2];
            }
            if (dbg.blend_quality)
                dbg.blend_quality[o] = (T.n_views == 1 || !(acc_q[pp] > 0.f)) ? acc_q[pp] : powf(acc_q[pp], T.inv_blend_exp);
            if (dbg.inpaint_source) {
                dbg.inpaint_source[o * 2 + 0] = x;
                dbg.inpaint_source[o * 2 + 1] = y;
            }
        }
        codes_s[p] = code;
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
            const uint64_t c00 = codes_s[l], c01 = codes_s[l + 1], c10 = codes_s[l + TILE], c11 = codes_s[l + TILE + 1];
            const size_t o = (size_t)y * T.wo + x;
            codes[o] = c00;
            codes[o + 1] = c01;
            codes[o + T.wo] = c10;
            codes[o + T.wo + 1] = c11;
            if (!((c00 | c01 | c10 | c11) & kHoleBit)) {
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

}  // namespace

void launch_tile(const SynthBuffers& b, const ViewTable& tab, const LaunchShape& sh, const DebugPtrs& dbg, uint16_t* out_y,
                 uint16_t* out_u, uint16_t* out_v, cudaStream_t s) {
    tile_kernel<<<sh.ntx * sh.nty, TILE_THREADS, 0, s>>>(tab, b.counts, b.offsets, b.list, b.status,
                                                         b.codes, out_y, out_u, out_v, dbg);
}

}  // namespace rvsb
