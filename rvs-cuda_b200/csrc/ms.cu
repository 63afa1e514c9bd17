// Multispectral blending (BlendedViewMultiSpec, rvs/src/BlendedView.cpp:63-88),
// after the raster has stored every view's resolved colour and quality:
// split_frequencies (blending.cpp:371-395; YUV: only luma is blurred) with
// calcBlurring (blending.cpp:62-105: box mean over the masked pixels of a
// (2r+1)^2 window clipped to the image, r = max(W, H) / 20, the window sum
// truncated to an integer before the division by the count, 0 outside the
// mask of quality > 0), then the low band (blur(Y), U, V) and the high band
// (Y - blur(Y), 0, 0) blended separately with their own factors and added.
// The window sums are accumulated in double as the reference's integral
// image is; only their order differs, which can change a truncated sum only
// when it lies within about 1e-10 of an integer.
#include "device_common.cuh"
#include "kernels.hpp"
#include "resolve.cuh"

namespace rvsb {
namespace {

using namespace dev;

constexpr int MS_THREADS = 256;

// Row-window sums of masked luma: one CTA per (row, view, slot).  The row's
// exclusive prefix (double sums, integer counts) is built in shared memory.
template <class Tabs>
__global__ void __launch_bounds__(MS_THREADS) ms_rows_kernel(const __grid_constant__ Tabs tabs) {
    grid_dep_wait();
    extern __shared__ __align__(16) unsigned char s_raw[];
    const SlotTable& tab = tabs.at(blockIdx.z);
    const MsPtrs& M = tab.ms;
    if (!M.on) return;
    const DevTarget& T = tab.t;
    const int v = blockIdx.y, y = blockIdx.x;
    if (v >= T.n_views || y >= T.ho) return;
    const int w = T.wo;
    double* P = reinterpret_cast<double*>(s_raw);                     // w + 1 prefix sums
    int* C = reinterpret_cast<int*>(s_raw + sizeof(double) * (w + 1));  // w + 1 prefix counts
    __shared__ double s_wsum[MS_THREADS / 32];
    __shared__ int s_wcnt[MS_THREADS / 32];
    const size_t npo = (size_t)T.wo * T.ho;
    const float4* row = M.view + (size_t)v * npo + (size_t)y * w;
    // Each thread sums a contiguous chunk, then a block scan of the chunks.
    const int per = (w + MS_THREADS - 1) / MS_THREADS;
    const int beg = min(w, (int)threadIdx.x * per), end = min(w, beg + per);
    double ls = 0.0;
    int lc = 0;
    for (int x = beg; x < end; ++x) {
        const float4 c = row[x];
        if (c.w > 0.f && isfinite(c.x)) {
            ls += (double)c.x;
            ++lc;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double is = ls;
    int ic = lc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double a = __shfl_up_sync(0xffffffffu, is, o);
        const int b = __shfl_up_sync(0xffffffffu, ic, o);
        if (lane >= o) {
            is += a;
            ic += b;
        }
    }
    if (lane == 31) {
        s_wsum[warp] = is;
        s_wcnt[warp] = ic;
    }
    __syncthreads();
    double base = 0.0;
    int cbase = 0;
    for (int k = 0; k < warp; ++k) {
        base += s_wsum[k];
        cbase += s_wcnt[k];
    }
    double run = base + is - ls;
    int crun = cbase + ic - lc;
    if (threadIdx.x == 0) {
        P[0] = 0.0;
        C[0] = 0;
    }
    for (int x = beg; x < end; ++x) {
        const float4 c = row[x];
        if (c.w > 0.f && isfinite(c.x)) {
            run += (double)c.x;
            ++crun;
        }
        P[x + 1] = run;
        C[x + 1] = crun;
    }
    __syncthreads();
    const int rad = M.rad;
    double* hs = M.hsum + (size_t)v * npo + (size_t)y * w;
    int* hc = M.hcnt + (size_t)v * npo + (size_t)y * w;
    for (int x = threadIdx.x; x < w; x += MS_THREADS) {
        const int a = max(0, x - rad), b = min(w, x - rad + 2 * rad + 1);
        hs[x] = P[b] - P[a];
        hc[x] = C[b] - C[a];
    }
}

// Column windows of the row sums, one thread per column and view, sliding
// down the column; writes the blurred luma.
template <class Tabs>
__global__ void ms_cols_kernel(const __grid_constant__ Tabs tabs) {
    grid_dep_wait();
    const SlotTable& tab = tabs.at(blockIdx.z);
    const MsPtrs& M = tab.ms;
    if (!M.on) return;
    const DevTarget& T = tab.t;
    const int v = blockIdx.y, x = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= T.n_views || x >= T.wo) return;
    const int w = T.wo, h = T.ho, rad = M.rad;
    const size_t npo = (size_t)w * h;
    const double* hs = M.hsum + (size_t)v * npo;
    const int* hc = M.hcnt + (size_t)v * npo;
    const float4* vw = M.view + (size_t)v * npo;
    float* out = M.blur + (size_t)v * npo;
    double s = 0.0;
    int c = 0;
    for (int y = 0; y <= min(rad, h - 1); ++y) {
        s += hs[(size_t)y * w + x];
        c += hc[(size_t)y * w + x];
    }
    for (int y = 0; y < h; ++y) {
        const size_t o = (size_t)y * w + x;
        float b = 0.f;
        if (vw[o].w > 0.f && c > 0) {
            const unsigned sum = (unsigned)(int)s;
            b = __fdiv_rn((float)sum, (float)c);
        }
        out[o] = b;
        const int yin = y + rad + 1, yout = y - rad;
        if (yin < h) {
            s += hs[(size_t)yin * w + x];
            c += hc[(size_t)yin * w + x];
        }
        if (yout >= 0) {
            s -= hs[(size_t)yout * w + x];
            c -= hc[(size_t)yout * w + x];
        }
    }
}

// The two bands' blends per pixel, added; one thread per 2x2 output block
// rewrites the colour part of the codes (the hole bits from the raster stay)
// and the output samples of hole-free blocks.
template <class Tabs>
__global__ void ms_blend_kernel(const __grid_constant__ Tabs tabs) {
    grid_dep_wait();
    const SlotTable& tab = tabs.at(blockIdx.z);
    const MsPtrs& M = tab.ms;
    if (!M.on) return;
    const DevTarget& T = tab.t;
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y;
    const int x0 = 2 * bx, y0 = 2 * by;
    if (x0 >= T.wo || y0 >= T.ho) return;
    const size_t npo = (size_t)T.wo * T.ho;
    uint64_t code[4];
    bool any_hole = false;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        code[p] = 0;
        // partial blocks of a raster of odd width or height (Precision != 1)
        if (x0 + (p & 1) >= T.wo || y0 + (p >> 1) >= T.ho) continue;
        const size_t o = (size_t)(y0 + (p >> 1)) * T.wo + x0 + (p & 1);
        BlendAcc lo = {0.f, 0.f, 0.f, 0.f}, hi = {0.f, 0.f, 0.f, 0.f};
        for (int v = 0; v < T.n_views; ++v) {
            const float4 c = M.view[(size_t)v * npo + o];
            const float b = M.blur[(size_t)v * npo + o];
            const float3 lowc = make_float3(b, c.y, c.z);
            const float3 highc = make_float3(__fsub_rn(c.x, b), __fsub_rn(c.y, c.y), __fsub_rn(c.z, c.z));
            blend_view(lo, v, lowc, c.w, M.low_exp, M.low_int, M.low_exp < 0.f);
            blend_view(hi, v, highc, c.w, M.high_exp, M.high_int, M.high_exp < 0.f);
        }
        const float f0 = __fadd_rn(lo.c0, hi.c0), f1 = __fadd_rn(lo.c1, hi.c1), f2 = __fadd_rn(lo.c2, hi.c2);
        if (T.rescale) tab.b.pcolor[o] = make_float4(f0, f1, f2, 0.f);
        const uint64_t hole = tab.b.codes[o] & kHoleBit;
        any_hole |= hole != 0;
        code[p] = (uint64_t)quantize(f0, T.max_val) | ((uint64_t)quantize(f1, T.max_val) << 16) |
                  ((uint64_t)quantize(f2, T.max_val) << 32) | hole;
        tab.b.codes[o] = code[p];
        if (tab.dbg.blend_color) {
            tab.dbg.blend_color[o * 3 + 0] = f0;
            tab.dbg.blend_color[o * 3 + 1] = f1;
            tab.dbg.blend_color[o * 3 + 2] = f2;
        }
    }
    if (any_hole || T.rescale) return;  // written by the inpainting passes or the resize
    const size_t o = (size_t)y0 * T.wo + x0;
    tab.out_y[o] = (uint16_t)(code[0] & 0xffff);
    tab.out_y[o + 1] = (uint16_t)(code[1] & 0xffff);
    tab.out_y[o + T.wo] = (uint16_t)(code[2] & 0xffff);
    tab.out_y[o + T.wo + 1] = (uint16_t)(code[3] & 0xffff);
    uint32_t su = 0, sv = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        su += (uint32_t)((code[p] >> 16) & 0xffff);
        sv += (uint32_t)((code[p] >> 32) & 0xffff);
    }
    const size_t co = (size_t)by * (T.wo / 2) + bx;
    tab.out_u[co] = quarter_round(su, T.chroma_ties_up);
    tab.out_v[co] = quarter_round(sv, T.chroma_ties_up);
}

}  // namespace

template <class Tabs>
int launch_ms(const Tabs& tabs, const BatchShape& sh, cudaStream_t s) {
    const size_t smem = (sizeof(double) + sizeof(int)) * (size_t)(sh.max_wo + 1);
    launch_dependent(ms_rows_kernel<Tabs>, dim3(sh.max_ho, sh.max_views, sh.slots), dim3(MS_THREADS), smem, s, tabs);
    launch_dependent(ms_cols_kernel<Tabs>, dim3((sh.max_wo + 127) / 128, sh.max_views, sh.slots), dim3(128), 0, s, tabs);
    launch_dependent(ms_blend_kernel<Tabs>, dim3(((sh.max_wo + 1) / 2 + 127) / 128, (sh.max_ho + 1) / 2, sh.slots),
                     dim3(128), 0, s, tabs);
    return 3;
}

void prepare_ms_kernels(int max_wo) {
    const int smem = (int)((sizeof(double) + sizeof(int)) * (size_t)(max_wo + 1));
    if (smem > 48 * 1024) {
        cudaFuncSetAttribute(ms_rows_kernel<TableParam>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(ms_rows_kernel<TablePtr>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    }
}

template int launch_ms<TableParam>(const TableParam&, const BatchShape&, cudaStream_t);
template int launch_ms<TablePtr>(const TablePtr&, const BatchShape&, cudaStream_t);

}  // namespace rvsb
