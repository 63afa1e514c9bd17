// Device helpers shared by the synthesis kernels.
//
// Exactness: every float operation whose result decides coverage (the
// warped u, v and the barycentric tests) or feeds the colour is written with
// explicit round-to-nearest intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, ...)
// in the reference's operation order, so nvcc cannot contract them into
// fused multiply-adds.  The translation units are also built with -fmad=false.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "device_types.hpp"

namespace rvsb {
namespace dev {

constexpr uint64_t kEmptyKey = ~0ull;
constexpr uint64_t kHoleBit = 1ull << 48;
constexpr uint64_t kCodeMask = (1ull << 48) - 1;

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fffffff); }

// First statement of every synthesis kernel: with programmatic dependent
// launch (launch_dependent in kernels.hpp) the kernel's CTAs may be resident
// before the previous kernel on the stream has finished; this waits until
// it has, and its writes are visible.  Without that launch attribute it
// returns at once.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// static_cast<int>(float) as compiled for x86-64 (cvttss2si): INT_MIN for
// NaN or out-of-range values.
__device__ __forceinline__ int x86_cvt(float x) {
    return (x >= -2147483648.0f && x < 2147483648.0f) ? __float2int_rz(x) : INT_MIN;
}
// std::min / std::max argument order (NaN handling).
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

// Depth decode of process_input_frame.cu:346-385 (normalize kernel, built by
// nvcc with fused multiply-add: near + d*(far-near) is one fma).
// A depth sample takes one of 65536 values, so the warp reads the decoded
// depth from a per-view table built with this function (depth_lut_kernel).
__device__ __forceinline__ float decode_depth_raw(float near_, float far_, float depth_scale, int has_invalid,
                                                 uint32_t raw) {
    const float dd = __fmul_rn((float)raw, depth_scale);
    float z;
    if (far_ >= 1000.f)
        z = __fdiv_rn(near_, dd);
    else
        z = __fdiv_rn(__fmul_rn(far_, near_), __fmaf_rn(dd, __fsub_rn(far_, near_), near_));
    if (has_invalid && z == 0.f) z = qnan();
    return z;
}

// One warped vertex (u, v, virtual depth): SynthesizedView.cpp:320-331 with
// PerspectiveUnprojector.cpp:59-86 / EquirectangularUnprojector.cpp:55-98,
// SynthesizedView.cpp:68-79 and PerspectiveProjector.cpp:59-87 /
// EquirectangularProjector.cpp:60-99.
// View: DevView, or a copy of the fields used here (the warp kernel keeps
// them in registers).
// The depth-table entry of input pixel (i, j): the decoded depth and the
// perspective factors of its raw sample.
template <class View>
__device__ __forceinline__ float4 depth_entry(const View& V, int i, int j) {
    return __ldg(V.depth_lut + __ldg(V.pd + (size_t)i * V.w + j));
}

// L: depth_entry(V, i, j), loaded by the caller (the warp kernel issues a
// thread's loads ahead of its arithmetic).
template <class View>
__device__ __forceinline__ float4 warp_vertex(const View& V, const DevTarget& T, int i, int j, float4 L) {
    const float d = L.x;
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
            // L.y = -(d / f0), L.z = -(d / f1), divided once per sample
            // value when the table was built.
            x1 = __fmul_rn(L.y, __fsub_rn(pu, V.p0));
            x2 = __fmul_rn(L.z, __fsub_rn(pv, V.p1));
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
    if (T.rescale) {
        // cv::transform with Matx22f(sx, 0, 0, sy) (SynthesizedView.cpp:330-331)
        const float su = __fadd_rn(__fmul_rn(T.uv_sx, u), __fmul_rn(0.f, v));
        const float sv = __fadd_rn(__fmul_rn(0.f, u), __fmul_rn(T.uv_sy, v));
        u = su;
        v = sv;
    }
    return make_float4(u, v, z, 0.f);
}

template <class View>
__device__ __forceinline__ float4 warp_vertex(const View& V, const DevTarget& T, int i, int j) {
    return warp_vertex(V, T, i, j, depth_entry(V, i, j));
}

// Triangle quality of transform.cpp:62-75 (valid_tri): the longest edge by
// cv::norm (double sum of squared float differences, double sqrt), then
// clamp(10000 - 1000 * stretch, 1, 10000) in float.  sqrt is monotone, so
// the square root of the largest squared length equals the largest length.
__device__ __forceinline__ double sq_len(float ax, float ay, float bx, float by) {
    const double dx = (double)__fsub_rn(ax, bx), dy = (double)__fsub_rn(ay, by);
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}
__device__ __forceinline__ float tri_quality(float ax, float ay, float bx, float by, float cx, float cy,
                                            float precision = 1.f) {
    const double m = fmax(sq_len(bx, by, cx, cy), fmax(sq_len(ax, ay, bx, by), sq_len(ax, ay, cx, cy)));
    float stretch = (float)__dsqrt_rn(m);
    if (precision != 1.f) stretch = __fdiv_rn(stretch, precision);  // stretch /= g_rescale
    float q = __fsub_rn(10000.f, __fmul_rn(1000.f, stretch));
    q = smax(1.f, q);
    q = smin(10000.f, q);
    return q;
}

struct TriSetup {
    float b1c1, c0b0, c1a1, a0c0, den;
    int x0, x1, y0, y1;  // candidate pixel range
    float rinv;          // approximate 1 / den (at most 1 ulp off)
};

// Reciprocal with at most 1 ulp error (PTX rcp.approx.f32, subnormals kept).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Edge coefficients and den of colorize_triangle (transform.cpp:82-84).
// Returns false when den <= 0 (the reference returns) or den is not finite
// (a non-finite vertex: no pixel can pass the barycentric test).
__device__ __forceinline__ bool tri_coef(float4 A, float4 B, float4 C, TriSetup& s) {
    s.b1c1 = __fsub_rn(B.y, C.y);
    s.a0c0 = __fsub_rn(A.x, C.x);
    s.c0b0 = __fsub_rn(C.x, B.x);
    s.c1a1 = __fsub_rn(C.y, A.y);
    const float a1c1 = __fsub_rn(A.y, C.y);
    s.den = __fadd_rn(__fmul_rn(s.b1c1, s.a0c0), __fmul_rn(s.c0b0, a1c1));
    return s.den > 0.f && !isinf(s.den);
}

// Candidate pixel range of a triangle, clipped to [cx0, cx1] x [cy0, cy1].
//
// A point whose computed barycentric coordinates are all >= -1e-6 lies
// within 2e-6 * L (L = the larger bounding-box extent) of the triangle's
// bounding box, plus the float error of the coordinates (about 1.2e-7 of
// the distance); delta = 4e-3 + 1e-5 * L covers both with margin and the
// rounding of this computation.  For delta < 0.5 this range lies inside the
// CPU's bounding box [floor(min), ceil(max)] (transform.cpp:90-96), so the
// CPU box is evaluated, with its static_cast<int> semantics, only for very
// large or far-away triangles.
__device__ __forceinline__ bool tri_range(float4 A, float4 B, float4 C, int wo, int ho, int cx0, int cx1, int cy0,
                                          int cy1, TriSetup& s) {
    const float mnx = fminf(fminf(A.x, B.x), C.x), mxx = fmaxf(fmaxf(A.x, B.x), C.x);
    const float mny = fminf(fminf(A.y, B.y), C.y), mxy = fmaxf(fmaxf(A.y, B.y), C.y);
    const float L = fmaxf(mxx - mnx, mxy - mny);
    int x0 = cx0, x1 = cx1, y0 = cy0, y1 = cy1;
    if (!(L < 4.0e4f && mnx > -1.0e7f && mxx < 1.0e7f && mny > -1.0e7f && mxy < 1.0e7f)) {
        x0 = max(x0, max(0, x86_cvt(floorf(smin(smin(A.x, B.x), C.x)))));
        y0 = max(y0, max(0, x86_cvt(floorf(smin(smin(A.y, B.y), C.y)))));
        x1 = min(x1, min(wo - 1, x86_cvt(ceilf(smax(smax(A.x, B.x), C.x)))));
        y1 = min(y1, min(ho - 1, x86_cvt(ceilf(smax(smax(A.y, B.y), C.y)))));
        if (x0 > x1 || y0 > y1) return false;
    }
    const float delta = 4e-3f + 1e-5f * L;
    const float fx0 = ceilf(mnx - 0.5f - delta), fx1 = floorf(mxx - 0.5f + delta);
    const float fy0 = ceilf(mny - 0.5f - delta), fy1 = floorf(mxy - 0.5f + delta);
    if (fx0 > (float)x0) x0 = fx0 > 2.0e9f ? INT_MAX : (int)fx0;
    if (fx1 < (float)x1) x1 = fx1 < -2.0e9f ? INT_MIN : (int)fx1;
    if (fy0 > (float)y0) y0 = fy0 > 2.0e9f ? INT_MAX : (int)fy0;
    if (fy1 < (float)y1) y1 = fy1 < -2.0e9f ? INT_MIN : (int)fy1;
    s.x0 = x0; s.x1 = x1; s.y0 = y0; s.y1 = y1;
    return x0 <= x1 && y0 <= y1;
}

// Candidate x range of row y for a large triangle.  Each edge test
// n_k = a_k*tx + b_k*ty + c_k >= -1e-6*den (n_3 = den - n_1 - n_2) bounds tx
// on one side; the bound is widened by 16 ulp of its terms plus 1e-3 and
// then by one pixel, and an edge whose bound is not reliable to half a pixel
// (nearly horizontal edges) is not used.  Every pixel of the span is still
// tested exactly, so the span only has to contain the covered pixels.
__device__ __forceinline__ void row_span(const TriSetup& s, float cx, float cy, int y, int& xl, int& xr) {
    const float eps = 1e-6f, u = 5.9604645e-8f;
    const float ty = __fsub_rn(__fadd_rn((float)y, 0.5f), cy);
    const float a[3] = {s.b1c1, s.c1a1, -(s.b1c1 + s.c1a1)};
    const float b[3] = {s.c0b0, s.a0c0, -(s.c0b0 + s.a0c0)};
    const float c[3] = {0.f, 0.f, s.den};
    float lo = -INFINITY, hi = INFINITY;
    bool empty = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float rhs = -eps * s.den - b[k] * ty - c[k];
        const float mag = fabsf(eps * s.den) + fabsf(b[k] * ty) + fabsf(c[k]);
        if (a[k] == 0.f) {
            if (rhs > 16.f * u * mag) empty = true;
            continue;
        }
        const float bd = __fdividef(rhs, a[k]);
        const float err = 16.f * u * (__fdividef(mag, fabsf(a[k])) + fabsf(bd)) + 1e-3f;
        if (!(err <= 0.5f)) continue;
        if (a[k] > 0.f)
            lo = fmaxf(lo, bd - err);
        else
            hi = fminf(hi, bd + err);
    }
    xl = s.x0;
    xr = s.x1;
    if (lo > -INFINITY) xl = max(xl, (int)fmaxf(-1.0e9f, floorf(cx - 0.5f + lo) - 1.f));
    if (hi < INFINITY) xr = min(xr, (int)fminf(1.0e9f, ceilf(cx - 0.5f + hi) + 1.f));
    if (empty) xr = xl - 1;
}

// Barycentric coordinates at pixel (x, y) exactly as transform.cpp:108-111.
__device__ __forceinline__ void barycentric(const TriSetup& s, float cx, float cy, int x, int y, float& l1,
                                            float& l2, float& l3) {
    const float tx = __fsub_rn(__fadd_rn((float)x, 0.5f), cx);
    const float ty = __fsub_rn(__fadd_rn((float)y, 0.5f), cy);
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

// Vertex pixel coordinates of triangle `t` of quad (i, j) (transform.cpp:162-174).
__device__ __forceinline__ void tri_vertices(int w, int i, int j, int t, int& ax, int& ay, int& bx, int& by,
                                             int& cx, int& cy) {
    switch (t) {
        case 0: ax = j; ay = i; bx = j + 1; by = i; cx = j; cy = i + 1; break;
        case 1: ax = j + 1; ay = i + 1; bx = j; by = i + 1; cx = j + 1; cy = i; break;
        case 2: ax = w - 1; ay = i; bx = 0; by = i; cx = w - 1; cy = i + 1; break;
        default: ax = 0; ay = i + 1; bx = w - 1; by = i + 1; cx = 0; cy = i; break;
    }
}

// Upsampled chroma of the loader (resizeUV, process_input_frame.cu:22-81)
// for an even-sized view: source x = x * 0.5, so the bilinear weights are
// 0 or 1/2 and the float result is exact; 4x the value is the integer sum
// computed here.
__device__ __forceinline__ uint32_t chroma4(const uint16_t* p, int cw, int ch, int x, int y) {
    const int x1 = x >> 1, y1 = y >> 1;
    const int x2 = min(x1 + 1, cw - 1), y2 = min(y1 + 1, ch - 1);
    const uint32_t ox = x & 1, oy = y & 1;
    const uint32_t a = p[y1 * cw + x1], b = p[y1 * cw + x2], c = p[y2 * cw + x1], d = p[y2 * cw + x2];
    return a * (2 - ox) * (2 - oy) + b * ox * (2 - oy) + c * (2 - ox) * oy + d * ox * oy;
}

// Colour of input pixel (x, y): mergeYUV (process_input_frame.cu:211-238),
// float3(Y * s, U * s, V * s), s = 1 / (2^bits - 1).
__device__ __forceinline__ float3 input_color(const DevView& V, int x, int y) {
    const float cs = V.color_scale;
    float3 c;
    c.x = __fmul_rn((float)V.py[(size_t)y * V.w + x], cs);
    c.y = __fmul_rn(__fmul_rn((float)chroma4(V.pu, V.cw, V.ch, x, y), 0.25f), cs);
    c.z = __fmul_rn(__fmul_rn((float)chroma4(V.pv, V.cw, V.ch, x, y), 0.25f), cs);
    return c;
}

// powf(x, BlendingFactor) of blend_img (blending.cpp:332-337).  Integer
// exponents are evaluated as a double product and rounded once, which is
// the correctly rounded result except within about 2^-28 of a rounding
// boundary.
__device__ __forceinline__ float blend_pow(float x, float e, int e_int) {
    if (e == 1.f) return x;
    if (e_int > 0) {
        const double b = (double)x;
        double r = b;
        for (int k = 1; k < e_int; ++k) r = __dmul_rn(r, b);
        return __double2float_rn(r);
    }
    return powf(x, e);
}

// cv::resize(0.5, 0.5, INTER_LINEAR) of a uint16 plane at one output
// sample (image_writing.cpp:83-84): the 2x2 sum s over 4, rounded; ties go
// up in OpenCV's own code and to even in its IPP build.
__device__ __forceinline__ uint16_t quarter_round(uint32_t s, int ties_up) {
    const uint32_t q = s >> 2, r = s & 3u;
    const uint32_t up = ties_up ? (r >= 2u) : ((r > 2u) | ((r == 2u) & q));
    return (uint16_t)(q + (up & 1u));
}

// cv::resize with INTER_LINEAR (write_color's resize, image_writing.cpp:190;
// the depth resize of Pipeline.cpp:323-333): source coordinate of
// destination index d, (d + 0.5) * scale - 0.5, giving the left (top) tap and
// the weight of the right (bottom) one, clamped at both borders.
__device__ __forceinline__ void linear_tap(int d, double scale, int n, int& s0, int& s1, float& f) {
    f = (float)__dadd_rn(__dmul_rn((double)d + 0.5, scale), -0.5);
    int s = (int)floorf(f);
    f = __fsub_rn(f, (float)s);
    if (s < 0) {
        f = 0.f;
        s = 0;
    }
    if (s >= n - 1) {
        f = 0.f;
        s = n - 1;
    }
    s0 = s;
    s1 = min(s + 1, n - 1);
}

__device__ __forceinline__ float lerp2(float a, float b, float wa, float wb) {
    return __fadd_rn(__fmul_rn(a, wa), __fmul_rn(b, wb));
}

// static_cast<ushort>(v * max_level) (image_writing.cpp:165-172).
__device__ __forceinline__ uint32_t quantize(float c, unsigned max_val) {
    const uint32_t q = __float2uint_rz(__fmul_rn(c, (float)max_val));
    return q > 65535u ? 65535u : q;
}

}  // namespace dev
}  // namespace rvsb
