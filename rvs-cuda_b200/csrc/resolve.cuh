// Resolve and blend of one output pixel, used by the raster kernel once a
// view's z-buffer is final: re-evaluate the winning fragment exactly, fold it
// into the running blend in blend order (BlendedViewSimple::blendBasicMode +
// blend_img, BlendedView.cpp:180-212, blending.cpp:310-369).
#pragma once

#include "device_common.cuh"

namespace rvsb {
namespace dev {

struct Fragment {
    float3 col;
    float depth;      // +inf when uncovered
    float validity;   // triangle quality, 0 when uncovered
};

__device__ __forceinline__ float3 packed_color(const DevView& V, int x, int y) {
    const uint64_t c = __ldg(reinterpret_cast<const unsigned long long*>(V.color) + (size_t)y * V.w + x);
    const float cs = V.color_scale;
    float3 r;
    r.x = __fmul_rn((float)(uint32_t)(c & 0x3ffffu), cs);
    r.y = __fmul_rn(__fmul_rn((float)(uint32_t)((c >> 18) & 0x3ffffu), 0.25f), cs);
    r.z = __fmul_rn(__fmul_rn((float)(uint32_t)((c >> 36) & 0x3ffffu), 0.25f), cs);
    return r;
}

// Re-evaluates the winning triangle at pixel (x, y) exactly as the CPU's
// colorize_triangle does for the fragment it keeps (transform.cpp:109-135).
__device__ __forceinline__ Fragment resolve_fragment(const DevView& V, unsigned long long key, int x, int y,
                                                     float precision = 1.f) {
    Fragment f;
    f.col = make_float3(0.f, 0.f, 0.f);
    f.depth = INFINITY;
    f.validity = 0.f;
    if (key == kEmptyKey) return f;
    const uint32_t tri = (uint32_t)(key & 0xffffffffull);
    const int t = (int)(tri & 3u);
    const int i = (int)(tri >> V.tri_shift), j = (int)((tri >> 2) & ((1u << (V.tri_shift - 2)) - 1u));
    int ax, ay, bx, by, cx, cy;
    if (t < 2) {
        // The two triangles of quad (i, j) without a branch per case:
        // t = 0: (j, i), (j+1, i), (j, i+1); t = 1: (j+1, i+1), (j, i+1), (j+1, i).
        ax = j + t; ay = i + t;
        bx = j + 1 - t; by = i + t;
        cx = j + t; cy = i + 1 - t;
    } else {
        tri_vertices(V.w, i, j, t, ax, ay, bx, by, cx, cy);
    }
    const float4* vt = V.vert;
    const float4 A = __ldg(vt + (size_t)ay * V.w + ax);
    const float4 B = __ldg(vt + (size_t)by * V.w + bx);
    const float4 C = __ldg(vt + (size_t)cy * V.w + cx);
    const float3 ca = packed_color(V, ax, ay), cb = packed_color(V, bx, by), cc = packed_color(V, cx, cy);
    TriSetup s;
    tri_coef(A, B, C, s);
    float l1, l2, l3;
    barycentric(s, C.x, C.y, x, y, l1, l2, l3);
    f.col.x = interp(ca.x, cb.x, cc.x, l1, l2, l3);
    f.col.y = interp(ca.y, cb.y, cc.y, l1, l2, l3);
    f.col.z = interp(ca.z, cb.z, cc.z, l1, l2, l3);
    f.depth = interp(A.z, B.z, C.z, l1, l2, l3);
    f.validity = tri_quality(A.x, A.y, B.x, B.y, C.x, C.y, precision);
    return f;
}

// Running blend of one pixel: colour and, after view 0, the weight sum
// (view 0: its own quality).
struct BlendAcc {
    float c0, c1, c2, q;
};

// Folds view v's fragment (colour, quality = validity / depth, the quality
// of SynthetisedViewTriangle::transform) into the accumulator.  blend_img
// over {accumulator, new view}: weights quality^exp for quality > 0, colour
// * (1 / sum), quality = sum^(1/exp).  After view 0 the accumulator keeps the
// weight sum itself: the reference re-powers its stored sum^(1/exp) by exp,
// which returns the sum up to a few ulp, and quality > 0 exactly when the
// sum is > 0.
__device__ __forceinline__ void blend_view(BlendAcc& a, int v, float3 col, float qv, float blend_exp, int exp_int,
                                           bool by_max) {
    if (v == 0) {
        a.c0 = col.x;
        a.c1 = col.y;
        a.c2 = col.z;
        a.q = qv;
        return;
    }
    if (by_max) {
        // blend_img_by_max (blending.cpp:293-308): the empty colour and
        // quality 0, replaced by the accumulator where its quality is
        // positive, then by the view where its quality is larger still.
        BlendAcc r = {0.f, 1.f, 0.f, 0.f};
        if (a.q > r.q) r = a;
        if (qv > r.q) {
            r.c0 = col.x;
            r.c1 = col.y;
            r.c2 = col.z;
            r.q = qv;
        }
        a = r;
        return;
    }
    float sum = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    if (a.q > 0.f) {
        const float w = v == 1 ? blend_pow(a.q, blend_exp, exp_int) : a.q;
        sum = __fadd_rn(sum, w);
        c0 = __fadd_rn(c0, __fmul_rn(w, a.c0));
        c1 = __fadd_rn(c1, __fmul_rn(w, a.c1));
        c2 = __fadd_rn(c2, __fmul_rn(w, a.c2));
    }
    if (qv > 0.f) {
        const float w = blend_pow(qv, blend_exp, exp_int);
        sum = __fadd_rn(sum, w);
        c0 = __fadd_rn(c0, __fmul_rn(w, col.x));
        c1 = __fadd_rn(c1, __fmul_rn(w, col.y));
        c2 = __fadd_rn(c2, __fmul_rn(w, col.z));
    }
    if (sum == 0.f) {
        a.c0 = 0.f; a.c1 = 1.f; a.c2 = 0.f;
        a.q = 0.f;
    } else {
        const float inv = __frcp_rn(sum);
        a.c0 = __fmul_rn(c0, inv);
        a.c1 = __fmul_rn(c1, inv);
        a.c2 = __fmul_rn(c2, inv);
        a.q = sum;
    }
}

__device__ __forceinline__ void blend_view(BlendAcc& a, int v, const Fragment& f, float qv, const DevTarget& T) {
    blend_view(a, v, f.col, qv, T.blend_exp, T.blend_exp_int, T.blend_max != 0);
}

}  // namespace dev
}  // namespace rvsb
