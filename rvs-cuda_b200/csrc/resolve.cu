// Resolve stage: per output 2x2 block, re-evaluate each view's winning
// fragment exactly, fold the views into the running blend in blend order
// (BlendedViewSimple::blendBasicMode + blend_img, BlendedView.cpp:180-212,
// blending.cpp:310-369), quantise (image_writing.cpp:142-180), write the
// 4:2:0 output of blocks without holes and leave packed codes for the
// inpainting passes.
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

using namespace dev;

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
__device__ __forceinline__ Fragment resolve(const DevView& V, unsigned long long key, int x, int y) {
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
    f.validity = tri_quality(A.x, A.y, B.x, B.y, C.x, C.y);
    return f;
}

// One thread per output 2x2 block; block (32, 8) covers 64 x 16 pixels.
__global__ void __launch_bounds__(256) resolve_kernel(const __grid_constant__ ViewTable tab,
                                                      const uint64_t* __restrict__ keys, DevStatus* __restrict__ st,
                                                      uint64_t* __restrict__ codes, uint8_t* __restrict__ holes,
                                                      uint16_t* __restrict__ out_y,
                                                      uint16_t* __restrict__ out_u, uint16_t* __restrict__ out_v,
                                                      DebugPtrs dbg) {
    const DevTarget& T = tab.t;
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y * blockDim.y + threadIdx.y;
    const bool inside = 2 * bx < T.wo && 2 * by < T.ho;
    const int x0 = 2 * bx, y0 = 2 * by;
    const size_t npo = (size_t)T.wo * T.ho;
    float acc_c[4][3];
    float acc_q[4];
    uint64_t code[4] = {0, 0, 0, 0};
    bool any_hole = false;
    if (inside) {
        for (int v = 0; v < T.n_views; ++v) {
            const DevView& V = tab.v[v];
            const uint64_t* kv = keys + (size_t)v * npo;
            const ulonglong2 k0 = __ldg(reinterpret_cast<const ulonglong2*>(kv + (size_t)y0 * T.wo + x0));
            const ulonglong2 k1 = __ldg(reinterpret_cast<const ulonglong2*>(kv + (size_t)(y0 + 1) * T.wo + x0));
            const unsigned long long kk[4] = {k0.x, k0.y, k1.x, k1.y};
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const int x = x0 + (p & 1), y = y0 + (p >> 1);
                const Fragment f = resolve(V, kk[p], x, y);
                // SynthetisedViewTriangle::transform: quality = validity / depth.
                const float qv = __fdiv_rn(f.validity, f.depth);
                if (dbg.view_color || dbg.view_depth || dbg.view_validity) {
                    const size_t o = (size_t)y * T.wo + x;
                    if (dbg.view_color) {
                        float* c = dbg.view_color + ((size_t)v * npo + o) * 3;
                        c[0] = f.col.x; c[1] = f.col.y; c[2] = f.col.z;
                    }
                    if (dbg.view_depth) dbg.view_depth[(size_t)v * npo + o] = f.depth;
                    if (dbg.view_validity) dbg.view_validity[(size_t)v * npo + o] = f.validity;
                }
                if (v == 0) {
                    acc_c[p][0] = f.col.x; acc_c[p][1] = f.col.y; acc_c[p][2] = f.col.z;
                    acc_q[p] = qv;
                } else {
                    // blend_img over {accumulator, new view}: weights quality^exp
                    // for quality > 0, colour * (1 / sum), quality = sum^(1/exp).
                    // acc_q holds the first view's quality after view 0 and the
                    // weight sum afterwards: the reference re-powers its stored
                    // quality sum^(1/exp) by exp, which returns the sum up to a
                    // few ulp, and quality > 0 exactly when the sum is > 0.
                    float sum = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
                    if (acc_q[p] > 0.f) {
                        const float w = v == 1 ? blend_pow(acc_q[p], T.blend_exp, T.blend_exp_int) : acc_q[p];
                        sum = __fadd_rn(sum, w);
                        c0 = __fadd_rn(c0, __fmul_rn(w, acc_c[p][0]));
                        c1 = __fadd_rn(c1, __fmul_rn(w, acc_c[p][1]));
                        c2 = __fadd_rn(c2, __fmul_rn(w, acc_c[p][2]));
                    }
                    if (qv > 0.f) {
                        const float w = blend_pow(qv, T.blend_exp, T.blend_exp_int);
                        sum = __fadd_rn(sum, w);
                        c0 = __fadd_rn(c0, __fmul_rn(w, f.col.x));
                        c1 = __fadd_rn(c1, __fmul_rn(w, f.col.y));
                        c2 = __fadd_rn(c2, __fmul_rn(w, f.col.z));
                    }
                    if (sum == 0.f) {
                        acc_c[p][0] = 0.f; acc_c[p][1] = 1.f; acc_c[p][2] = 0.f;
                        acc_q[p] = 0.f;
                    } else {
                        const float inv = __frcp_rn(sum);
                        acc_c[p][0] = __fmul_rn(c0, inv);
                        acc_c[p][1] = __fmul_rn(c1, inv);
                        acc_c[p][2] = __fmul_rn(c2, inv);
                        acc_q[p] = sum;
                    }
                }
            }
        }
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int x = x0 + (p & 1), y = y0 + (p >> 1);
            const bool hole = !(acc_q[p] > 0.f);
            any_hole |= hole;
            code[p] = (uint64_t)quantize(acc_c[p][0], T.max_val) | ((uint64_t)quantize(acc_c[p][1], T.max_val) << 16) |
                      ((uint64_t)quantize(acc_c[p][2], T.max_val) << 32) | (hole ? kHoleBit : 0ull);
            const size_t o = (size_t)y * T.wo + x;
            if (dbg.blend_color) {
                dbg.blend_color[o * 3 + 0] = acc_c[p][0];
                dbg.blend_color[o * 3 + 1] = acc_c[p][1];
                dbg.blend_color[o * 3 + 2] = acc_c[p][2];
            }
            if (dbg.blend_quality)
                dbg.blend_quality[o] = (T.n_views == 1 || !(acc_q[p] > 0.f)) ? acc_q[p] : powf(acc_q[p], T.inv_blend_exp);
            if (dbg.inpaint_source) {
                dbg.inpaint_source[o * 2 + 0] = x;
                dbg.inpaint_source[o * 2 + 1] = y;
            }
        }
        const size_t o = (size_t)y0 * T.wo + x0;
        reinterpret_cast<ulonglong2*>(codes + o)[0] = make_ulonglong2(code[0], code[1]);
        reinterpret_cast<ulonglong2*>(codes + o + T.wo)[0] = make_ulonglong2(code[2], code[3]);
        auto hole_of = [](uint64_t c) -> uint16_t { return (c & kHoleBit) ? 1 : 0; };
        reinterpret_cast<uint16_t*>(holes + o)[0] = (uint16_t)(hole_of(code[0]) | (hole_of(code[1]) << 8));
        reinterpret_cast<uint16_t*>(holes + o + T.wo)[0] = (uint16_t)(hole_of(code[2]) | (hole_of(code[3]) << 8));
        if (!any_hole) {
            reinterpret_cast<uint32_t*>(out_y + o)[0] = (uint32_t)(code[0] & 0xffff) | ((uint32_t)(code[1] & 0xffff) << 16);
            reinterpret_cast<uint32_t*>(out_y + o + T.wo)[0] =
                (uint32_t)(code[2] & 0xffff) | ((uint32_t)(code[3] & 0xffff) << 16);
            uint32_t su = 0, sv = 0;
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                su += (uint32_t)((code[p] >> 16) & 0xffff);
                sv += (uint32_t)((code[p] >> 32) & 0xffff);
            }
            const size_t co = (size_t)by * (T.wo / 2) + bx;
            out_u[co] = quarter_round(su, T.chroma_ties_up);
            out_v[co] = quarter_round(sv, T.chroma_ties_up);
        }
    }
    // Bounding box of the holes: warp reduction, one atomic per warp.
    int hx0 = INT_MAX, hy0 = INT_MAX, hx1 = INT_MIN, hy1 = INT_MIN;
    if (any_hole) {
        const bool left = (code[0] & kHoleBit) || (code[2] & kHoleBit);
        const bool right = (code[1] & kHoleBit) || (code[3] & kHoleBit);
        const bool top = (code[0] & kHoleBit) || (code[1] & kHoleBit);
        const bool bottom = (code[2] & kHoleBit) || (code[3] & kHoleBit);
        hx0 = left ? x0 : x0 + 1;
        hx1 = right ? x0 + 1 : x0;
        hy0 = top ? y0 : y0 + 1;
        hy1 = bottom ? y0 + 1 : y0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, any_hole);
    if (m) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            hx0 = min(hx0, __shfl_xor_sync(0xffffffffu, hx0, o));
            hy0 = min(hy0, __shfl_xor_sync(0xffffffffu, hy0, o));
            hx1 = max(hx1, __shfl_xor_sync(0xffffffffu, hx1, o));
            hy1 = max(hy1, __shfl_xor_sync(0xffffffffu, hy1, o));
        }
        if (threadIdx.x == 0) {
            atomicMin(&st->hole_x0, hx0);
            atomicMin(&st->hole_y0, hy0);
            atomicMax(&st->hole_x1, hx1);
            atomicMax(&st->hole_y1, hy1);
            atomicAdd(&st->n_holes, 1);
        }
    }
}

}  // namespace

void launch_resolve(const SynthBuffers& b, const ViewTable& tab, const LaunchShape& sh, const DebugPtrs& dbg,
                    uint16_t* out_y, uint16_t* out_u, uint16_t* out_v, cudaStream_t s) {
    dim3 block(32, 8);
    dim3 grid((sh.wo / 2 + 31) / 32, (sh.ho / 2 + 7) / 8);
    resolve_kernel<<<grid, block, 0, s>>>(tab, b.keys, b.status, b.codes, b.holes, out_y, out_u, out_v, dbg);
}

}  // namespace rvsb
