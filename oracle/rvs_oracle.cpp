/*
 * rvs_oracle.cpp - TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of the reference RVS CPU synthesis path (the `RVS`
 * executable without --cuda/--opengl), used by the tests, by
 * __graft_entry__.smoke() and by bench.py's CPU baseline as the checker.  The
 * product library never links, loads or calls this code.
 *
 * Each function cites the reference file:line it restates (paths relative to
 * the reference project root).  OpenCV operations on the path are written
 * out from their mathematical definitions:
 *   - cv::Matx33f * cv::Vec3f / Matx * Matx: s = 0; s += a(i,k)*b(k) in float
 *   - cv::norm(Vec2f a, Vec2f b): sqrt in double of sum of (double)(a-b)^2,
 *     the difference taken in float (OpenCV 4.9's normL2Sqr<float, double>)
 *   - cv::norm(Vec3f): sqrt in double of sum of (double)x^2, cast to float
 *   - Vec3f / float: multiplication by (1.f / alpha)
 *   - cv::resize(0.5, 0.5, INTER_LINEAR) of uint16 planes: the 2x2 sum s
 *     divided by 4 and rounded; ties go to even in an OpenCV built with
 *     Intel IPP (the default of a source build on x86-64, and the opencv-python
 *     wheel) and up, (s+2) >> 2, in one built without it.
 *     orc_set_chroma_round selects the mode (0: half to even, the default;
 *     1: half up).  Both are pinned against cv2 by tests/golden.
 * Float arithmetic follows the reference's operation order; the file is
 * compiled with -ffp-contract=off so no multiply-add is fused, except where
 * the reference itself runs a CUDA loader kernel built with nvcc's default
 * fused multiply-add (depth decode, process_input_frame.cu:369-376), which is
 * restated with fmaf.
 *
 * Trigonometry: the reference calls std::cos/sin/atan2/asin on float
 * arguments.  Their last bit depends on the platform's libm (glibc 2.39
 * rounds 1.3% of cosf and 16% of atan2f results differently from the
 * correctly rounded value).  By default this oracle evaluates them as the
 * correctly rounded float result (double evaluation, then rounding);
 * orc_set_trig_mode(1) switches to the host libm float functions.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <limits>
#include <vector>
#include <algorithm>

#include "../include/rvsb.h"

namespace {

int g_trig_mode = 0;  // 0: correctly rounded float trig, 1: host libm float trig
int g_chroma_round = 0;  // 0: ties to even (OpenCV with IPP), 1: ties up (without)
// BlendingMethod Multispectral (BlendedViewMultiSpec, BlendedView.cpp:63-88):
// on, BlendingLowFreqFactor, BlendingHighFreqFactor.
int g_ms_on = 0;
float g_ms_low = 0.f, g_ms_high = 0.f;
// "Precision" (detail::g_rescale, Config.cpp:389-399).
float g_precision = 1.f;

// Rounded quarter of a 2x2 sum of uint16 samples (cv::resize 0.5 x 0.5).
inline uint16_t quarter_round(unsigned s) {
    if (g_chroma_round) return (uint16_t)((s + 2) >> 2);
    const unsigned q = s >> 2, r = s & 3;
    return (uint16_t)(q + (r > 2 || (r == 2 && (q & 1))));
}

inline float f_cos(float x) { return g_trig_mode ? std::cos(x) : (float)std::cos((double)x); }
inline float f_sin(float x) { return g_trig_mode ? std::sin(x) : (float)std::sin((double)x); }
inline float f_atan2(float y, float x) {
    return g_trig_mode ? std::atan2(y, x) : (float)std::atan2((double)y, (double)x);
}
inline float f_asin(float x) { return g_trig_mode ? std::asin(x) : (float)std::asin((double)x); }

const float kNaN = std::numeric_limits<float>::quiet_NaN();
const float kInf = std::numeric_limits<float>::infinity();

// std::min / std::max as the reference uses them (NaN handling included).
inline float smin(float a, float b) { return (b < a) ? b : a; }
inline float smax(float a, float b) { return (a < b) ? b : a; }
inline int imin(int a, int b) { return (b < a) ? b : a; }
inline int imax(int a, int b) { return (a < b) ? b : a; }

// static_cast<int>(float) as compiled on x86-64 (cvttss2si): truncation, and
// INT_MIN for NaN or values outside the int range.
inline int cvt_trunc_i32(float x) {
    if (!(x >= -2147483648.0f && x < 2147483648.0f)) return std::numeric_limits<int>::min();
    return (int)x;
}

struct M33 { float m[9]; };

// cv::Matx multiplication (Matx_MatMulOp): s = 0; s += a(i,k) * b(k,j).
M33 matmul(const M33& a, const M33& b) {
    M33 c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float s = 0.f;
            for (int k = 0; k < 3; ++k) s += a.m[i * 3 + k] * b.m[k * 3 + j];
            c.m[i * 3 + j] = s;
        }
    return c;
}

M33 transpose(const M33& a) {
    M33 t;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t.m[i * 3 + j] = a.m[j * 3 + i];
    return t;
}

// Parameters.cpp:67-89 rotation about x, y, z.
M33 rot_x(float r) {
    float c = f_cos(r), s = f_sin(r);
    return M33{{1.f, 0.f, 0.f, 0.f, c, -s, 0.f, s, c}};
}
M33 rot_y(float r) {
    float c = f_cos(r), s = f_sin(r);
    return M33{{c, 0.f, s, 0.f, 1.f, 0.f, -s, 0.f, c}};
}
M33 rot_z(float r) {
    float c = f_cos(r), s = f_sin(r);
    return M33{{c, -s, 0.f, s, c, 0.f, 0.f, 0.f, 1.f}};
}

// Parameters.cpp:151-155 getRotationMatrix -> EulerAnglesToRotationMatrix
// (Parameters.cpp:91-97): Rz(yaw) * Ry(pitch) * Rx(roll) of radperdeg * rotation.
M33 rotation_matrix(const float rot[3]) {
    const float radperdeg = 0.01745329252f;
    float r0 = radperdeg * rot[0], r1 = radperdeg * rot[1], r2 = radperdeg * rot[2];
    return matmul(matmul(rot_z(r0), rot_y(r1)), rot_x(r2));
}

// SpaceTransformer.cpp:77-92.
void relative_pose(const rvsb_camera& in, const rvsb_camera& vt, M33& R, float t[3]) {
    M33 R_from = rotation_matrix(in.rotation);
    M33 R_to = rotation_matrix(vt.rotation);
    M33 R_to_t = transpose(R_to);
    R = matmul(R_to_t, R_from);
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = vt.position[k] - in.position[k];
    // -R_to.t() * (t_to - t_from): unary minus on the matrix, then Matx * Vec.
    for (int i = 0; i < 3; ++i) {
        float s = 0.f;
        for (int k = 0; k < 3; ++k) s += (-R_to_t.m[i * 3 + k]) * d[k];
        t[i] = s;
    }
}

unsigned max_level(int bit_depth) { return (1u << bit_depth) - 1u; }

}  // namespace

extern "C" {

void orc_set_trig_mode(int mode) { g_trig_mode = mode; }
void orc_set_chroma_round(int mode) { g_chroma_round = mode; }
void orc_set_precision(float p) { g_precision = p; }
void orc_set_multispectral(int on, float low, float high) {
    g_ms_on = on;
    g_ms_low = low;
    g_ms_high = high;
}

/* Colour loader: image_loading.cpp:74-145 read_color_YUV, chroma upsample
 * resizeUV (process_input_frame.cu:22-81, srcX = x * (inW/outW), no
 * half-pixel shift, x2 = min(x1+1, inW-1)), then mergeYUV
 * (process_input_frame.cu:211-238): float3(Y*s, U*s, V*s), s = 1/(2^bits-1).
 * The bilinear blend a*(1-dx) + b*dx is restated as fmaf(b, dx, a*(1-dx));
 * at an exact 2x upsample every term is exact, so the form does not matter. */
int orc_decode_color(const uint16_t* y, const uint16_t* u, const uint16_t* v, int w, int h,
                     int bits, float* out) {
    if (!y || !u || !v || !out || w <= 0 || h <= 0 || bits < 1 || bits > 16) return RVSB_E_ARG;
    const int iw = w / 2, ih = h / 2;
    const float color_scale = 1.0f / (float)max_level(bits);
    const float scale_x = (float)iw / w, scale_y = (float)ih / h;
    for (int yy = 0; yy < h; ++yy)
        for (int xx = 0; xx < w; ++xx) {
            float src_x = xx * scale_x, src_y = yy * scale_y;
            int x1 = (int)src_x, y1 = (int)src_y;
            int x2 = (int)std::fmin((float)(x1 + 1), (float)(iw - 1));
            int y2 = (int)std::fmin((float)(y1 + 1), (float)(ih - 1));
            float dx = src_x - x1, dy = src_y - y1;
            float uv[2];
            const uint16_t* planes[2] = {u, v};
            for (int c = 0; c < 2; ++c) {
                const uint16_t* p = planes[c];
                float a = p[y1 * iw + x1], b = p[y1 * iw + x2];
                float cc = p[y2 * iw + x1], d = p[y2 * iw + x2];
                float val1 = std::fmaf(b, dx, a * (1 - dx));
                float val2 = std::fmaf(d, dx, cc * (1 - dx));
                uv[c] = std::fmaf(val2, dy, val1 * (1 - dy));
            }
            size_t idx = (size_t)yy * w + xx;
            out[idx * 3 + 0] = (float)y[idx] * color_scale;
            out[idx * 3 + 1] = uv[0] * color_scale;
            out[idx * 3 + 2] = uv[1] * color_scale;
        }
    return RVSB_OK;
}

/* Depth loader: image_loading.cpp:147-211 read_depth_YUV and the normalize
 * kernel (process_input_frame.cu:346-385):
 *   d = raw * (1/(2^bits-1));
 *   z = far >= 1000 ? near / d : far*near / (near + d*(far-near));
 *   NaN if hasInvalidDepth && z == 0.
 * nvcc contracts near + d*(far-near) into one fused multiply-add. */
int orc_decode_depth(const uint16_t* raw, int w, int h, int bits, float near_, float far_,
                     int has_invalid, float* out) {
    if (!raw || !out || w <= 0 || h <= 0 || bits < 1 || bits > 16) return RVSB_E_ARG;
    const float scale = 1.0f / (float)max_level(bits);
    const size_t n = (size_t)w * h;
    for (size_t i = 0; i < n; ++i) {
        float d = (float)raw[i] * scale;
        float z;
        if (far_ >= 1000.f)
            z = near_ / d;
        else
            z = (far_ * near_) / std::fmaf(d, far_ - near_, near_);
        if (has_invalid && z == 0) z = kNaN;
        out[i] = z;
    }
    return RVSB_OK;
}

void orc_rotation_matrix(const float rot_deg[3], float R[9]) {
    M33 m = rotation_matrix(rot_deg);
    std::memcpy(R, m.m, sizeof(m.m));
}

int orc_relative_pose(const rvsb_camera* in, const rvsb_camera* vt, float R[9], float t[3]) {
    if (!in || !vt || !R || !t) return RVSB_E_ARG;
    M33 m;
    relative_pose(*in, *vt, m, t);
    std::memcpy(R, m.m, sizeof(m.m));
    return RVSB_OK;
}

/* Warp of one input view into the virtual camera: SynthesizedView.cpp:320-331
 *   generateImagePos   Unprojector.cpp:63-74, ERP rows EquirectangularUnprojector.cpp:87-98
 *   unproject          PerspectiveUnprojector.cpp:59-86 / EquirectangularUnprojector.cpp:55-85
 *   affine_transform   SynthesizedView.cpp:68-79 (R * x + t)
 *   project            PerspectiveProjector.cpp:59-87 / EquirectangularProjector.cpp:60-99
 * The Precision rescale (cv::transform by the identity at Precision 1) is a
 * no-op.  Outputs uv (H*W*2), virtual depth (H*W) and the wrapping flag. */
int orc_warp(const rvsb_camera* in, const rvsb_camera* vt, const float* depth, float* uv,
             float* vdepth, int* wrap) {
    if (!in || !vt || !depth || !uv || !vdepth) return RVSB_E_ARG;
    const int w = in->width, h = in->height;
    M33 R;
    float t[3];
    relative_pose(*in, *vt, R, t);

    // Unprojector parameters.
    const float radperdeg = 0.01745329252f;
    float phi0 = 0, theta0 = 0, dphi_du = 0, dtheta_dv = 0;
    if (in->projection == RVSB_PROJ_EQUIRECTANGULAR) {
        phi0 = radperdeg * in->hor_range[1];
        theta0 = radperdeg * in->ver_range[1];
        dphi_du = -radperdeg * (in->hor_range[1] - in->hor_range[0]) / w;
        dtheta_dv = -radperdeg * (in->ver_range[1] - in->ver_range[0]) / h;
    }
    // Projector parameters.
    const float degperrad = 57.295779513f;
    const int wo = vt->width, ho = vt->height;
    float u0 = 0, v0 = 0, du_dphi = 0, dv_dtheta = 0;
    if (vt->projection == RVSB_PROJ_EQUIRECTANGULAR) {
        u0 = wo * vt->hor_range[1] / (vt->hor_range[1] - vt->hor_range[0]);
        v0 = ho * vt->ver_range[1] / (vt->ver_range[1] - vt->ver_range[0]);
        du_dphi = -degperrad * wo / (vt->hor_range[1] - vt->hor_range[0]);
        dv_dtheta = -degperrad * ho / (vt->ver_range[1] - vt->ver_range[0]);
    }

    for (int i = 0; i < h; ++i)
        for (int j = 0; j < w; ++j) {
            size_t idx = (size_t)i * w + j;
            float pu = j + 0.5f, pv = i + 0.5f;
            float x[3];
            float d = depth[idx];
            if (in->projection == RVSB_PROJ_EQUIRECTANGULAR) {
                if (i == 0) pv = 1e-3f;
                if (i == h - 1) pv = h - 1e-3f;
                float phi = phi0 + dphi_du * pu;
                float theta = theta0 + dtheta_dv * pv;
                float ct = f_cos(theta);
                float a = ct * f_cos(phi), b = ct * f_sin(phi), c = f_sin(theta);
                x[0] = d * a;
                x[1] = d * b;
                x[2] = d * c;
            } else {
                if (d > 0.f) {
                    x[0] = d;
                    x[1] = -(d / in->focal[0]) * (pu - in->principle_point[0]);
                    x[2] = -(d / in->focal[1]) * (pv - in->principle_point[1]);
                } else {
                    x[0] = x[1] = x[2] = kNaN;
                }
            }
            float y[3];
            for (int r = 0; r < 3; ++r) {
                float s = 0.f;
                for (int k = 0; k < 3; ++k) s += R.m[r * 3 + k] * x[k];
                y[r] = s + t[r];
            }
            if (vt->projection == RVSB_PROJ_EQUIRECTANGULAR) {
                double s2 = 0.0;
                for (int k = 0; k < 3; ++k) {
                    double v = y[k];
                    s2 += v * v;
                }
                float radius = (float)std::sqrt(s2);
                vdepth[idx] = radius;
                float phi = f_atan2(y[1], y[0]);
                float theta = f_asin(y[2] / radius);
                uv[idx * 2 + 0] = u0 + du_dphi * phi;
                uv[idx * 2 + 1] = v0 + dv_dtheta * theta;
            } else {
                if (y[0] > 0.f) {
                    uv[idx * 2 + 0] = -vt->focal[0] * y[1] / y[0] + vt->principle_point[0];
                    uv[idx * 2 + 1] = -vt->focal[1] * y[2] / y[0] + vt->principle_point[1];
                    vdepth[idx] = y[0];
                } else {
                    uv[idx * 2 + 0] = uv[idx * 2 + 1] = kNaN;
                    vdepth[idx] = kNaN;
                }
            }
        }
    if (wrap) *wrap = (vt->projection == RVSB_PROJ_EQUIRECTANGULAR && vt->full_hor_range) ? 1 : 0;
    return RVSB_OK;
}

/* The camera-model steps one at a time, as the reference's unit tests
 * exercise them (unit_test.cpp:90-308): image positions
 * (Unprojector::generateImagePos, Unprojector.cpp:63-74 and
 * EquirectangularUnprojector.cpp:87-98), unprojection and projection of
 * the camera `c` (no pose).  uv: H*W*2, depth: H*W, xyz: H*W*3. */
int orc_image_pos(const rvsb_camera* c, float* uv) {
    if (!c || !uv) return RVSB_E_ARG;
    for (int i = 0; i < c->height; ++i)
        for (int j = 0; j < c->width; ++j) {
            size_t o = ((size_t)i * c->width + j) * 2;
            uv[o] = j + 0.5f;
            uv[o + 1] = i + 0.5f;
        }
    if (c->projection == RVSB_PROJ_EQUIRECTANGULAR)
        for (int j = 0; j < c->width; ++j) {
            uv[(size_t)j * 2 + 1] = 1e-3f;
            uv[((size_t)(c->height - 1) * c->width + j) * 2 + 1] = c->height - 1e-3f;
        }
    return RVSB_OK;
}

int orc_unproject(const rvsb_camera* c, const float* uv, const float* depth, float* xyz) {
    if (!c || !uv || !depth || !xyz) return RVSB_E_ARG;
    const int w = c->width, h = c->height;
    const float radperdeg = 0.01745329252f;
    for (size_t p = 0; p < (size_t)w * h; ++p) {
        const float u = uv[p * 2], v = uv[p * 2 + 1], d = depth[p];
        if (c->projection == RVSB_PROJ_EQUIRECTANGULAR) {
            const float phi0 = radperdeg * c->hor_range[1];
            const float theta0 = radperdeg * c->ver_range[1];
            const float dphi_du = -radperdeg * (c->hor_range[1] - c->hor_range[0]) / w;
            const float dtheta_dv = -radperdeg * (c->ver_range[1] - c->ver_range[0]) / h;
            const float phi = phi0 + dphi_du * u, theta = theta0 + dtheta_dv * v;
            const float ct = f_cos(theta);
            const float a = ct * f_cos(phi), b = ct * f_sin(phi), cc = f_sin(theta);
            xyz[p * 3] = d * a;
            xyz[p * 3 + 1] = d * b;
            xyz[p * 3 + 2] = d * cc;
        } else if (d > 0.f) {
            xyz[p * 3] = d;
            xyz[p * 3 + 1] = -(d / c->focal[0]) * (u - c->principle_point[0]);
            xyz[p * 3 + 2] = -(d / c->focal[1]) * (v - c->principle_point[1]);
        } else {
            xyz[p * 3] = xyz[p * 3 + 1] = xyz[p * 3 + 2] = kNaN;
        }
    }
    return RVSB_OK;
}

int orc_project(const rvsb_camera* c, const float* xyz, float* uv, float* depth, int* wrap) {
    if (!c || !xyz || !uv || !depth) return RVSB_E_ARG;
    const int w = c->width, h = c->height;
    const float degperrad = 57.295779513f;
    for (size_t p = 0; p < (size_t)w * h; ++p) {
        const float* y = xyz + p * 3;
        if (c->projection == RVSB_PROJ_EQUIRECTANGULAR) {
            const float u0 = w * c->hor_range[1] / (c->hor_range[1] - c->hor_range[0]);
            const float v0 = h * c->ver_range[1] / (c->ver_range[1] - c->ver_range[0]);
            const float du_dphi = -degperrad * w / (c->hor_range[1] - c->hor_range[0]);
            const float dv_dtheta = -degperrad * h / (c->ver_range[1] - c->ver_range[0]);
            double s2 = 0.0;
            for (int k = 0; k < 3; ++k) s2 += (double)y[k] * (double)y[k];
            const float radius = (float)std::sqrt(s2);
            depth[p] = radius;
            const float phi = f_atan2(y[1], y[0]);
            const float theta = f_asin(y[2] / radius);
            uv[p * 2] = u0 + du_dphi * phi;
            uv[p * 2 + 1] = v0 + dv_dtheta * theta;
        } else if (y[0] > 0.f) {
            uv[p * 2] = -c->focal[0] * y[1] / y[0] + c->principle_point[0];
            uv[p * 2 + 1] = -c->focal[1] * y[2] / y[0] + c->principle_point[1];
            depth[p] = y[0];
        } else {
            uv[p * 2] = uv[p * 2 + 1] = depth[p] = kNaN;
        }
    }
    if (wrap) *wrap = (c->projection == RVSB_PROJ_EQUIRECTANGULAR && c->full_hor_range) ? 1 : 0;
    return RVSB_OK;
}

/* cv::norm(Vec2f a, Vec2f b) as valid_tri uses it (transform.cpp:63-65). */
double orc_edge_norm(const float* a, const float* b) {
    double s = 0.0;
    for (int k = 0; k < 2; ++k) {
        double v = (double)(a[k] - b[k]);
        s += v * v;
    }
    return std::sqrt(s);
}

}  // extern "C"

namespace {

// transform.cpp:62-75 valid_tri with cv::norm(Vec2f, Vec2f) = sqrt(sum (double)(a-b)^2).
float valid_tri(const float* A, const float* B, const float* C, float rescale) {
    auto nrm = [](const float* p, const float* q) {
        double s = 0.0;
        for (int k = 0; k < 2; ++k) {
            double v = (double)(p[k] - q[k]);
            s += v * v;
        }
        return std::sqrt(s);
    };
    double dab = nrm(A, B), dac = nrm(A, C), dbc = nrm(B, C);
    float stretch = static_cast<float>(std::max(dbc, std::max(dab, dac)));
    stretch /= rescale;
    float quality = 10000.f - 1000.f * stretch;
    quality = smax(1.f, quality);
    quality = smin(10000.f, quality);
    return quality;
}

struct RasterState {
    int w, wo, ho;
    const float* color;   // input colour H*W*3
    const float* vdepth;  // virtual depth H*W (also the prolongation mask source)
    const float* uv;      // H*W*2
    float* res;           // output colour Ho*Wo*3
    float* new_depth;     // Ho*Wo
    float* shape;         // Ho*Wo (triangle validity)
    uint8_t* new_prol;    // Ho*Wo, initialised to 1
};

// transform.cpp:77-145 colorize_triangle.
void colorize_triangle(RasterState& st, int ax, int ay, int bx, int by, int cx, int cy) {
    const size_t ia = (size_t)ay * st.w + ax, ib = (size_t)by * st.w + bx,
                 ic = (size_t)cy * st.w + cx;
    const float* A = st.uv + ia * 2;
    const float* B = st.uv + ib * 2;
    const float* C = st.uv + ic * 2;
    float den = (B[1] - C[1]) * (A[0] - C[0]) + (C[0] - B[0]) * (A[1] - C[1]);
    if (den <= 0.f) return;
    float triangle_validity = valid_tri(A, B, C, g_precision);
    if (triangle_validity == 0.f) return;

    int Xmin = imax(0, cvt_trunc_i32(std::floor(smin(smin(A[0], B[0]), C[0]))));
    int Ymin = imax(0, cvt_trunc_i32(std::floor(smin(smin(A[1], B[1]), C[1]))));
    int Xmax = imin(st.wo - 1, cvt_trunc_i32(std::ceil(smax(smax(A[0], B[0]), C[0]))));
    int Ymax = imin(st.ho - 1, cvt_trunc_i32(std::ceil(smax(smax(A[1], B[1]), C[1]))));
    if (Ymin > Ymax || Xmin > Xmax) return;

    const float* colA = st.color + ia * 3;
    const float* colB = st.color + ib * 3;
    const float* colC = st.color + ic * 3;
    float dA = st.vdepth[ia], dB = st.vdepth[ib], dC = st.vdepth[ic];
    // depth_prologation_mask = input_depth > 0 (transform.cpp:152).
    bool prol = (dA > 0.f) || (dB > 0.f) || (dC > 0.f);

    for (int y = Ymin; y <= Ymax; ++y)
        for (int x = Xmin; x <= Xmax; ++x) {
            const float offset = 0.5f;
            float lambda_1 = ((B[1] - C[1]) * ((float)x + offset - C[0]) +
                              (C[0] - B[0]) * ((float)y + offset - C[1])) / den;
            float lambda_2 = ((C[1] - A[1]) * ((float)x + offset - C[0]) +
                              (A[0] - C[0]) * ((float)y + offset - C[1])) / den;
            float lambda_3 = 1.f - lambda_1 - lambda_2;
            const float eps = 1e-6f;
            if (lambda_1 >= -eps && lambda_2 >= -eps && lambda_3 >= -eps) {
                float col[3];
                for (int k = 0; k < 3; ++k)
                    col[k] = colA[k] * lambda_1 + colB[k] * lambda_2 + colC[k] * lambda_3;
                float d = dA * lambda_1 + dB * lambda_2 + dC * lambda_3;
                size_t o = (size_t)y * st.wo + x;
                float& new_d = st.new_depth[o];
                float& shape = st.shape[o];
                float ratio = d / new_d;
                bool is_valid = ratio * ratio * ratio * shape < triangle_validity;
                uint8_t& new_prol = st.new_prol[o];
                if ((is_valid || new_prol) && !prol) {
                    new_d = d;
                    new_prol = 0;
                    shape = triangle_validity;
                    for (int k = 0; k < 3; ++k) st.res[o * 3 + k] = col[k];
                } else if (is_valid && new_prol && prol) {
                    new_d = d;
                    shape = triangle_validity;
                    for (int k = 0; k < 3; ++k) st.res[o * 3 + k] = col[k];
                }
            }
        }
}

}  // namespace

extern "C" {

/* transform_trianglesMethod (transform.cpp:148-181).  Outputs colour
 * (zeros where uncovered), depth (+inf where uncovered) and the triangle
 * validity map (0 where uncovered), all Ho*Wo. */
int orc_raster(const float* color, const float* vdepth, const float* uv, int w, int h, int wo,
               int ho, int wrap, float* out_color, float* out_depth, float* out_validity) {
    if (!color || !vdepth || !uv || !out_color || !out_depth || !out_validity) return RVSB_E_ARG;
    const size_t no = (size_t)wo * ho;
    std::fill(out_color, out_color + no * 3, 0.f);
    std::fill(out_depth, out_depth + no, kInf);
    std::fill(out_validity, out_validity + no, 0.f);
    std::vector<uint8_t> prol(no, 1);
    RasterState st{w, wo, ho, color, vdepth, uv, out_color, out_depth, out_validity, prol.data()};
    auto D = [&](int i, int j) { return vdepth[(size_t)i * w + j]; };
    auto U = [&](int i, int j) { return uv[((size_t)i * w + j) * 2]; };
    for (int i = 0; i < h - 1; ++i)
        for (int j = 0; j < w - 1; ++j) {
            if (D(i, j + 1) > 0.f && D(i + 1, j) > 0.f && U(i, j + 1) > 0.f && U(i + 1, j) > 0.f) {
                if (D(i, j) > 0.f && U(i, j) > 0.f)
                    colorize_triangle(st, j, i, j + 1, i, j, i + 1);
                if (D(i + 1, j + 1) > 0.f && U(i + 1, j + 1) > 0.f)
                    colorize_triangle(st, j + 1, i + 1, j, i + 1, j + 1, i);
                if (wrap && j == 0) {
                    colorize_triangle(st, w - 1, i, 0, i, w - 1, i + 1);
                    colorize_triangle(st, 0, i + 1, w - 1, i + 1, 0, i);
                }
            }
        }
    return RVSB_OK;
}

/* Incremental blending of BlendedViewSimple::blendBasicMode
 * (BlendedView.cpp:180-212) with blend_img (blending.cpp:310-369), including
 * its two weight buckets and the depth-prolongation masks
 * (View::get_depth_mask, View.cpp:192-196).  Views are blended in order:
 * the first is assigned as is, every later one is blended into the
 * accumulator.  color_i: Ho*Wo*3, quality_i = validity_i / depth_i and
 * depth_i: Ho*Wo.  Outputs the blended colour and quality. */
}  // extern "C"

/* One step of the incremental blend: view v (colour, quality, depth) into
 * the accumulator (colour, quality, depth-prolongation mask). */
static void blend_step(int v, const float* vcol, const float* vq, const float* vd, size_t no, float exponent,
                       float* out_color, float* out_quality, uint8_t* acc_mask) {
    if (v == 0) {
        std::memcpy(out_color, vcol, no * 3 * sizeof(float));
        std::memcpy(out_quality, vq, no * sizeof(float));
        for (size_t p = 0; p < no; ++p) acc_mask[p] = vd[p] > 0.f;
        return;
    }
    const float empty[3] = {0.f, 1.f, 0.f};
    if (exponent < 0) {
        // blend_img_by_max (blending.cpp:293-308) over {accumulator, view}:
        // start from the empty colour and quality 0, then each image
        // replaces the result where its quality is strictly larger.
        for (size_t p = 0; p < no; ++p) {
            float c[3] = {empty[0], empty[1], empty[2]};
            float q = 0.f;
            bool prol = false;
            if (out_quality[p] > q) {
                for (int k = 0; k < 3; ++k) c[k] = out_color[p * 3 + k];
                q = out_quality[p];
                prol = acc_mask[p] != 0;
            }
            if (vq[p] > q) {
                for (int k = 0; k < 3; ++k) c[k] = vcol[p * 3 + k];
                q = vq[p];
                prol = vd[p] > 0.f;
            }
            for (int k = 0; k < 3; ++k) out_color[p * 3 + k] = c[k];
            out_quality[p] = q;
            acc_mask[p] = prol;
        }
        return;
    }
    for (size_t p = 0; p < no; ++p) {
        const float* cols[2] = {out_color + p * 3, vcol + p * 3};
        float quals[2] = {out_quality[p], vq[p]};
        bool prolong[2] = {acc_mask[p] != 0, vd[p] > 0.f};
        float sumWeights = 0.0f;
        float finalColor[3] = {0, 0, 0};
        float inpaintedDepthColor[3] = {0, 0, 0};
        float inpaintedDepthSumWeights = 0.0f;
        for (int i = 0; i < 2; ++i) {
            float quality = quals[i];
            bool isValidDepth = quals[i] > 0 && !prolong[i];
            if (quality > 0 && isValidDepth) {
                quality = powf(quality, exponent);
                sumWeights += quality;
                for (int k = 0; k < 3; ++k) finalColor[k] += quality * cols[i][k];
            } else if (quality > 0 && quals[i] > 0) {
                quality = powf(quality, exponent);
                inpaintedDepthSumWeights += quality;
                for (int k = 0; k < 3; ++k) inpaintedDepthColor[k] += quality * cols[i][k];
            }
        }
        float outc[3];
        float outq;
        bool outprol;
        if (sumWeights == 0) {
            if (inpaintedDepthSumWeights == 0.0) {
                for (int k = 0; k < 3; ++k) outc[k] = empty[k];
                outprol = true;
                outq = 0.0f;
            } else {
                float inv = 1.f / inpaintedDepthSumWeights;
                for (int k = 0; k < 3; ++k) outc[k] = inpaintedDepthColor[k] * inv;
                outprol = true;
                outq = powf(inpaintedDepthSumWeights, 1.0f / exponent);
            }
        } else {
            float inv = 1.f / sumWeights;
            for (int k = 0; k < 3; ++k) outc[k] = finalColor[k] * inv;
            outprol = false;
            outq = powf(sumWeights, 1.0f / exponent);
        }
        for (int k = 0; k < 3; ++k) out_color[p * 3 + k] = outc[k];
        out_quality[p] = outq;
        acc_mask[p] = outprol;
    }
}

extern "C" {

int orc_blend(int n, const float* const* colors, const float* const* qualities,
              const float* const* depths, int wo, int ho, float exponent, float* out_color,
              float* out_quality) {
    if (n <= 0 || !colors || !qualities || !depths || !out_color || !out_quality) return RVSB_E_ARG;
    const size_t no = (size_t)wo * ho;
    std::vector<uint8_t> acc_mask(no);  // m_depth_mask
    for (int v = 0; v < n; ++v)
        blend_step(v, colors[v], qualities[v], depths[v], no, exponent, out_color, out_quality, acc_mask.data());
    return RVSB_OK;
}

/* Inpainting by nearest source: View::get_inpaint_mask (View.cpp:198-203),
 * inpaint_color's compute_by_nearest branch (inpainting.cpp:179-199) and
 * compute_nearest (inpainting.cpp:104-136): alternating column-major
 * Gauss-Seidel sweeps over a (x, y, dist) map until no change, visiting the
 * neighbours (x-1,y), (x,y-1), (x,y+1), (x+1,y) with strict improvement.
 * out_color may alias color.  out_source (optional, Ho*Wo*2 int32) receives
 * the (x, y) each pixel copies (itself for non-holes).  Returns the number
 * of sweeps through *n_sweeps when given. */
int orc_inpaint(const float* color, const float* quality, int w, int h, float* out_color,
                int32_t* out_source, int* n_sweeps) {
    if (!color || !quality || !out_color || w <= 0 || h <= 0) return RVSB_E_ARG;
    const size_t n = (size_t)w * h;
    std::vector<int32_t> map(n * 3);
    std::vector<uint8_t> mask(n);
    for (size_t p = 0; p < n; ++p) mask[p] = !(quality[p] > 0.f);
    for (int x = 0; x < w; x++)
        for (int y = 0; y < h; y++) {
            size_t p = (size_t)y * w + x;
            map[p * 3 + 0] = x;
            map[p * 3 + 1] = y;
            map[p * 3 + 2] = mask[p] ? w + h : 0;
        }
    bool change = true, odd = true;
    int sweeps = 0;
    while (change) {
        odd = !odd;
        change = false;
        ++sweeps;
        int A = 0, B = 1, C = 0, D = 1;
        if (odd) {
            A = w - 1; B = -1;
            C = h - 1; D = -1;
        }
        for (int x = A; x < w && x > -1; x += B)
            for (int y = C; y < h && y > -1; y += D) {
                size_t p = (size_t)y * w + x;
                if (map[p * 3 + 2] > 0) {
                    for (int i = std::max(x - 1, 0); i < std::min(x + 2, w); ++i)
                        for (int j = std::max(y - 1, 0); j < std::min(y + 2, h); ++j) {
                            if (std::abs(x - i) + std::abs(y - j) == 1) {
                                size_t q = (size_t)j * w + i;
                                if (map[q * 3 + 2] + 1 < map[p * 3 + 2]) {
                                    map[p * 3 + 0] = map[q * 3 + 0];
                                    map[p * 3 + 1] = map[q * 3 + 1];
                                    map[p * 3 + 2] = map[q * 3 + 2] + 1;
                                    change = true;
                                }
                            }
                        }
                }
            }
    }
    if (out_color != color) std::memcpy(out_color, color, n * 3 * sizeof(float));
    // The source pixel of a hole is never a hole, so reading from the
    // partly-filled image equals reading from the input.
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            size_t p = (size_t)y * w + x;
            if (mask[p]) {
                size_t s = (size_t)map[p * 3 + 1] * w + map[p * 3 + 0];
                for (int k = 0; k < 3; ++k) out_color[p * 3 + k] = out_color[s * 3 + k];
            }
        }
    if (out_source)
        for (size_t p = 0; p < n; ++p) {
            out_source[p * 2 + 0] = map[p * 3 + 0];
            out_source[p * 2 + 1] = map[p * 3 + 1];
        }
    if (n_sweeps) *n_sweeps = sweeps;
    return RVSB_OK;
}

/* write_color (image_writing.cpp:182-203): quantization
 * (image_writing.cpp:142-180: static_cast<ushort>(v * max_level)), then
 * write_color_YUV (image_writing.cpp:72-89): Y as is, U and V through
 * cv::resize(0.5, 0.5, INTER_LINEAR) of the quantised uint16 planes, which
 * at an exact 2x reduction is the rounded 2x2 mean (quarter_round).
 * out: Y (w*h) then U and V ((w/2)*(h/2) each).  w and h must be even. */
int orc_write_yuv420(const float* color, int w, int h, int bits, uint16_t* out) {
    if (!color || !out || w <= 0 || h <= 0 || (w & 1) || (h & 1) || bits < 9 || bits > 16)
        return RVSB_E_ARG;
    const unsigned max_val = max_level(bits);
    const size_t n = (size_t)w * h;
    std::vector<uint16_t> q(n * 3);
    for (size_t i = 0; i < n * 3; ++i) q[i] = static_cast<uint16_t>(color[i] * max_val);
    for (size_t i = 0; i < n; ++i) out[i] = q[i * 3];
    const int cw = w / 2, ch = h / 2;
    for (int c = 1; c <= 2; ++c) {
        uint16_t* dst = out + n + (size_t)(c - 1) * cw * ch;
        for (int y = 0; y < ch; ++y)
            for (int x = 0; x < cw; ++x) {
                size_t p00 = ((size_t)(2 * y) * w + 2 * x) * 3 + c;
                size_t p01 = p00 + 3;
                size_t p10 = p00 + (size_t)w * 3;
                size_t p11 = p10 + 3;
                unsigned s = (unsigned)q[p00] + q[p01] + q[p10] + q[p11];
                dst[(size_t)y * cw + x] = quarter_round(s);
            }
    }
    return RVSB_OK;
}

/* calcBlurring of one channel (blending.cpp:62-105): box mean of the
 * masked, finite values over [x - rad, x + rad] x [y - rad, y + rad]
 * clipped to the image, from an integral image in double
 * (IntegralImage2D<float, 1>, IntegralImage2D.h:735-770: the recurrence
 * I(y+1, x+1) = I(y, x+1) + I(y+1, x) - I(y, x) + v); the window sum is
 * truncated to an integer before the division by the count; 0 outside the
 * mask.  src: channel 0 of a 3-channel image. */
static void blur_channel0(const float* src, const uint8_t* mask, int w, int h, int rad, float* out) {
    const size_t W1 = (size_t)w + 1;
    std::vector<double> I(W1 * (h + 1), 0.0);
    std::vector<unsigned> C(W1 * (h + 1), 0u);
    for (int y = 0; y < h; ++y) {
        double* prev = &I[(size_t)y * W1];
        double* cur = prev + W1;
        unsigned* cprev = &C[(size_t)y * W1];
        unsigned* ccur = cprev + W1;
        cur[0] = 0.0;
        ccur[0] = 0;
        for (int x = 0; x < w; ++x) {
            cur[x + 1] = prev[x + 1] + cur[x] - prev[x];
            ccur[x + 1] = cprev[x + 1] + ccur[x] - cprev[x];
            const float v = src[((size_t)y * w + x) * 3];
            if (mask[(size_t)y * w + x] == 255 && v == v && std::isfinite(v)) {
                cur[x + 1] += v;
                ccur[x + 1] += 1;
            }
        }
    }
    for (int i = 0; i < h; ++i)
        for (int j = 0; j < w; ++j) {
            float& o = out[(size_t)i * w + j];
            if (mask[(size_t)i * w + j] == 0) {
                o = 0.f;
                continue;
            }
            const int sx = std::max(0, j - rad), sy = std::max(0, i - rad);
            const int ex = std::min(j - rad + 2 * rad + 1, w), ey = std::min(i - rad + 2 * rad + 1, h);
            const size_t ul = (size_t)sy * W1 + sx, ur = (size_t)sy * W1 + ex;
            const size_t ll = (size_t)ey * W1 + sx, lr = (size_t)ey * W1 + ex;
            const unsigned cnt = C[lr] + C[ul] - C[ur] - C[ll];
            const unsigned sum = (unsigned)(int)(I[lr] + I[ul] - I[ur] - I[ll]);
            o = cnt > 0 ? float(float(sum) / float(cnt)) : 0.f;
        }
}

/* cv::resize(src, dst, dsize) with INTER_LINEAR on a 3-channel float image
 * (imgproc resize.cpp): an exact 2x reduction takes the area fast path,
 * ((a + b) + c + d) * 0.25 over each 2x2 block; otherwise bilinear with
 * source coordinate (d + 0.5) * scale - 0.5, weights (1 - f, f) in float,
 * coordinates clamped to the first and last pixel (weight 0 beyond), a
 * horizontal pass per source row and a vertical pass. */
static void resize_linear(const float* src, int ws, int hs, int cn, float* dst, int wd, int hd) {
    const double scale_x = 1.0 / ((double)wd / ws), scale_y = 1.0 / ((double)hd / hs);
    const int iscale_x = (int)std::lrint(scale_x), iscale_y = (int)std::lrint(scale_y);
    const bool area_fast = std::fabs(scale_x - iscale_x) < 2.220446049250313e-16 &&
                           std::fabs(scale_y - iscale_y) < 2.220446049250313e-16;
    if (area_fast && iscale_x == 2 && iscale_y == 2) {
        for (int y = 0; y < hd; ++y)
            for (int x = 0; x < wd; ++x)
                for (int k = 0; k < cn; ++k) {
                    const float a = src[((size_t)(2 * y) * ws + 2 * x) * cn + k];
                    const float b = src[((size_t)(2 * y) * ws + 2 * x + 1) * cn + k];
                    const float c = src[((size_t)(2 * y + 1) * ws + 2 * x) * cn + k];
                    const float d = src[((size_t)(2 * y + 1) * ws + 2 * x + 1) * cn + k];
                    dst[((size_t)y * wd + x) * cn + k] = (((a + b) + c) + d) * 0.25f;
                }
        return;
    }
    auto coord = [](int d, double scale, int n, int& s0, float& f) {
        f = (float)((d + 0.5) * scale - 0.5);
        int s = (int)std::floor(f);
        f -= (float)s;
        if (s < 0) {
            f = 0.f;
            s = 0;
        }
        if (s >= n - 1) {
            f = 0.f;
            s = n - 1;
        }
        s0 = s;
    };
    std::vector<float> rows((size_t)hs * wd * cn);
    for (int x = 0; x < wd; ++x) {
        int sx;
        float fx;
        coord(x, scale_x, ws, sx, fx);
        const float a0 = 1.f - fx, a1 = fx;
        const int sx1 = std::min(sx + 1, ws - 1);
        for (int y = 0; y < hs; ++y)
            for (int k = 0; k < cn; ++k)
                rows[((size_t)y * wd + x) * cn + k] =
                    src[((size_t)y * ws + sx) * cn + k] * a0 + src[((size_t)y * ws + sx1) * cn + k] * a1;
    }
    for (int y = 0; y < hd; ++y) {
        int sy;
        float fy;
        coord(y, scale_y, hs, sy, fy);
        const float b0 = 1.f - fy, b1 = fy;
        const int sy1 = std::min(sy + 1, hs - 1);
        for (int x = 0; x < wd; ++x)
            for (int k = 0; k < cn; ++k)
                dst[((size_t)y * wd + x) * cn + k] =
                    rows[((size_t)sy * wd + x) * cn + k] * b0 + rows[((size_t)sy1 * wd + x) * cn + k] * b1;
    }
}

static void resize_linear3(const float* src, int ws, int hs, float* dst, int wd, int hd) {
    resize_linear(src, ws, hs, 3, dst, wd, hd);
}

/* cv::resize(src, dst, dsize, 0, 0, INTER_NEAREST) of a one-byte image
 * (imgproc resize.cpp resizeNN): destination x reads source
 * min(floor(x * (1 / (wd / ws))), ws - 1), the ratio and product in double;
 * the same for y.  Pinned against cv2 by tests/golden. */
static void resize_nearest_u8(const uint8_t* src, int ws, int hs, uint8_t* dst, int wd, int hd) {
    const double ifx = 1.0 / ((double)wd / ws), ify = 1.0 / ((double)hd / hs);
    for (int y = 0; y < hd; ++y) {
        const int sy = std::min((int)std::floor(y * ify), hs - 1);
        for (int x = 0; x < wd; ++x) {
            const int sx = std::min((int)std::floor(x * ifx), ws - 1);
            dst[(size_t)y * wd + x] = src[(size_t)sy * ws + sx];
        }
    }
}

extern "C" void orc_resize_nearest_u8(const uint8_t* src, int ws, int hs, uint8_t* dst, int wd, int hd) {
    resize_nearest_u8(src, ws, hs, dst, wd, hd);
}

extern "C" void orc_resize_linear3(const float* src, int ws, int hs, float* dst, int wd, int hd) {
    resize_linear3(src, ws, hs, dst, wd, hd);
}

/* Depth of the blended view (BlendedView.cpp:205-208): the first view's
 * depth, then at every later view the view's depth where its quality is
 * larger than the accumulator's quality before the blend; validity is the
 * running maximum (cv::max).  acc_q_before: the accumulator's quality
 * before view v (view 0: unused). */
static void blend_depth_validity(int v, const float* acc_q_before, const float* vq, const float* vd,
                                 const float* vv, size_t no, float* depth, float* validity) {
    for (size_t p = 0; p < no; ++p) {
        if (v == 0) {
            depth[p] = vd[p];
            validity[p] = vv[p];
        } else {
            if (vq[p] > acc_q_before[p]) depth[p] = vd[p];
            validity[p] = std::max(validity[p], vv[p]);
        }
    }
}

/* write_maskedDepth (image_writing.cpp:237-268) for integer bit depths:
 * normalised disparity near / depth (far >= 1000) or
 * (far * near / depth - near) / (far - near), masked pixels set to 0, then
 * convertTo(CV_16U, 2^bits - 1): rounded to nearest (ties to even) and
 * saturated, NaN to 0. */
static uint16_t encode_depth(float depth, const rvsb_camera* vt, bool masked) {
    const float near_ = vt->depth_range[0], far_ = vt->depth_range[1];
    float d;
    if (far_ >= 1000.f)
        d = near_ / depth;
    else
        d = ((far_ * near_) / depth - near_) / (far_ - near_);
    if (masked) d = 0.f;
    const float v = d * (float)max_level(vt->bit_depth_depth);
    if (std::isnan(v)) return 0;
    const float r = std::nearbyint(v);
    return (uint16_t)std::min(65535.f, std::max(0.f, r));
}

/* One output frame of Pipeline::computeView in CPU mode
 * (Pipeline.cpp:169-336): for every input view in order, load, warp,
 * raster (SynthetisedViewTriangle::transform, SynthesizedView.cpp:428-441:
 * quality = validity / depth) and blend; then inpaint and write.
 * planes: n entries of {y, u, v, depth} host pointers.  Optional outputs:
 * out_quality (blended quality, Ho*Wo), out_color (blended colour before
 * inpainting, Ho*Wo*3).  orc_synthesize_aux adds the outputs of
 * Pipeline.cpp:303-336 (all optional): the validity mask (Ho*Wo bytes, 255
 * where the blended validity is not above `threshold`), the masked colour
 * (YUV420 of the inpainted colour with masked pixels set to 0.5), the
 * blended depth and the masked depth (Ho*Wo uint16 each, encoded with the
 * virtual camera's depth range and bit depth). */
int orc_synthesize_aux(int n, const rvsb_camera* cams, const rvsb_view_planes* planes,
                       const rvsb_camera* vt, float exponent, uint16_t* out_yuv, float* out_quality,
                       float* out_color, float threshold, uint8_t* out_mask, uint16_t* out_masked_yuv,
                       uint16_t* out_depth, uint16_t* out_masked_depth) {
    if (n <= 0 || !cams || !planes || !vt || !out_yuv) return RVSB_E_ARG;
    // Precision: rasterise at (int(0.5 + W * P), int(0.5 + H * P))
    // (SynthesizedView.cpp:325-333); the colour is resized to W x H when
    // written (image_writing.cpp:188-190).
    const float P = g_precision;
    const bool rescale = P != 1.f;
    // MaskedOutputFiles at Precision != 1: the reference sets the raster-sized
    // colour with the mask resized to the output size (Pipeline.cpp:314-318),
    // which OpenCV's setTo rejects (the sizes differ).
    if (rescale && out_masked_yuv) return RVSB_E_UNSUPPORTED;
    const int wo = rescale ? (int)(0.5f + vt->width * P) : vt->width;
    const int ho = rescale ? (int)(0.5f + vt->height * P) : vt->height;
    const float sxu = (float)wo / vt->width, syv = (float)ho / vt->height;
    const size_t no = (size_t)wo * ho;
    std::vector<std::vector<float>> vcol(n), vq(n), vd(n), vv(n);
    for (int v = 0; v < n; ++v) {
        const rvsb_camera& c = cams[v];
        const size_t ni = (size_t)c.width * c.height;
        std::vector<float> col(ni * 3), dep(ni), uv(ni * 2), vdep(ni);
        int rc = orc_decode_color(planes[v].y, planes[v].u, planes[v].v, c.width, c.height,
                                  c.bit_depth_color, col.data());
        if (rc) return rc;
        rc = orc_decode_depth(planes[v].depth, c.width, c.height, c.bit_depth_depth,
                              c.depth_range[0], c.depth_range[1], c.has_invalid_depth, dep.data());
        if (rc) return rc;
        int wrap = 0;
        orc_warp(&c, vt, dep.data(), uv.data(), vdep.data(), &wrap);
        if (rescale)  // cv::transform with Matx22f(sx, 0, 0, sy)
            for (size_t p = 0; p < ni; ++p) {
                const float u = uv[p * 2], w = uv[p * 2 + 1];
                uv[p * 2] = sxu * u + 0.f * w;
                uv[p * 2 + 1] = 0.f * u + syv * w;
            }
        vcol[v].resize(no * 3);
        vd[v].resize(no);
        vq[v].resize(no);
        vv[v].resize(no);
        orc_raster(col.data(), vdep.data(), uv.data(), c.width, c.height, wo, ho, wrap,
                   vcol[v].data(), vd[v].data(), vv[v].data());
        for (size_t p = 0; p < no; ++p) vq[v][p] = vv[v][p] / vd[v][p];
    }
    // Blend view by view; the accumulator's quality before each view feeds
    // the depth rule.
    std::vector<float> bc(no * 3), bq(no), prev_q(no), depth(no), validity(no);
    std::vector<uint8_t> acc_mask(no);
    const bool want_aux = out_mask || out_masked_yuv || out_depth || out_masked_depth;
    // Multispectral: a second (high-frequency) blender beside the first.
    std::vector<float> hc, hq;
    std::vector<uint8_t> hmask;
    std::vector<float> low, high, blur;
    if (g_ms_on) {
        hc.resize(no * 3);
        hq.resize(no);
        hmask.resize(no);
        low.resize(no * 3);
        high.resize(no * 3);
        blur.resize(no);
    }
    for (int v = 0; v < n; ++v) {
        if (want_aux) prev_q = bq;
        if (g_ms_on) {
            // split_frequencies (blending.cpp:371-395), YUV: blur Y only;
            // low = (blur(Y), U, V), high = colour - low.
            std::vector<uint8_t> m(no);
            for (size_t p = 0; p < no; ++p) m[p] = vq[v][p] > 0.f ? 255 : 0;
            blur_channel0(vcol[v].data(), m.data(), wo, ho, std::max(wo, ho) / 20, blur.data());
            for (size_t p = 0; p < no; ++p) {
                low[p * 3 + 0] = blur[p];
                low[p * 3 + 1] = vcol[v][p * 3 + 1];
                low[p * 3 + 2] = vcol[v][p * 3 + 2];
                for (int k = 0; k < 3; ++k) high[p * 3 + k] = vcol[v][p * 3 + k] - low[p * 3 + k];
            }
            blend_step(v, low.data(), vq[v].data(), vd[v].data(), no, g_ms_low, bc.data(), bq.data(),
                       acc_mask.data());
            blend_step(v, high.data(), vq[v].data(), vd[v].data(), no, g_ms_high, hc.data(), hq.data(),
                       hmask.data());
        } else {
            blend_step(v, vcol[v].data(), vq[v].data(), vd[v].data(), no, exponent, bc.data(), bq.data(),
                       acc_mask.data());
        }
        if (want_aux)
            blend_depth_validity(v, prev_q.data(), vq[v].data(), vd[v].data(), vv[v].data(), no, depth.data(),
                                 validity.data());
    }
    if (g_ms_on)
        for (size_t p = 0; p < no * 3; ++p) bc[p] = bc[p] + hc[p];
    if (out_quality) std::memcpy(out_quality, bq.data(), no * sizeof(float));
    if (out_color) std::memcpy(out_color, bc.data(), no * 3 * sizeof(float));
    std::vector<float> filled(no * 3);
    orc_inpaint(bc.data(), bq.data(), wo, ho, filled.data(), nullptr, nullptr);
    if (rescale) {
        std::vector<float> small((size_t)vt->width * vt->height * 3);
        resize_linear3(filled.data(), wo, ho, small.data(), vt->width, vt->height);
        int rc = orc_write_yuv420(small.data(), vt->width, vt->height, vt->bit_depth_color, out_yuv);
        if (rc || !want_aux) return rc;
        // Pipeline.cpp:303-336 at Precision != 1: the validity mask resized
        // with INTER_NEAREST, the blended depth with INTER_LINEAR, both to the
        // output size before they are written.
        const int W = vt->width, H = vt->height;
        const size_t nw = (size_t)W * H;
        std::vector<uint8_t> rmask(no), mask(nw);
        for (size_t p = 0; p < no; ++p) rmask[p] = (validity[p] > threshold) ? 0 : 255;
        resize_nearest_u8(rmask.data(), wo, ho, mask.data(), W, H);
        std::vector<float> dsmall(nw);
        resize_linear(depth.data(), wo, ho, 1, dsmall.data(), W, H);
        if (out_mask) std::memcpy(out_mask, mask.data(), nw);
        if (out_depth)
            for (size_t p = 0; p < nw; ++p) out_depth[p] = encode_depth(dsmall[p], vt, false);
        if (out_masked_depth)
            for (size_t p = 0; p < nw; ++p) out_masked_depth[p] = encode_depth(dsmall[p], vt, mask[p] != 0);
        return RVSB_OK;
    }
    int rc = orc_write_yuv420(filled.data(), wo, ho, vt->bit_depth_color, out_yuv);
    if (rc) return rc;
    std::vector<uint8_t> mask(no);
    for (size_t p = 0; p < no; ++p) mask[p] = (validity[p] > threshold) ? 0 : 255;
    if (out_mask) std::memcpy(out_mask, mask.data(), no);
    if (out_masked_yuv) {
        std::vector<float> masked = filled;
        for (size_t p = 0; p < no; ++p)
            if (mask[p])
                for (int k = 0; k < 3; ++k) masked[p * 3 + k] = 0.5f;
        rc = orc_write_yuv420(masked.data(), wo, ho, vt->bit_depth_color, out_masked_yuv);
        if (rc) return rc;
    }
    if (out_depth)
        for (size_t p = 0; p < no; ++p) out_depth[p] = encode_depth(depth[p], vt, false);
    if (out_masked_depth)
        for (size_t p = 0; p < no; ++p) out_masked_depth[p] = encode_depth(depth[p], vt, mask[p] != 0);
    return RVSB_OK;
}

int orc_synthesize(int n, const rvsb_camera* cams, const rvsb_view_planes* planes,
                   const rvsb_camera* vt, float exponent, uint16_t* out_yuv, float* out_quality,
                   float* out_color) {
    return orc_synthesize_aux(n, cams, planes, vt, exponent, out_yuv, out_quality, out_color, 0.f, nullptr,
                              nullptr, nullptr, nullptr);
}

}  // extern "C"
