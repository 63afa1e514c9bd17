// Host camera math.  Trigonometric functions are evaluated in double and
// rounded to float, which gives the correctly rounded float result of the
// reference's float cos/sin calls.
#include "camera.hpp"

#include <cmath>

namespace rvsb {
namespace {

struct M33 {
    float m[9];
};

// cv::Matx product: s = 0; s += a(i,k) * b(k,j), in float.
M33 mul(const M33& a, const M33& b) {
    M33 c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float s = 0.f;
            for (int k = 0; k < 3; ++k) s += a.m[i * 3 + k] * b.m[k * 3 + j];
            c.m[i * 3 + j] = s;
        }
    return c;
}

inline float fcos(float x) { return (float)std::cos((double)x); }
inline float fsin(float x) { return (float)std::sin((double)x); }

}  // namespace

void rotation_matrix(const float rot[3], float R[9]) {
    const float radperdeg = 0.01745329252f;
    const float a = radperdeg * rot[0], b = radperdeg * rot[1], c = radperdeg * rot[2];
    const M33 rz{{fcos(a), -fsin(a), 0.f, fsin(a), fcos(a), 0.f, 0.f, 0.f, 1.f}};
    const M33 ry{{fcos(b), 0.f, fsin(b), 0.f, 1.f, 0.f, -fsin(b), 0.f, fcos(b)}};
    const M33 rx{{1.f, 0.f, 0.f, 0.f, fcos(c), -fsin(c), 0.f, fsin(c), fcos(c)}};
    const M33 r = mul(mul(rz, ry), rx);
    for (int k = 0; k < 9; ++k) R[k] = r.m[k];
}

void relative_pose(const rvsb_camera& in, const rvsb_camera& virt, float R[9], float t[3]) {
    M33 rf, rt, rtt;
    rotation_matrix(in.rotation, rf.m);
    rotation_matrix(virt.rotation, rt.m);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) rtt.m[i * 3 + j] = rt.m[j * 3 + i];
    const M33 r = mul(rtt, rf);
    for (int k = 0; k < 9; ++k) R[k] = r.m[k];
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = virt.position[k] - in.position[k];
    for (int i = 0; i < 3; ++i) {
        float s = 0.f;
        for (int k = 0; k < 3; ++k) s += (-rtt.m[i * 3 + k]) * d[k];
        t[i] = s;
    }
}

void erp_tables(const rvsb_camera& in, std::vector<float>& rows, std::vector<float>& cols) {
    const int w = in.width, h = in.height;
    const float radperdeg = 0.01745329252f;
    const float phi0 = radperdeg * in.hor_range[1];
    const float theta0 = radperdeg * in.ver_range[1];
    const float dphi_du = -radperdeg * (in.hor_range[1] - in.hor_range[0]) / w;
    const float dtheta_dv = -radperdeg * (in.ver_range[1] - in.ver_range[0]) / h;
    rows.resize(2 * (size_t)h);
    cols.resize(2 * (size_t)w);
    for (int i = 0; i < h; ++i) {
        float v = i + 0.5f;
        if (i == 0) v = 1e-3f;
        if (i == h - 1) v = h - 1e-3f;
        const float theta = theta0 + dtheta_dv * v;
        rows[2 * i] = fcos(theta);
        rows[2 * i + 1] = fsin(theta);
    }
    for (int j = 0; j < w; ++j) {
        const float u = j + 0.5f;
        const float phi = phi0 + dphi_du * u;
        cols[2 * j] = fcos(phi);
        cols[2 * j + 1] = fsin(phi);
    }
}

void erp_projector_constants(const rvsb_camera& v, float& u0, float& v0, float& du_dphi, float& dv_dtheta) {
    const float degperrad = 57.295779513f;
    const int w = v.width, h = v.height;
    u0 = w * v.hor_range[1] / (v.hor_range[1] - v.hor_range[0]);
    v0 = h * v.ver_range[1] / (v.ver_range[1] - v.ver_range[0]);
    du_dphi = -degperrad * w / (v.hor_range[1] - v.hor_range[0]);
    dv_dtheta = -degperrad * h / (v.ver_range[1] - v.ver_range[0]);
}

const char* camera_problem(const rvsb_camera& c, bool as_output) {
    if (c.projection != RVSB_PROJ_PERSPECTIVE && c.projection != RVSB_PROJ_EQUIRECTANGULAR)
        return "unknown projection type";
    if (c.width < 2 || c.height < 2 || c.width > 16384 || c.height > 16384) return "resolution out of range";
    if ((c.width & 1) || (c.height & 1)) return "YUV420 planes need an even resolution";
    if (c.bit_depth_color < 9 || c.bit_depth_color > 16)
        return "colour bit depth must be 9..16 (16-bit samples)";
    if (!as_output) {
        if (c.bit_depth_depth < 9 || c.bit_depth_depth > 16)
            return "depth bit depth must be 9..16 (16-bit samples)";
        if (!(c.depth_range[0] < c.depth_range[1])) return "inverted depth range";
        int bits = 0;
        while ((1 << bits) < c.width - 1) ++bits;
        if (((int64_t)(c.height - 1) << (bits + 2)) > ((int64_t)1 << 32)) return "input too large";
    }
    if (c.projection == RVSB_PROJ_PERSPECTIVE && (c.focal[0] == 0.f || c.focal[1] == 0.f)) return "zero focal length";
    if (c.projection == RVSB_PROJ_EQUIRECTANGULAR &&
        (c.hor_range[1] == c.hor_range[0] || c.ver_range[1] == c.ver_range[0]))
        return "empty equirectangular range";
    return nullptr;
}

}  // namespace rvsb
