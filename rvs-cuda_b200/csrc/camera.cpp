// Host camera math.  Trigonometric functions are evaluated in double and
// rounded to float, which gives the correctly rounded float result of the
// reference's float cos/sin calls.
#include "camera.hpp"

#include <algorithm>
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

void erp_tile_cones(const rvsb_camera& in, const std::vector<float>& rows, const std::vector<float>& cols,
                    int tile, std::vector<float>& out) {
    const int w = in.width, h = in.height;
    const int ntx = (w + tile - 1) / tile, nty = (h + tile - 1) / tile;
    out.assign((size_t)ntx * nty * 4, 0.f);
    auto dir = [&](int i, int j, double d[3]) {
        d[0] = (double)rows[2 * i] * cols[2 * j];
        d[1] = (double)rows[2 * i] * cols[2 * j + 1];
        d[2] = rows[2 * i + 1];
        const double n = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int k = 0; k < 3; ++k) d[k] /= n;
    };
    auto angle = [](const double a[3], const double b[3]) {
        // atan2(|a x b|, a . b): accurate for small angles
        const double cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2], cz = a[0] * b[1] - a[1] * b[0];
        return std::atan2(std::sqrt(cx * cx + cy * cy + cz * cz), a[0] * b[0] + a[1] * b[1] + a[2] * b[2]);
    };
    for (int ty = 0; ty < nty; ++ty)
        for (int tx = 0; tx < ntx; ++tx) {
            const int r0 = std::max(0, ty * tile - 1), r1 = std::min(h - 1, ty * tile + tile);
            const int c0 = std::max(0, tx * tile - 1), c1 = std::min(w - 1, tx * tile + tile);
            double dc[3], d[3], prev[3];
            dir((r0 + r1) / 2, (c0 + c1) / 2, dc);
            double rho = 0.0, step = 0.0;
            // The angle to a fixed direction peaks on the region's boundary;
            // between two boundary samples it can exceed both by at most
            // their separation, so the largest separation is added.
            auto visit = [&](int i, int j, bool first) {
                dir(i, j, d);
                rho = std::max(rho, angle(dc, d));
                if (!first) step = std::max(step, angle(prev, d));
                prev[0] = d[0]; prev[1] = d[1]; prev[2] = d[2];
            };
            for (int j = c0; j <= c1; ++j) visit(r0, j, j == c0);
            for (int i = r0; i <= r1; ++i) visit(i, c1, i == r0);
            for (int j = c1; j >= c0; --j) visit(r1, j, j == c1);
            for (int i = r1; i >= r0; --i) visit(i, c0, i == r1);
            float* o = &out[((size_t)ty * ntx + tx) * 4];
            o[0] = (float)dc[0];
            o[1] = (float)dc[1];
            o[2] = (float)dc[2];
            o[3] = (float)(rho + step + 1e-4);
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
