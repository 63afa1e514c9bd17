// Seeded synthetic scene renderer (input planes for the benchmark and test
// workloads).  Not part of the synthesis path: it writes the raw YUV420 and
// depth planes a camera would store for an analytic scene of rectangles,
// spheres and boxes, textured with 3-D value noise and flat patches.
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t h) {
    h ^= h >> 33;
    h *= 0xFF51AFD7ED558CCDull;
    h ^= h >> 33;
    h *= 0xC4CEB9FE1A85EC53ull;
    h ^= h >> 33;
    return h;
}

inline float lattice(int64_t ix, int64_t iy, int64_t iz, uint64_t seed) {
    uint64_t h = ((uint64_t)ix * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)iy * 0xC2B2AE3D27D4EB4Full) ^
                 ((uint64_t)iz * 0x165667B19E3779F9ull) ^ seed;
    h = mix64(h);
    return (float)(h >> 40) * (1.0f / (1 << 24));
}

float value_noise(const double p[3], uint64_t seed, int octaves, double base_freq) {
    double total = 0, amp = 1, norm = 0, freq = base_freq;
    for (int o = 0; o < octaves; ++o) {
        double q[3], t[3];
        int64_t i0[3];
        for (int k = 0; k < 3; ++k) {
            q[k] = p[k] * freq;
            double f = std::floor(q[k]);
            i0[k] = (int64_t)f;
            double tt = q[k] - f;
            t[k] = tt * tt * (3 - 2 * tt);
        }
        double acc = 0;
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    double w = (dx ? t[0] : 1 - t[0]) * (dy ? t[1] : 1 - t[1]) * (dz ? t[2] : 1 - t[2]);
                    acc += w * lattice(i0[0] + dx, i0[1] + dy, i0[2] + dz, seed + 7919ull * o);
                }
        total += amp * acc;
        norm += amp;
        amp *= 0.5;
        freq *= 2;
    }
    return (float)(total / norm);
}

struct Cam {
    int proj, w, h, bits_color, bits_depth;
    double pos[3], R[9], focal[2], pp[2], hor[2], ver[2], near_, far_;
};

}  // namespace

extern "C" {

/* cam: proj, w, h, bits_color, bits_depth (int[5]);
 * camd: pos[3], R[9] (camera to world), focal[2], pp[2], hor[2], ver[2], near, far (double[22]);
 * rects: n_rect x 12 (center, half-axis u, half-axis v, normal); spheres: n_sph x 4;
 * boxes: n_box x 7 (lo, hi, inward); patches: n_patch x 7 (center, radius, Y, U, V).
 * Outputs: Y (h*w), U, V ((h/2)*(w/2)), D (h*w) uint16. */
int sg_render(const int* cam_i, const double* camd, const double* rects, int n_rect, const double* spheres,
              int n_sph, const double* boxes, int n_box, const double* patches, int n_patch, uint64_t seed,
              uint16_t* Y, uint16_t* U, uint16_t* V, uint16_t* D) {
    Cam c;
    c.proj = cam_i[0];
    c.w = cam_i[1];
    c.h = cam_i[2];
    c.bits_color = cam_i[3];
    c.bits_depth = cam_i[4];
    for (int k = 0; k < 3; ++k) c.pos[k] = camd[k];
    for (int k = 0; k < 9; ++k) c.R[k] = camd[3 + k];
    c.focal[0] = camd[12]; c.focal[1] = camd[13];
    c.pp[0] = camd[14]; c.pp[1] = camd[15];
    c.hor[0] = camd[16]; c.hor[1] = camd[17];
    c.ver[0] = camd[18]; c.ver[1] = camd[19];
    c.near_ = camd[20];
    c.far_ = camd[21];
    const int w = c.w, h = c.h;
    if (w <= 0 || h <= 0 || (w & 1) || (h & 1)) return 1;
    const double maxc = (double)((1u << c.bits_color) - 1u);
    const double maxd = (double)((1u << c.bits_depth) - 1u);
    std::vector<float> chroma((size_t)w * h * 2);
    const double rpd = M_PI / 180.0;
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < h; ++i) {
        for (int j = 0; j < w; ++j) {
            double local[3];
            const double u = j + 0.5;
            double v = i + 0.5;
            if (c.proj == 0) {
                local[0] = 1.0;
                local[1] = -(u - c.pp[0]) / c.focal[0];
                local[2] = -(v - c.pp[1]) / c.focal[1];
            } else {
                if (i == 0) v = 1e-3;
                if (i == h - 1) v = h - 1e-3;
                const double phi = rpd * c.hor[1] - rpd * (c.hor[1] - c.hor[0]) / w * u;
                const double theta = rpd * c.ver[1] - rpd * (c.ver[1] - c.ver[0]) / h * v;
                local[0] = std::cos(theta) * std::cos(phi);
                local[1] = std::cos(theta) * std::sin(phi);
                local[2] = std::sin(theta);
            }
            double d[3];
            for (int r = 0; r < 3; ++r) d[r] = c.R[r * 3] * local[0] + c.R[r * 3 + 1] * local[1] + c.R[r * 3 + 2] * local[2];
            double best = INFINITY;
            for (int k = 0; k < n_rect; ++k) {
                const double* q = rects + k * 12;
                const double* n = q + 9;
                const double den = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
                if (den == 0) continue;
                const double s = ((q[0] - c.pos[0]) * n[0] + (q[1] - c.pos[1]) * n[1] + (q[2] - c.pos[2]) * n[2]) / den;
                if (!(s > 1e-6) || s >= best) continue;
                double hit[3];
                for (int r = 0; r < 3; ++r) hit[r] = c.pos[r] + s * d[r] - q[r];
                const double* au = q + 3;
                const double* av = q + 6;
                const double lu = (hit[0] * au[0] + hit[1] * au[1] + hit[2] * au[2]) /
                                  (au[0] * au[0] + au[1] * au[1] + au[2] * au[2]);
                const double lv = (hit[0] * av[0] + hit[1] * av[1] + hit[2] * av[2]) /
                                  (av[0] * av[0] + av[1] * av[1] + av[2] * av[2]);
                if (std::fabs(lu) <= 1 && std::fabs(lv) <= 1) best = s;
            }
            for (int k = 0; k < n_sph; ++k) {
                const double* q = spheres + k * 4;
                double oc[3] = {c.pos[0] - q[0], c.pos[1] - q[1], c.pos[2] - q[2]};
                const double b = d[0] * oc[0] + d[1] * oc[1] + d[2] * oc[2];
                const double a = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                const double cc = oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2] - q[3] * q[3];
                const double disc = b * b - a * cc;
                if (disc < 0) continue;
                const double sq = std::sqrt(disc);
                double s = (-b - sq) / a;
                if (!(s > 1e-6)) s = (-b + sq) / a;
                if (s > 1e-6 && s < best) best = s;
            }
            for (int k = 0; k < n_box; ++k) {
                const double* q = boxes + k * 7;
                double tmin = -INFINITY, tmax = INFINITY;
                for (int r = 0; r < 3; ++r) {
                    if (d[r] == 0) {
                        if (c.pos[r] < q[r] || c.pos[r] > q[3 + r]) { tmin = INFINITY; tmax = -INFINITY; }
                        continue;
                    }
                    double t1 = (q[r] - c.pos[r]) / d[r], t2 = (q[3 + r] - c.pos[r]) / d[r];
                    if (t1 > t2) std::swap(t1, t2);
                    tmin = std::max(tmin, t1);
                    tmax = std::min(tmax, t2);
                }
                if (tmax < tmin) continue;
                const double s = q[6] != 0 ? tmax : tmin;
                if (s > 1e-6 && s < best) best = s;
            }
            const bool miss = !std::isfinite(best);
            const double z = miss ? c.far_ : std::min(best, c.far_);
            const double st = miss ? c.far_ : best;
            const double pt[3] = {c.pos[0] + d[0] * st, c.pos[1] + d[1] * st, c.pos[2] + d[2] * st};
            double yy = 0.12 + 0.76 * value_noise(pt, seed ^ 0x1111, 4, 2.0);
            double p7[3] = {pt[0] * 0.7, pt[1] * 0.7, pt[2] * 0.7};
            double uu = 0.5 + 0.36 * (value_noise(p7, seed ^ 0x2222, 3, 2.0) - 0.5);
            double p8[3] = {p7[0] + 3.1, p7[1] + 3.1, p7[2] + 3.1};
            double vv = 0.5 + 0.36 * (value_noise(p8, seed ^ 0x3333, 3, 2.0) - 0.5);
            for (int k = 0; k < n_patch; ++k) {
                const double* q = patches + k * 7;
                const double dd = (pt[0] - q[0]) * (pt[0] - q[0]) + (pt[1] - q[1]) * (pt[1] - q[1]) +
                                  (pt[2] - q[2]) * (pt[2] - q[2]);
                if (dd <= q[3] * q[3]) {
                    yy = q[4];
                    uu = q[5];
                    vv = q[6];
                }
            }
            const size_t o = (size_t)i * w + j;
            Y[o] = (uint16_t)std::lround(std::min(1.0, std::max(0.0, yy)) * maxc);
            chroma[o * 2] = (float)std::min(1.0, std::max(0.0, uu));
            chroma[o * 2 + 1] = (float)std::min(1.0, std::max(0.0, vv));
            double dn = c.far_ >= 1000.0 ? c.near_ / z : (c.far_ * c.near_ / z - c.near_) / (c.far_ - c.near_);
            dn = std::min(1.0, std::max(0.0, dn));
            D[o] = (uint16_t)std::lround(dn * maxd);
        }
    }
    const int cw = w / 2, ch = h / 2;
#pragma omp parallel for
    for (int i = 0; i < ch; ++i)
        for (int j = 0; j < cw; ++j) {
            double su = 0, sv = 0;
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const size_t o = ((size_t)(2 * i + dy) * w + 2 * j + dx) * 2;
                    su += chroma[o];
                    sv += chroma[o + 1];
                }
            U[(size_t)i * cw + j] = (uint16_t)std::lround(su * 0.25 * maxc);
            V[(size_t)i * cw + j] = (uint16_t)std::lround(sv * 0.25 * maxc);
        }
    return 0;
}

}  // extern "C"
