// TEST INFRASTRUCTURE ONLY.
//
// A minimal stand-in for the part of the OpenCV 4 core API that the
// reference's CPU synthesis sources use (rvs/src/transform.cpp,
// blending.cpp, inpainting.cpp, BlendedView.cpp, View.cpp,
// image_writing.cpp, Parameters.cpp, the (Un)Projector files, ...), so that
// those files compile unmodified into oracle/_ref/ and the oracle can be
// checked against the reference's own code.  It is written from OpenCV's
// documented behaviour; no OpenCV source is used.  Only what those files
// call exists, and operations they only reference on paths this harness
// never runs (morphology, colour conversion, OpenCV's own inpainting,
// bilateral filtering, image files) throw when called.
//
// Arithmetic that decides output bits follows OpenCV 4.9 as the oracle
// (oracle/rvs_oracle.cpp) restates it:
//   - Matx * Matx / Matx * Vec: s = 0; s += a(i,k) * b(k,j) in the element
//     type;
//   - Vec * scalar: element * scalar in the wider of the two types, then
//     converted (float * float stays float); Vec / scalar multiplies by
//     the reciprocal (1.f / alpha for float, 1. / alpha for double);
//   - cv::norm(Vec a, Vec b): differences in the element type, squares
//     summed in double, square root in double; cv::norm(Vec): the same
//     without the difference;
//   - element-wise Mat arithmetic and comparisons in the element type,
//     comparisons against a scalar after converting it to that type;
//   - resize by exactly 0.5 x 0.5 of 16-bit samples with INTER_LINEAR: the
//     2x2 mean rounded half to even (OpenCV with Intel IPP, its default on
//     x86-64) or half up (cvshim_set_resize_ties_up(1)).
#pragma once

#include <algorithm>
#include <array>
#include <cassert>
#include <iostream>
#include <sstream>
#include <functional>
#include <map>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <limits>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

typedef unsigned char uchar;
typedef signed char schar;
typedef unsigned short ushort;

#ifndef MAX
#define MAX(a, b) ((a) < (b) ? (b) : (a))
#endif
#ifndef MIN
#define MIN(a, b) ((a) > (b) ? (b) : (a))
#endif

#define CV_8U 0
#define CV_8S 1
#define CV_16U 2
#define CV_16S 3
#define CV_32S 4
#define CV_32F 5
#define CV_64F 6
#define CV_CN_SHIFT 3
#define CV_MAT_DEPTH(t) ((t) & 7)
#define CV_MAT_CN(t) ((((t) >> CV_CN_SHIFT) & 511) + 1)
#define CV_MAKETYPE(depth, cn) (CV_MAT_DEPTH(depth) + (((cn) - 1) << CV_CN_SHIFT))
#define CV_MAKE_TYPE CV_MAKETYPE
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_8UC4 CV_MAKETYPE(CV_8U, 4)
#define CV_16UC1 CV_MAKETYPE(CV_16U, 1)
#define CV_16UC3 CV_MAKETYPE(CV_16U, 3)
#define CV_32SC1 CV_MAKETYPE(CV_32S, 1)
#define CV_32SC3 CV_MAKETYPE(CV_32S, 3)
#define CV_32SC4 CV_MAKETYPE(CV_32S, 4)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC2 CV_MAKETYPE(CV_32F, 2)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)
#define CV_32FC4 CV_MAKETYPE(CV_32F, 4)
#define CV_64FC1 CV_MAKETYPE(CV_64F, 1)

namespace cv {

class Exception : public std::runtime_error {
public:
    explicit Exception(const std::string& what) : std::runtime_error(what) {}
};

[[noreturn]] inline void shim_fail(const std::string& what) { throw Exception("cv stand-in: " + what); }

}  // namespace cv

#define CV_Assert(expr)                                                                     \
    do {                                                                                    \
        if (!(expr)) ::cv::shim_fail(std::string("assertion failed: ") + #expr + " at " + \
                                     __FILE__ + ":" + std::to_string(__LINE__));            \
    } while (0)
#define CV_DbgAssert(expr) ((void)0)
#define CV_Error(code, msg) ::cv::shim_fail(msg)

namespace cv {

// ---------------------------------------------------------------------------
// saturate_cast: integers saturate, floating point to integer rounds to
// nearest (ties to even, the SSE conversion OpenCV's cvRound uses).
template <typename T>
struct SatHelper {
    template <typename S>
    static T cast(S v) {
        if constexpr (std::is_floating_point<T>::value) {
            return static_cast<T>(v);
        } else if constexpr (std::is_same<T, bool>::value) {
            return v != 0;
        } else {
            double d;
            if constexpr (std::is_floating_point<S>::value) {
                d = std::nearbyint((double)v);
            } else {
                d = (double)v;
            }
            const double lo = (double)std::numeric_limits<T>::min();
            const double hi = (double)std::numeric_limits<T>::max();
            if (!(d >= lo)) return std::numeric_limits<T>::min();
            if (d > hi) return std::numeric_limits<T>::max();
            return static_cast<T>(d);
        }
    }
};
template <typename T, typename S>
inline T saturate_cast(S v) {
    return SatHelper<T>::cast(v);
}

inline int cvRound(double v) { return (int)std::nearbyint(v); }
inline int cvFloor(double v) { return (int)std::floor(v); }
inline int cvCeil(double v) { return (int)std::ceil(v); }

// ---------------------------------------------------------------------------
template <typename T, int m, int n>
class Matx;
template <typename T, int cn>
class Vec;

template <typename T>
struct DepthOf;
template <> struct DepthOf<bool> { enum { value = CV_8U }; };
template <> struct DepthOf<uchar> { enum { value = CV_8U }; };
template <> struct DepthOf<schar> { enum { value = CV_8S }; };
template <> struct DepthOf<ushort> { enum { value = CV_16U }; };
template <> struct DepthOf<short> { enum { value = CV_16S }; };
template <> struct DepthOf<int> { enum { value = CV_32S }; };
template <> struct DepthOf<float> { enum { value = CV_32F }; };
template <> struct DepthOf<double> { enum { value = CV_64F }; };

template <typename T>
struct DataType {
    typedef T value_type;
    typedef T channel_type;
    typedef typename std::conditional<std::is_floating_point<T>::value, T, int>::type work_type;
    enum { depth = DepthOf<T>::value, channels = 1, type = CV_MAKETYPE(depth, 1) };
};
template <typename T, int cn>
struct DataType<Vec<T, cn>> {
    typedef Vec<T, cn> value_type;
    typedef T channel_type;
    enum { depth = DepthOf<T>::value, channels = cn, type = CV_MAKETYPE(depth, cn) };
};

// The type in which element (x) scalar products are formed: C++'s usual
// arithmetic conversions of the two (float * float stays float).
template <typename T, typename S>
struct ScaleType {
    typedef decltype(T() * S()) type;
};

// ---------------------------------------------------------------------------
template <typename T, int m, int n>
class Matx {
public:
    enum { rows = m, cols = n, channels = m * n };
    typedef T value_type;
    T val[m * n];

    Matx() {
        for (int i = 0; i < m * n; ++i) val[i] = T(0);
    }
    explicit Matx(const T* vals) {
        for (int i = 0; i < m * n; ++i) val[i] = vals[i];
    }
    Matx(std::initializer_list<T> l) {
        int i = 0;
        for (T v : l) {
            if (i < m * n) val[i++] = v;
        }
        for (; i < m * n; ++i) val[i] = T(0);
    }
    Matx(T v0, T v1, T v2, T v3) : Matx({v0, v1, v2, v3}) {}
    Matx(T v0, T v1, T v2, T v3, T v4, T v5, T v6, T v7, T v8) : Matx({v0, v1, v2, v3, v4, v5, v6, v7, v8}) {}

    static Matx all(T a) {
        Matx r;
        for (int i = 0; i < m * n; ++i) r.val[i] = a;
        return r;
    }
    static Matx zeros() { return all(T(0)); }
    static Matx ones() { return all(T(1)); }
    static Matx eye() {
        Matx r;
        for (int i = 0; i < std::min(m, n); ++i) r.val[i * n + i] = T(1);
        return r;
    }

    T& operator()(int i, int j) { return val[i * n + j]; }
    const T& operator()(int i, int j) const { return val[i * n + j]; }
    T& operator()(int i) { return val[i]; }
    const T& operator()(int i) const { return val[i]; }

    Matx<T, n, m> t() const {
        Matx<T, n, m> r;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < n; ++j) r(j, i) = (*this)(i, j);
        return r;
    }

    template <int l>
    Matx<T, m, l> mul_mat(const Matx<T, n, l>& b) const {
        Matx<T, m, l> c;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < l; ++j) {
                T s = 0;
                for (int k = 0; k < n; ++k) s += (*this)(i, k) * b(k, j);
                c(i, j) = s;
            }
        return c;
    }
};

template <typename T, int m, int n, int l>
inline Matx<T, m, l> operator*(const Matx<T, m, n>& a, const Matx<T, n, l>& b) {
    return a.mul_mat(b);
}
template <typename T, int m, int n>
inline Matx<T, m, n> operator+(const Matx<T, m, n>& a, const Matx<T, m, n>& b) {
    Matx<T, m, n> r;
    for (int i = 0; i < m * n; ++i) r.val[i] = saturate_cast<T>(a.val[i] + b.val[i]);
    return r;
}
template <typename T, int m, int n>
inline Matx<T, m, n> operator-(const Matx<T, m, n>& a, const Matx<T, m, n>& b) {
    Matx<T, m, n> r;
    for (int i = 0; i < m * n; ++i) r.val[i] = saturate_cast<T>(a.val[i] - b.val[i]);
    return r;
}
template <typename T, int m, int n>
inline Matx<T, m, n> operator-(const Matx<T, m, n>& a) {
    Matx<T, m, n> r;
    for (int i = 0; i < m * n; ++i) r.val[i] = saturate_cast<T>(-a.val[i]);
    return r;
}
template <typename T, int m, int n>
inline bool operator==(const Matx<T, m, n>& a, const Matx<T, m, n>& b) {
    for (int i = 0; i < m * n; ++i)
        if (!(a.val[i] == b.val[i])) return false;
    return true;
}
template <typename T, int m, int n>
inline bool operator!=(const Matx<T, m, n>& a, const Matx<T, m, n>& b) {
    return !(a == b);
}

typedef Matx<float, 2, 2> Matx22f;
typedef Matx<float, 3, 3> Matx33f;
typedef Matx<float, 4, 4> Matx44f;
typedef Matx<double, 3, 3> Matx33d;

// ---------------------------------------------------------------------------
template <typename T, int cn>
class Vec : public Matx<T, cn, 1> {
public:
    typedef T value_type;
    enum { channels = cn };

    Vec() {}
    Vec(T v0) {
        this->val[0] = v0;
    }
    Vec(T v0, T v1) {
        static_assert(cn >= 2, "too many values");
        this->val[0] = v0;
        this->val[1] = v1;
    }
    Vec(T v0, T v1, T v2) {
        static_assert(cn >= 3, "too many values");
        this->val[0] = v0;
        this->val[1] = v1;
        this->val[2] = v2;
    }
    Vec(T v0, T v1, T v2, T v3) {
        static_assert(cn >= 4, "too many values");
        this->val[0] = v0;
        this->val[1] = v1;
        this->val[2] = v2;
        this->val[3] = v3;
    }
    explicit Vec(const T* values) : Matx<T, cn, 1>(values) {}
    Vec(const Matx<T, cn, 1>& a) : Matx<T, cn, 1>(a) {}

    static Vec all(T a) {
        Vec r;
        for (int i = 0; i < cn; ++i) r.val[i] = a;
        return r;
    }

    T& operator[](int i) { return this->val[i]; }
    const T& operator[](int i) const { return this->val[i]; }
    T& operator()(int i) { return this->val[i]; }
    const T& operator()(int i) const { return this->val[i]; }

    template <typename T2>
    operator Vec<T2, cn>() const {
        Vec<T2, cn> r;
        for (int i = 0; i < cn; ++i) r.val[i] = saturate_cast<T2>(this->val[i]);
        return r;
    }
};

template <typename T, int cn>
inline Vec<T, cn> operator+(const Vec<T, cn>& a, const Vec<T, cn>& b) {
    Vec<T, cn> r;
    for (int i = 0; i < cn; ++i) r.val[i] = saturate_cast<T>(a.val[i] + b.val[i]);
    return r;
}
template <typename T, int cn>
inline Vec<T, cn> operator-(const Vec<T, cn>& a, const Vec<T, cn>& b) {
    Vec<T, cn> r;
    for (int i = 0; i < cn; ++i) r.val[i] = saturate_cast<T>(a.val[i] - b.val[i]);
    return r;
}
template <typename T, int cn>
inline Vec<T, cn> operator-(const Vec<T, cn>& a) {
    Vec<T, cn> r;
    for (int i = 0; i < cn; ++i) r.val[i] = saturate_cast<T>(-a.val[i]);
    return r;
}
template <typename T, int cn>
inline Vec<T, cn>& operator+=(Vec<T, cn>& a, const Vec<T, cn>& b) {
    for (int i = 0; i < cn; ++i) a.val[i] = saturate_cast<T>(a.val[i] + b.val[i]);
    return a;
}
template <typename T, int cn>
inline Vec<T, cn>& operator-=(Vec<T, cn>& a, const Vec<T, cn>& b) {
    for (int i = 0; i < cn; ++i) a.val[i] = saturate_cast<T>(a.val[i] - b.val[i]);
    return a;
}

template <typename T, int cn, typename S>
inline Vec<T, cn> vec_scale(const Vec<T, cn>& a, S alpha) {
    typedef typename ScaleType<T, S>::type W;
    Vec<T, cn> r;
    for (int i = 0; i < cn; ++i) r.val[i] = saturate_cast<T>((W)a.val[i] * (W)alpha);
    return r;
}
template <typename T, int cn>
inline Vec<T, cn> operator*(const Vec<T, cn>& a, int alpha) { return vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator*(const Vec<T, cn>& a, float alpha) { return vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator*(const Vec<T, cn>& a, double alpha) { return vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator*(int alpha, const Vec<T, cn>& a) { return vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator*(float alpha, const Vec<T, cn>& a) { return vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator*(double alpha, const Vec<T, cn>& a) { return vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator/(const Vec<T, cn>& a, float alpha) { return vec_scale(a, 1.f / alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator/(const Vec<T, cn>& a, double alpha) { return vec_scale(a, 1. / alpha); }
template <typename T, int cn>
inline Vec<T, cn> operator/(const Vec<T, cn>& a, int alpha) { return vec_scale(a, 1. / alpha); }
template <typename T, int cn>
inline Vec<T, cn>& operator*=(Vec<T, cn>& a, float alpha) { return a = vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn>& operator*=(Vec<T, cn>& a, double alpha) { return a = vec_scale(a, alpha); }
template <typename T, int cn>
inline Vec<T, cn>& operator/=(Vec<T, cn>& a, float alpha) { return a = vec_scale(a, 1.f / alpha); }
template <typename T, int cn>
inline Vec<T, cn>& operator/=(Vec<T, cn>& a, double alpha) { return a = vec_scale(a, 1. / alpha); }

template <typename T, int m, int n>
inline Vec<T, m> operator*(const Matx<T, m, n>& a, const Vec<T, n>& b) {
    Matx<T, m, 1> c = a.mul_mat(static_cast<const Matx<T, n, 1>&>(b));
    return Vec<T, m>(c);
}

template <typename T, int cn>
inline std::ostream& operator<<(std::ostream& o, const Vec<T, cn>& v) {
    o << '[';
    for (int i = 0; i < cn; ++i) o << (i ? ", " : "") << v.val[i];
    return o << ']';
}

typedef Vec<uchar, 2> Vec2b;
typedef Vec<uchar, 3> Vec3b;
typedef Vec<uchar, 4> Vec4b;
typedef Vec<short, 2> Vec2s;
typedef Vec<short, 3> Vec3s;
typedef Vec<ushort, 2> Vec2w;
typedef Vec<ushort, 3> Vec3w;
typedef Vec<int, 2> Vec2i;
typedef Vec<int, 3> Vec3i;
typedef Vec<int, 4> Vec4i;
typedef Vec<float, 2> Vec2f;
typedef Vec<float, 3> Vec3f;
typedef Vec<float, 4> Vec4f;
typedef Vec<double, 2> Vec2d;
typedef Vec<double, 3> Vec3d;
typedef Vec<double, 4> Vec4d;

// Scalar: four doubles.
class Scalar : public Vec<double, 4> {
public:
    Scalar() {}
    Scalar(double v0) { val[0] = v0; }
    Scalar(double v0, double v1, double v2 = 0, double v3 = 0) {
        val[0] = v0;
        val[1] = v1;
        val[2] = v2;
        val[3] = v3;
    }
    template <typename T, int cn>
    Scalar(const Vec<T, cn>& v) {
        static_assert(cn <= 4, "Scalar holds at most 4 values");
        for (int i = 0; i < cn; ++i) val[i] = (double)v.val[i];
    }
    static Scalar all(double v) { return Scalar(v, v, v, v); }
};

template <typename T, int cn>
inline Scalar sum(const Vec<T, cn>& v) {
    double s = 0;
    for (int i = 0; i < cn; ++i) s += (double)v.val[i];
    return Scalar(s);
}

enum NormTypes { NORM_INF = 1, NORM_L1 = 2, NORM_L2 = 4 };

template <typename T, int cn>
inline double norm(const Vec<T, cn>& a, const Vec<T, cn>& b, int normType = NORM_L2) {
    if (normType != NORM_L2) shim_fail("norm: only NORM_L2");
    double s = 0;
    for (int i = 0; i < cn; ++i) {
        const double v = (double)(T)(a.val[i] - b.val[i]);
        s += v * v;
    }
    return std::sqrt(s);
}
template <typename T, int m, int n>
inline double norm(const Matx<T, m, n>& a) {
    double s = 0;
    for (int i = 0; i < m * n; ++i) {
        const double v = (double)a.val[i];
        s += v * v;
    }
    return std::sqrt(s);
}

// ---------------------------------------------------------------------------
template <typename T>
class Point_ {
public:
    T x, y;
    Point_() : x(0), y(0) {}
    Point_(T x_, T y_) : x(x_), y(y_) {}
    Point_(const Vec<T, 2>& v) : x(v[0]), y(v[1]) {}
    template <typename U>
    explicit Point_(const Point_<U>& p) : x(saturate_cast<T>(p.x)), y(saturate_cast<T>(p.y)) {}
    operator Vec<T, 2>() const { return Vec<T, 2>(x, y); }
    bool operator==(const Point_& o) const { return x == o.x && y == o.y; }
    bool operator!=(const Point_& o) const { return !(*this == o); }
};
typedef Point_<int> Point2i;
typedef Point_<int> Point;
typedef Point_<float> Point2f;
typedef Point_<double> Point2d;

template <typename T>
class Size_ {
public:
    T width, height;
    Size_() : width(0), height(0) {}
    Size_(T w, T h) : width(w), height(h) {}
    explicit Size_(const Vec<T, 2>& v) : width(v[0]), height(v[1]) {}
    explicit Size_(const Point_<T>& p) : width(p.x), height(p.y) {}
    T area() const { return width * height; }
    bool empty() const { return width <= 0 || height <= 0; }
    bool operator==(const Size_& o) const { return width == o.width && height == o.height; }
    bool operator!=(const Size_& o) const { return !(*this == o); }
};
typedef Size_<int> Size2i;
typedef Size_<int> Size;
typedef Size_<float> Size2f;

template <typename T>
inline Size_<T> operator/(const Size_<T>& a, T b) {
    return Size_<T>(a.width / b, a.height / b);
}
template <typename T>
inline Size_<T> operator*(const Size_<T>& a, T b) {
    return Size_<T>(a.width * b, a.height * b);
}
inline std::ostream& operator<<(std::ostream& o, const Size& s) { return o << '[' << s.width << " x " << s.height << ']'; }
template <typename T>
inline std::ostream& operator<<(std::ostream& o, const Point_<T>& p) {
    return o << '[' << p.x << ", " << p.y << ']';
}

template <typename T>
class Rect_ {
public:
    T x, y, width, height;
    Rect_() : x(0), y(0), width(0), height(0) {}
    Rect_(T x_, T y_, T w, T h) : x(x_), y(y_), width(w), height(h) {}
    Rect_(const Point_<T>& org, const Size_<T>& sz) : x(org.x), y(org.y), width(sz.width), height(sz.height) {}
    Point_<T> tl() const { return Point_<T>(x, y); }
    Point_<T> br() const { return Point_<T>(x + width, y + height); }
    Size_<T> size() const { return Size_<T>(width, height); }
    T area() const { return width * height; }
    bool empty() const { return width <= 0 || height <= 0; }
    bool operator==(const Rect_& o) const {
        return x == o.x && y == o.y && width == o.width && height == o.height;
    }
    bool operator!=(const Rect_& o) const { return !(*this == o); }
};
template <typename T>
inline std::ostream& operator<<(std::ostream& o, const Rect_<T>& r) {
    return o << '[' << r.width << " x " << r.height << " from (" << r.x << ", " << r.y << ")]";
}
typedef Rect_<int> Rect2i;
typedef Rect_<int> Rect;

// ---------------------------------------------------------------------------
// Mat: a 2-D, continuous, reference-counted array of rows x cols elements of
// `type` (depth and channel count).
class Mat {
public:
    int flags = 0;  // the type
    int dims = 0;
    int rows = 0, cols = 0;
    uchar* data = nullptr;
    size_t step = 0;  // bytes per row

    Mat() {}
    Mat(int r, int c, int type) { create(r, c, type); }
    Mat(Size sz, int type) { create(sz.height, sz.width, type); }
    Mat(int r, int c, int type, const Scalar& s) {
        create(r, c, type);
        *this = s;
    }
    Mat(Size sz, int type, const Scalar& s) {
        create(sz.height, sz.width, type);
        *this = s;
    }
    // External data, not owned.
    Mat(int r, int c, int type, void* ext, size_t stp = 0) {
        flags = type;
        dims = 2;
        rows = r;
        cols = c;
        data = static_cast<uchar*>(ext);
        step = stp ? stp : (size_t)c * elemSize();
    }
    Mat(Size sz, int type, void* ext, size_t stp = 0) : Mat(sz.height, sz.width, type, ext, stp) {}

    void create(int r, int c, int type) {
        if (data && rows == r && cols == c && flags == type) return;
        flags = type;
        dims = 2;
        rows = r;
        cols = c;
        step = (size_t)c * elemSize();
        const size_t bytes = std::max<size_t>(1, step * (size_t)r);
        holder_ = std::shared_ptr<uchar>(new uchar[bytes], std::default_delete<uchar[]>());
        data = holder_.get();
    }
    void create(Size sz, int type) { create(sz.height, sz.width, type); }
    void release() {
        holder_.reset();
        data = nullptr;
        rows = cols = 0;
        step = 0;
    }

    int type() const { return flags; }
    int depth() const { return CV_MAT_DEPTH(flags); }
    int channels() const { return CV_MAT_CN(flags); }
    size_t elemSize1() const {
        static const size_t sz[] = {1, 1, 2, 2, 4, 4, 8, 2};
        return sz[depth()];
    }
    size_t elemSize() const { return elemSize1() * (size_t)channels(); }
    size_t total() const { return (size_t)rows * (size_t)cols; }
    bool empty() const { return data == nullptr || total() == 0; }
    bool isContinuous() const { return step == (size_t)cols * elemSize(); }
    Size size() const { return Size(cols, rows); }

    template <typename T>
    T& at(int y, int x) {
        return reinterpret_cast<T*>(data + (size_t)y * step)[x];
    }
    template <typename T>
    const T& at(int y, int x) const {
        return reinterpret_cast<const T*>(data + (size_t)y * step)[x];
    }
    template <typename T>
    T& at(Point p) {
        return at<T>(p.y, p.x);
    }
    template <typename T>
    const T& at(Point p) const {
        return at<T>(p.y, p.x);
    }
    template <typename T>
    T& at(int i) {
        return reinterpret_cast<T*>(data)[i];
    }
    template <typename T>
    const T& at(int i) const {
        return reinterpret_cast<const T*>(data)[i];
    }
    template <typename T = uchar>
    T* ptr(int y = 0) {
        return reinterpret_cast<T*>(data + (size_t)y * step);
    }
    template <typename T = uchar>
    const T* ptr(int y = 0) const {
        return reinterpret_cast<const T*>(data + (size_t)y * step);
    }

    // A header for the region `r`, sharing this Mat's data.
    Mat operator()(const Rect& r) const {
        CV_Assert(r.x >= 0 && r.y >= 0 && r.width >= 0 && r.height >= 0 && r.x + r.width <= cols &&
                  r.y + r.height <= rows);
        Mat m(*this);
        m.data = data + (size_t)r.y * step + (size_t)r.x * elemSize();
        m.rows = r.height;
        m.cols = r.width;
        return m;
    }

    Mat clone() const {
        Mat m;
        copyTo(m);
        return m;
    }
    void copyTo(Mat& dst) const {
        if (empty()) {
            dst.release();
            return;
        }
        if (dst.data == data) return;
        dst.create(rows, cols, flags);
        for (int y = 0; y < rows; ++y) std::memcpy(dst.ptr(y), ptr(y), (size_t)cols * elemSize());
    }
    // Elements where the (one-channel, 8-bit) mask is nonzero; a destination
    // that had to be (re)allocated starts at zero.
    void copyTo(Mat& dst, const Mat& mask) const {
        if (mask.empty()) {
            copyTo(dst);
            return;
        }
        CV_Assert(mask.depth() == CV_8U && mask.channels() == 1 && mask.rows == rows && mask.cols == cols);
        uchar* before = dst.data;
        if (dst.data == data) {
            return;  // copying onto itself changes nothing
        }
        dst.create(rows, cols, flags);
        if (dst.data != before) dst = Scalar(0);
        const size_t es = elemSize();
        for (int y = 0; y < rows; ++y)
            for (int x = 0; x < cols; ++x)
                if (mask.at<uchar>(y, x)) std::memcpy(dst.ptr(y) + x * es, ptr(y) + x * es, es);
    }

    Mat& setTo(const Scalar& s, const Mat& mask = Mat());
    Mat& operator=(const Scalar& s) { return setTo(s); }
    void convertTo(Mat& dst, int rtype, double alpha = 1, double beta = 0) const;

    static Mat zeros(int r, int c, int type) { return Mat(r, c, type, Scalar(0)); }
    static Mat zeros(Size sz, int type) { return Mat(sz, type, Scalar(0)); }
    static Mat ones(int r, int c, int type) { return Mat(r, c, type, Scalar(1)); }
    static Mat ones(Size sz, int type) { return Mat(sz, type, Scalar(1)); }

    // Element access as double, channel c of element i (row-major).
    double get(size_t i, int c) const;
    void put(size_t i, int c, double v);

protected:
    std::shared_ptr<uchar> holder_;
};

namespace shim {
template <typename T>
inline double load(const uchar* p) {
    return (double)*reinterpret_cast<const T*>(p);
}
template <typename T>
inline void store(uchar* p, double v) {
    *reinterpret_cast<T*>(p) = saturate_cast<T>(v);
}
// Calls f.template operator()<T>() with T the C++ type of `depth`.
template <typename F>
inline void dispatch(int depth, F&& f) {
    switch (depth) {
    case CV_8U: f((uchar)0); break;
    case CV_8S: f((schar)0); break;
    case CV_16U: f((ushort)0); break;
    case CV_16S: f((short)0); break;
    case CV_32S: f((int)0); break;
    case CV_32F: f((float)0); break;
    case CV_64F: f((double)0); break;
    default: shim_fail("unsupported depth");
    }
}
}  // namespace shim

inline double Mat::get(size_t i, int c) const {
    const size_t y = i / (size_t)cols, x = i % (size_t)cols;
    const uchar* p = data + y * step + x * elemSize() + (size_t)c * elemSize1();
    double r = 0;
    shim::dispatch(depth(), [&](auto t) { r = shim::load<decltype(t)>(p); });
    return r;
}
inline void Mat::put(size_t i, int c, double v) {
    const size_t y = i / (size_t)cols, x = i % (size_t)cols;
    uchar* p = data + y * step + x * elemSize() + (size_t)c * elemSize1();
    shim::dispatch(depth(), [&](auto t) { shim::store<decltype(t)>(p, v); });
}

inline Mat& Mat::setTo(const Scalar& s, const Mat& mask) {
    if (empty()) return *this;
    const int cn = channels();
    CV_Assert(cn <= 4);
    if (!mask.empty())
        CV_Assert(mask.depth() == CV_8U && mask.channels() == 1 && mask.rows == rows && mask.cols == cols);
    shim::dispatch(depth(), [&](auto t) {
        typedef decltype(t) T;
        T v[4];
        for (int c = 0; c < cn; ++c) v[c] = saturate_cast<T>(s.val[c]);
        for (int y = 0; y < rows; ++y) {
            T* row = ptr<T>(y);
            for (int x = 0; x < cols; ++x) {
                if (!mask.empty() && !mask.at<uchar>(y, x)) continue;
                for (int c = 0; c < cn; ++c) row[x * cn + c] = v[c];
            }
        }
    });
    return *this;
}

inline void Mat::convertTo(Mat& dst, int rtype, double alpha, double beta) const {
    const int ddepth = rtype < 0 ? depth() : CV_MAT_DEPTH(rtype);
    Mat src = *this;  // keeps the data alive if dst aliases this
    Mat out(rows, cols, CV_MAKETYPE(ddepth, channels()));
    const size_t n = total();
    const int cn = channels();
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < cn; ++c) out.put(i, c, src.get(i, c) * alpha + beta);
    dst = out;
}

// Mat_<T>: a Mat whose element type is T.
template <typename T>
class Mat_ : public Mat {
public:
    typedef T value_type;
    Mat_() { flags = DataType<T>::type; }
    Mat_(int r, int c) : Mat(r, c, DataType<T>::type) {}
    Mat_(int r, int c, const T& v) : Mat(r, c, DataType<T>::type) { fill(v); }
    explicit Mat_(Size sz) : Mat(sz, DataType<T>::type) {}
    Mat_(Size sz, const T& v) : Mat(sz, DataType<T>::type) { fill(v); }
    Mat_(const Mat& m) { assign_from(m); }
    Mat_(const Mat_& m) = default;
    Mat_& operator=(const Mat& m) {
        assign_from(m);
        return *this;
    }
    Mat_& operator=(const Mat_& m) = default;
    Mat_& operator=(const Scalar& s) {
        setTo(s);
        return *this;
    }

    T& operator()(int y, int x) { return at<T>(y, x); }
    const T& operator()(int y, int x) const { return at<T>(y, x); }
    T& operator()(Point p) { return at<T>(p.y, p.x); }
    const T& operator()(Point p) const { return at<T>(p.y, p.x); }

    static Mat_ zeros(Size sz) { return Mat_(Mat::zeros(sz, DataType<T>::type)); }
    static Mat_ zeros(int r, int c) { return Mat_(Mat::zeros(r, c, DataType<T>::type)); }
    static Mat_ ones(Size sz) { return Mat_(Mat::ones(sz, DataType<T>::type)); }
    static Mat_ ones(int r, int c) { return Mat_(Mat::ones(r, c, DataType<T>::type)); }

    Mat_ clone() const { return Mat_(Mat::clone()); }

private:
    void fill(const T& v) {
        for (int y = 0; y < rows; ++y)
            for (int x = 0; x < cols; ++x) at<T>(y, x) = v;
    }
    void assign_from(const Mat& m) {
        if (m.data == nullptr) {
            static_cast<Mat&>(*this) = Mat();
            flags = DataType<T>::type;
            return;
        }
        if (m.type() == DataType<T>::type) {
            static_cast<Mat&>(*this) = m;
            return;
        }
        CV_Assert(m.channels() == DataType<T>::channels);
        Mat c;
        m.convertTo(c, DataType<T>::type);
        static_cast<Mat&>(*this) = c;
    }
};

typedef Mat_<uchar> Mat1b;
typedef Mat_<Vec3b> Mat3b;
typedef Mat_<ushort> Mat1w;
typedef Mat_<int> Mat1i;
typedef Mat_<float> Mat1f;
typedef Mat_<Vec2f> Mat2f;
typedef Mat_<Vec3f> Mat3f;
typedef Mat_<Vec4f> Mat4f;
typedef Mat_<double> Mat1d;

// ---------------------------------------------------------------------------
// Element-wise operations.
namespace shim {

template <typename Op>
inline Mat compare_scalar(const Mat& a, double s, Op op) {
    Mat r(a.rows, a.cols, CV_MAKETYPE(CV_8U, a.channels()));
    const size_t n = a.total();
    const int cn = a.channels();
    dispatch(a.depth(), [&](auto t) {
        typedef decltype(t) T;
        const T sv = saturate_cast<T>(s);
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < cn; ++c) {
                const T v = (T)a.get(i, c);
                r.put(i, c, op(v, sv) ? 255 : 0);
            }
    });
    return r;
}
template <typename Op>
inline Mat compare_mat(const Mat& a, const Mat& b, Op op) {
    CV_Assert(a.type() == b.type() && a.rows == b.rows && a.cols == b.cols);
    Mat r(a.rows, a.cols, CV_MAKETYPE(CV_8U, a.channels()));
    const size_t n = a.total();
    const int cn = a.channels();
    dispatch(a.depth(), [&](auto t) {
        typedef decltype(t) T;
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < cn; ++c) r.put(i, c, op((T)a.get(i, c), (T)b.get(i, c)) ? 255 : 0);
    });
    return r;
}
template <typename Op>
inline Mat binary(const Mat& a, const Mat& b, Op op) {
    CV_Assert(a.type() == b.type() && a.rows == b.rows && a.cols == b.cols);
    Mat r(a.rows, a.cols, a.type());
    const size_t n = a.total();
    const int cn = a.channels();
    dispatch(a.depth(), [&](auto t) {
        typedef decltype(t) T;
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < cn; ++c) {
                const T x = (T)a.get(i, c), y = (T)b.get(i, c);
                if constexpr (std::is_floating_point<T>::value) {
                    const T z = op(x, y);
                    r.put(i, c, (double)z);
                } else {
                    r.put(i, c, (double)op((double)x, (double)y));
                }
            }
    });
    return r;
}

}  // namespace shim

#define CV_SHIM_CMP(OP)                                                                                     \
    inline Mat operator OP(const Mat& a, double s) {                                                        \
        return shim::compare_scalar(a, s, [](auto x, auto y) { return x OP y; });                           \
    }                                                                                                       \
    inline Mat operator OP(const Mat& a, const Mat& b) {                                                    \
        return shim::compare_mat(a, b, [](auto x, auto y) { return x OP y; });                              \
    }
CV_SHIM_CMP(>)
CV_SHIM_CMP(<)
CV_SHIM_CMP(>=)
CV_SHIM_CMP(<=)
CV_SHIM_CMP(==)
CV_SHIM_CMP(!=)
#undef CV_SHIM_CMP

inline Mat operator+(const Mat& a, const Mat& b) {
    return shim::binary(a, b, [](auto x, auto y) { return x + y; });
}
inline Mat operator-(const Mat& a, const Mat& b) {
    return shim::binary(a, b, [](auto x, auto y) { return x - y; });
}
inline Mat operator/(const Mat& a, const Mat& b) {
    return shim::binary(a, b, [](auto x, auto y) { return x / y; });
}
inline Mat max(const Mat& a, const Mat& b) {
    return shim::binary(a, b, [](auto x, auto y) { return std::max(x, y); });
}
inline Mat min(const Mat& a, const Mat& b) {
    return shim::binary(a, b, [](auto x, auto y) { return std::min(x, y); });
}
inline Mat operator*(const Mat& a, double s) {
    Mat r;
    a.convertTo(r, -1, s, 0);
    return r;
}
inline Mat operator*(double s, const Mat& a) { return a * s; }
inline Mat& operator*=(Mat& a, double s) {
    a.convertTo(a, -1, s, 0);
    return a;
}
inline Mat& operator/=(Mat& a, double s) {
    a.convertTo(a, -1, 1.0 / s, 0);
    return a;
}
namespace shim {
template <typename Op>
inline Mat with_scalar(const Mat& a, Op op) {
    Mat r(a.rows, a.cols, a.type());
    const size_t n = a.total();
    const int cn = a.channels();
    dispatch(a.depth(), [&](auto t) {
        typedef decltype(t) T;
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < cn; ++c) r.put(i, c, (double)op((T)a.get(i, c)));
    });
    return r;
}
}  // namespace shim
// Mat (op) scalar on floating-point Mats, in the element type.
inline Mat operator/(double s, const Mat& a) {
    return shim::with_scalar(a, [s](auto x) { return (decltype(x))s / x; });
}
inline Mat operator-(const Mat& a, double s) {
    return shim::with_scalar(a, [s](auto x) { return x - (decltype(x))s; });
}
inline Mat operator+(const Mat& a, double s) {
    return shim::with_scalar(a, [s](auto x) { return x + (decltype(x))s; });
}
inline Mat operator+(double s, const Mat& a) { return a + s; }
inline Mat operator/(const Mat& a, double s) {
    return shim::with_scalar(a, [s](auto x) { return x / (decltype(x))s; });
}
inline double max(double a, double b) { return std::max(a, b); }
inline double min(double a, double b) { return std::min(a, b); }

// Splits an n-channel Mat into n one-channel Mats, and back.
inline void split(const Mat& m, Mat* mv) {
    const int cn = m.channels();
    const size_t n = m.total();
    for (int c = 0; c < cn; ++c) {
        Mat o(m.rows, m.cols, CV_MAKETYPE(m.depth(), 1));
        const size_t es = m.elemSize1();
        for (size_t i = 0; i < n; ++i) {
            const size_t y = i / (size_t)m.cols, x = i % (size_t)m.cols;
            std::memcpy(o.ptr(y) + x * es, m.ptr(y) + x * m.elemSize() + c * es, es);
        }
        mv[c] = o;
    }
}
inline void split(const Mat& m, std::vector<Mat>& mv) {
    mv.resize(m.channels());
    split(m, mv.data());
}
inline void merge(const Mat* mv, size_t count, Mat& dst) {
    CV_Assert(count >= 1);
    const Mat first = mv[0];
    const int cn = (int)count;
    Mat o(first.rows, first.cols, CV_MAKETYPE(first.depth(), cn));
    const size_t es = first.elemSize1();
    for (int c = 0; c < cn; ++c) {
        CV_Assert(mv[c].type() == first.type() && mv[c].size() == first.size() && mv[c].channels() == 1);
        for (int y = 0; y < first.rows; ++y)
            for (int x = 0; x < first.cols; ++x)
                std::memcpy(o.ptr(y) + x * o.elemSize() + c * es, mv[c].ptr(y) + x * es, es);
    }
    dst = o;
}
inline void merge(const std::vector<Mat>& mv, Mat& dst) { merge(mv.data(), mv.size(), dst); }

inline void flip(const Mat& src, Mat& dst, int code) {
    Mat s = src.clone();
    Mat o(src.rows, src.cols, src.type());
    const size_t es = src.elemSize();
    for (int y = 0; y < src.rows; ++y)
        for (int x = 0; x < src.cols; ++x) {
            const int sy = code == 0 || code < 0 ? src.rows - 1 - y : y;
            const int sx = code > 0 || code < 0 ? src.cols - 1 - x : x;
            std::memcpy(o.ptr(y) + x * es, s.ptr(sy) + sx * es, es);
        }
    dst = o;
}

// Paths the harness never runs.
inline void transform(const Mat&, Mat&, const Matx22f&) { shim_fail("transform is not part of the stand-in"); }

}  // namespace cv
