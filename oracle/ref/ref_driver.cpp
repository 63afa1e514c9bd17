// TEST INFRASTRUCTURE ONLY.
//
// C entry points over the reference's own CPU synthesis code, compiled
// unmodified from the reference tree (rvs/src/*.cpp) against the OpenCV
// stand-in in cvshim/ (see Makefile).  The tests call these through ctypes
// (oracle/ref.py) to check the oracle (rvs_oracle.cpp) stage by stage
// against the reference itself.  The product library never links or loads
// this code.
//
// What runs here is the reference's code: camera parsing (Parameters.cpp,
// JsonParser.cpp), relative pose (SpaceTransformer.cpp), image positions,
// unprojection and projection ((Perspective|Equirectangular)(Un)Projector.cpp,
// Unprojector.cpp), the triangle raster (transform.cpp), blending
// (BlendedView.cpp, blending.cpp), inpainting (inpainting.cpp, View.cpp) and
// the colour writer (image_writing.cpp).  Restated here, because the
// reference keeps them in a translation unit that cannot run without a
// device or in an anonymous namespace:
//   - SynthesizedView::computeBasicMode's glue (SynthesizedView.cpp:273-299):
//     affine_transform (:68-79, R * x + t per pixel), the uv scale
//     (cv::transform with Matx22f(sx, 0, 0, sy), evaluated as OpenCV's
//     float transform does: m0 * u + m1 * v + 0) and
//     SynthetisedViewTriangle::transform's quality = validity / depth
//     (:428-441);
//   - the map set-up of inpaint_color's nearest mode (inpainting.cpp:179-188)
//     for ref_inpaint_sources, which then runs the reference's
//     compute_nearest.
// OpenCV itself is the stand-in's restatement (cvshim/opencv2/core.hpp).
#include <cstdio>
#include <cstring>
#include <exception>
#include <sstream>
#include <string>
#include <vector>

#include "BlendedView.hpp"
#include "Config.hpp"
#include "JsonParser.hpp"
#include "Parameters.hpp"
#include "SpaceTransformer.hpp"
#include "View.hpp"
#include "image_loading.hpp"
#include "image_writing.hpp"
#include "inpainting.hpp"
#include "transform.hpp"

// Defined in the reference's inpainting.cpp without a header declaration.
namespace rvs {
namespace detail {
void compute_nearest(cv::Mat& map);
}
}  // namespace rvs

namespace {

std::string g_err;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    } catch (...) {
        g_err = "unknown exception";
        return 1;
    }
}

cv::Mat wrap(const float* p, int w, int h, int cn) {
    cv::Mat m(h, w, CV_MAKETYPE(CV_32F, cn));
    std::memcpy(m.data, p, sizeof(float) * (size_t)w * h * cn);
    return m;
}

void unwrap(const cv::Mat& m, float* p) {
    CV_Assert(m.depth() == CV_32F);
    for (int y = 0; y < m.rows; ++y) std::memcpy(p + (size_t)y * m.cols * m.channels(), m.ptr(y), (size_t)m.cols * m.elemSize());
}

struct Cam {
    rvs::Parameters params;
};

// SynthesizedView.cpp:273-299 up to the raster: positions, unprojection,
// R * x + t, projection and the oversampling scale.
void warp_view(const rvs::Parameters& in, const rvs::Parameters& virt, const cv::Mat1f& depth, cv::Mat2f& uv_out,
               cv::Mat1f& vdepth, rvs::WrappingMethod& wrapping) {
    rvs::GenericTransformer t;
    t.set_inputPosition(&in);
    t.set_targetPosition(&virt);
    const cv::Matx33f R = t.get_rotation();
    const cv::Vec3f tr = t.get_translation();
    cv::Mat2f uv = t.generateImagePos();
    cv::Mat3f xyz = t.unproject(uv, depth);
    cv::Mat3f vxyz(xyz.size());
    for (int i = 0; i != vxyz.rows; ++i)
        for (int j = 0; j != vxyz.cols; ++j) vxyz(i, j) = R * xyz(i, j) + tr;
    cv::Mat2f vuv = t.project(vxyz, vdepth, wrapping);
    const cv::Size vs = virt.getSize();
    const cv::Size os(int(0.5f + vs.width * rvs::detail::g_rescale), int(0.5f + vs.height * rvs::detail::g_rescale));
    const float sx = float(os.width) / vs.width, sy = float(os.height) / vs.height;
    uv_out = cv::Mat2f(vuv.size());
    for (int i = 0; i != vuv.rows; ++i)
        for (int j = 0; j != vuv.cols; ++j) {
            const cv::Vec2f p = vuv(i, j);
            uv_out(i, j) = cv::Vec2f(sx * p[0] + 0.f * p[1] + 0.f, 0.f * p[0] + sy * p[1] + 0.f);
        }
}

// SynthetisedViewTriangle::transform (SynthesizedView.cpp:428-441).
void raster_view(const cv::Mat3f& color, const cv::Mat2f& uv, const cv::Mat1f& vdepth, cv::Size out, bool wrap,
                 cv::Mat3f& ocolor, cv::Mat1f& odepth, cv::Mat1f& oquality, cv::Mat1f& ovalidity) {
    cv::Mat1f depth, validity;
    ocolor = rvs::detail::transform_trianglesMethod(color, vdepth, uv, out, depth, validity, wrap);
    odepth = depth;
    ovalidity = validity;
    oquality = cv::Mat1f(validity / depth);
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_set_precision(float p) { rvs::detail::g_rescale = p; }

void ref_set_resize_ties_up(int on) { cv::cvshim_set_resize_ties_up(on); }

// A camera from one element of a camera-parameter file's "cameras" array.
void* ref_camera_new(const char* json_text) {
    Cam* c = nullptr;
    if (guarded([&] {
            std::istringstream s(json_text);
            c = new Cam{rvs::Parameters::readFrom(json::Node::readFrom(s))};
        }))
        return nullptr;
    return c;
}

void ref_camera_free(void* c) { delete static_cast<Cam*>(c); }

// SpaceTransformer::get_rotation / get_translation (SpaceTransformer.cpp:77-92).
int ref_relative_pose(void* in, void* virt, float* R, float* t) {
    return guarded([&] {
        rvs::GenericTransformer g;
        g.set_inputPosition(&static_cast<Cam*>(in)->params);
        g.set_targetPosition(&static_cast<Cam*>(virt)->params);
        const cv::Matx33f r = g.get_rotation();
        const cv::Vec3f v = g.get_translation();
        for (int i = 0; i < 9; ++i) R[i] = r.val[i];
        for (int i = 0; i < 3; ++i) t[i] = v[i];
    });
}

// The warp of one input view into the virtual camera: (u, v) per input pixel
// (scaled by the oversampling factor), the virtual depth and the wrapping
// flag.  depth: the decoded input depth, H*W floats.
int ref_warp(void* in, void* virt, const float* depth, float* uv, float* vdepth, int* wrapping) {
    return guarded([&] {
        const rvs::Parameters& pin = static_cast<Cam*>(in)->params;
        const cv::Size s = pin.getSize();
        cv::Mat1f d = wrap(depth, s.width, s.height, 1);
        cv::Mat2f ouv;
        cv::Mat1f ovd;
        rvs::WrappingMethod wm;
        warp_view(pin, static_cast<Cam*>(virt)->params, d, ouv, ovd, wm);
        unwrap(ouv, uv);
        unwrap(ovd, vdepth);
        *wrapping = wm == rvs::WrappingMethod::horizontal;
    });
}

// transform_trianglesMethod (transform.cpp:148-181) of one warped view and
// the synthesized view's quality (validity / depth).
int ref_raster(const float* color, const float* vdepth, const float* uv, int w, int h, int wo, int ho, int wrapping,
               float* out_color, float* out_depth, float* out_quality, float* out_validity) {
    return guarded([&] {
        cv::Mat3f c = wrap(color, w, h, 3);
        cv::Mat1f d = wrap(vdepth, w, h, 1);
        cv::Mat2f p = wrap(uv, w, h, 2);
        cv::Mat3f oc;
        cv::Mat1f od, oq, ov;
        raster_view(c, p, d, cv::Size(wo, ho), wrapping != 0, oc, od, oq, ov);
        unwrap(oc, out_color);
        unwrap(od, out_depth);
        unwrap(oq, out_quality);
        unwrap(ov, out_validity);
    });
}

// BlendedViewSimple (exponent) or BlendedViewMultiSpec (ms = 1: low, high)
// over n synthesized views in order (BlendedView.cpp:63-88, 180-212).
int ref_blend(int n, const float* const* colors, const float* const* depths, const float* const* qualities,
              const float* const* validities, int wo, int ho, float exponent, int ms, float low, float high,
              float* out_color, float* out_quality, float* out_depth, float* out_validity) {
    return guarded([&] {
        std::unique_ptr<rvs::BlendedView> b;
        if (ms)
            b.reset(new rvs::BlendedViewMultiSpec(low, high));
        else
            b.reset(new rvs::BlendedViewSimple(exponent));
        for (int i = 0; i < n; ++i) {
            rvs::View v(wrap(colors[i], wo, ho, 3), wrap(depths[i], wo, ho, 1), wrap(qualities[i], wo, ho, 1),
                        wrap(validities[i], wo, ho, 1));
            b->blend(v);
        }
        unwrap(b->get_color(), out_color);
        unwrap(b->get_quality(), out_quality);
        unwrap(b->get_depth(), out_depth);
        unwrap(b->get_validity(), out_validity);
    });
}

// inpaintBasicMode (inpainting.cpp:213-223) of a blended colour and quality.
int ref_inpaint(const float* color, const float* quality, int w, int h, float* out_color) {
    return guarded([&] {
        rvs::View v(wrap(color, w, h, 3), cv::Mat1f(), wrap(quality, w, h, 1), cv::Mat1f());
        cv::Mat r = rvs::detail::inpaintBasicMode(v);
        unwrap(r, out_color);
    });
}

// The (x, y) source of every pixel after compute_nearest
// (inpainting.cpp:104-136) on the map inpaint_color sets up for `holes`
// (nonzero = hole); `sources` holds w*h pairs.
int ref_inpaint_sources(const unsigned char* holes, int w, int h, int* sources) {
    return guarded([&] {
        cv::Mat map = cv::Mat::zeros(cv::Size(w, h), CV_32SC3);
        for (int x = 0; x < map.cols; x++)
            for (int y = 0; y < map.rows; y++) {
                map.at<cv::Vec3i>(y, x) = cv::Vec3i(x, y, 0);
                if (holes[(size_t)y * w + x]) map.at<cv::Vec3i>(y, x)[2] = map.cols + map.rows;
            }
        rvs::detail::compute_nearest(map);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const cv::Vec3i p = map.at<cv::Vec3i>(y, x);
                sources[((size_t)y * w + x) * 2 + 0] = p[0];
                sources[((size_t)y * w + x) * 2 + 1] = p[1];
            }
    });
}

// write_color (image_writing.cpp:182-203) of a colour image to `path` for
// the virtual camera `virt` (frame 0: the file is created).
int ref_write_color(const float* color, int w, int h, void* virt, const char* path) {
    return guarded([&] {
        rvs::write_color(path, cv::Mat3f(wrap(color, w, h, 3)), 0, static_cast<Cam*>(virt)->params);
    });
}

// write_depth / write_maskedDepth / write_mask (image_writing.cpp:226-302)
// of an output-sized depth map (and mask, nonzero = masked) to `path` for
// the virtual camera `virt`, frame 0.  kind: 0 depth, 1 masked depth, 2 mask.
int ref_write_aux(int kind, const float* depth, const unsigned char* mask, int w, int h, void* virt,
                  const char* path) {
    return guarded([&] {
        const rvs::Parameters& p = static_cast<Cam*>(virt)->params;
        cv::Mat1b m;
        if (mask) {
            m = cv::Mat1b(h, w);
            std::memcpy(m.data, mask, (size_t)w * h);
        }
        if (kind == 0)
            rvs::write_depth(path, cv::Mat1f(wrap(depth, w, h, 1)), 0, p);
        else if (kind == 1)
            rvs::write_maskedDepth(path, cv::Mat1f(wrap(depth, w, h, 1)), m, 0, p);
        else
            rvs::write_mask(path, m, 0, p);
    });
}

// One synthesized frame: every input view warped, rasterised and blended in
// order, then inpainted (Pipeline.cpp:169-262 without the loaders and the
// file writer).  colors: decoded input colour per view (H*W*3), depths:
// decoded input depth (H*W).  Outputs at the raster size: the inpainted
// colour, and before inpainting the blended quality.
int ref_synthesize(int n, void* const* in, const float* const* colors, const float* const* depths, void* virt,
                   float exponent, int ms, float low, float high, float* out_color, float* out_quality) {
    return guarded([&] {
        const rvs::Parameters& pv = static_cast<Cam*>(virt)->params;
        const cv::Size vs = pv.getSize();
        const cv::Size os(int(0.5f + vs.width * rvs::detail::g_rescale),
                          int(0.5f + vs.height * rvs::detail::g_rescale));
        std::unique_ptr<rvs::BlendedView> b;
        if (ms)
            b.reset(new rvs::BlendedViewMultiSpec(low, high));
        else
            b.reset(new rvs::BlendedViewSimple(exponent));
        for (int i = 0; i < n; ++i) {
            const rvs::Parameters& pin = static_cast<Cam*>(in[i])->params;
            const cv::Size s = pin.getSize();
            cv::Mat2f uv;
            cv::Mat1f vdepth;
            rvs::WrappingMethod wm;
            warp_view(pin, pv, wrap(depths[i], s.width, s.height, 1), uv, vdepth, wm);
            cv::Mat3f oc;
            cv::Mat1f od, oq, ov;
            raster_view(wrap(colors[i], s.width, s.height, 3), uv, vdepth, os, wm == rvs::WrappingMethod::horizontal,
                        oc, od, oq, ov);
            rvs::View v(oc, od, oq, ov);
            b->blend(v);
        }
        unwrap(b->get_quality(), out_quality);
        cv::Mat r = rvs::detail::inpaintBasicMode(*b);
        unwrap(r, out_color);
    });
}

// The reference's loaders (image_loading.cpp:74-211: read_color and
// read_depth with the loader kernels of process_input_frame.cu) for frame
// `frame` of a colour and a depth file of camera `cam`: decoded colour
// (H*W*3) and depth (H*W), copied back from the device.  Needs a CUDA
// device.  The loaders fix their colour and depth scale at their first call
// in the process (static const, image_loading.cpp:134, 193).
int ref_load_view(void* cam, const char* color_path, const char* depth_path, int frame, float* color, float* depth) {
    return guarded([&] {
        const rvs::Parameters& p = static_cast<Cam*>(cam)->params;
        const cv::Size s = p.getSize();
        float3* dc = rvs::read_color(color_path, frame, p);
        float* dd = rvs::read_depth(depth_path, frame, p);
        cudaError_t e1 = cudaMemcpy(color, dc, sizeof(float3) * (size_t)s.area(), cudaMemcpyDeviceToHost);
        cudaError_t e2 = cudaMemcpy(depth, dd, sizeof(float) * (size_t)s.area(), cudaMemcpyDeviceToHost);
        cudaFree(dc);
        cudaFree(dd);
        if (e1 != cudaSuccess || e2 != cudaSuccess)
            throw std::runtime_error(std::string("copy from the device failed: ") +
                                     cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    });
}

}  // extern "C"
