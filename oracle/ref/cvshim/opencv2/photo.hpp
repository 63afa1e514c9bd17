// TEST INFRASTRUCTURE ONLY: OpenCV's own inpainting is declared for the
// reference's inpaint_all (never run by the harness) and throws.
#pragma once
#include "imgproc.hpp"

namespace cv {
enum { INPAINT_NS = 0, INPAINT_TELEA = 1 };
inline void inpaint(const Mat&, const Mat&, Mat&, double, int) { shim_fail("inpaint is not part of the stand-in"); }
}  // namespace cv
