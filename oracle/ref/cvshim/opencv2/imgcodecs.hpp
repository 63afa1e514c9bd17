// TEST INFRASTRUCTURE ONLY: image files are not part of the OpenCV stand-in.
#pragma once
#include "core.hpp"

namespace cv {
enum ImreadModes { IMREAD_UNCHANGED = -1, IMREAD_GRAYSCALE = 0, IMREAD_COLOR = 1, IMREAD_ANYDEPTH = 2 };
inline bool imwrite(const std::string&, const Mat&) { shim_fail("imwrite is not part of the stand-in"); }
inline Mat imread(const std::string&, int = IMREAD_COLOR) { shim_fail("imread is not part of the stand-in"); }
}  // namespace cv
