// TEST INFRASTRUCTURE ONLY: the image-processing part of the OpenCV
// stand-in (see opencv2/core.hpp).  resize covers the cases the reference's
// writer reaches at Precision 1 (identity, and 16-bit planes reduced by
// exactly 0.5 x 0.5); everything else here is declared so the reference's
// files compile and throws when called.
#pragma once
#include "core.hpp"

namespace cv {

enum InterpolationFlags { INTER_NEAREST = 0, INTER_LINEAR = 1, INTER_CUBIC = 2, INTER_AREA = 3 };
enum MorphShapes { MORPH_RECT = 0, MORPH_CROSS = 1, MORPH_ELLIPSE = 2 };
enum MorphTypes { MORPH_ERODE = 0, MORPH_DILATE = 1, MORPH_OPEN = 2, MORPH_CLOSE = 3 };
enum ColorConversionCodes { COLOR_BGR2YCrCb = 36, COLOR_YCrCb2BGR = 38 };
enum BorderTypes { BORDER_CONSTANT = 0, BORDER_REPLICATE = 1, BORDER_DEFAULT = 4 };

// 0: the 2x2 mean of a 0.5 x 0.5 reduction rounds half to even (OpenCV built
// with Intel IPP); 1: half up (without IPP).
inline int& cvshim_resize_ties_up() {
    static int mode = 0;
    return mode;
}
inline void cvshim_set_resize_ties_up(int on) { cvshim_resize_ties_up() = on ? 1 : 0; }

inline void resize(const Mat& src, Mat& dst, Size dsize, double fx = 0, double fy = 0,
                   int interpolation = INTER_LINEAR) {
    if (dsize.empty()) dsize = Size(cvRound(src.cols * fx), cvRound(src.rows * fy));
    if (dsize == src.size()) {
        if (dst.data != src.data) src.copyTo(dst);
        return;
    }
    const bool half = dsize.width * 2 == src.cols && dsize.height * 2 == src.rows;
    if (interpolation == INTER_LINEAR && half && src.depth() == CV_16U && src.channels() == 1) {
        Mat out(dsize, src.type());
        const int up = cvshim_resize_ties_up();
        for (int y = 0; y < dsize.height; ++y)
            for (int x = 0; x < dsize.width; ++x) {
                const unsigned s = (unsigned)src.at<ushort>(2 * y, 2 * x) + src.at<ushort>(2 * y, 2 * x + 1) +
                                   src.at<ushort>(2 * y + 1, 2 * x) + src.at<ushort>(2 * y + 1, 2 * x + 1);
                const unsigned q = s >> 2, r = s & 3;
                out.at<ushort>(y, x) = (ushort)(up ? (s + 2) >> 2 : q + (r > 2 || (r == 2 && (q & 1))));
            }
        dst = out;
        return;
    }
    shim_fail("resize: only identity and an exact 0.5 x 0.5 INTER_LINEAR reduction of 16-bit planes");
}

inline Mat getStructuringElement(int, Size, Point = Point(-1, -1)) {
    shim_fail("getStructuringElement is not part of the stand-in");
}
inline void erode(const Mat&, Mat&, const Mat&, Point = Point(-1, -1), int = 1) {
    shim_fail("erode is not part of the stand-in");
}
inline void dilate(const Mat&, Mat&, const Mat&, Point = Point(-1, -1), int = 1) {
    shim_fail("dilate is not part of the stand-in");
}
inline void morphologyEx(const Mat&, Mat&, int, const Mat&, Point = Point(-1, -1), int = 1) {
    shim_fail("morphologyEx is not part of the stand-in");
}
inline void cvtColor(const Mat&, Mat&, int, int = 0) { shim_fail("cvtColor is not part of the stand-in"); }
inline void bilateralFilter(const Mat&, Mat&, int, double, double, int = BORDER_DEFAULT) {
    shim_fail("bilateralFilter is not part of the stand-in");
}
inline void bitwise_and(const Mat&, const Mat&, Mat&, const Mat& = Mat()) {
    shim_fail("bitwise_and is not part of the stand-in");
}

}  // namespace cv
