// TEST INFRASTRUCTURE ONLY: definitions for the CUDA-mode host wrappers of
// rvs_cuda_lib that the compiled reference files refer to on paths the
// harness never runs (the reference's CUDA raster, blend and inpainting and
// its device quantisation); each throws.  The loader wrappers the
// reference's CPU mode does run (resizeImage, mergeFrame, formatDepth) come
// from its process_input_frame.cu, compiled as it is.
#include <stdexcept>

#include "blend_img.cuh"
#include "inpaint_img.cuh"

namespace {
[[noreturn]] void not_in_harness(const char* what) {
    throw std::runtime_error(std::string(what) + " (CUDA mode) is not part of the reference harness");
}
}  // namespace

void blendImages(float3*, float*, float*, float3*, float*, float*, cv::Size, cv::Vec3f, float3*&, float*&, float*&,
                 float) {
    not_in_harness("blendImages");
}

void inpaintImg(float3*&, cv::Size) { not_in_harness("inpaintImg"); }
