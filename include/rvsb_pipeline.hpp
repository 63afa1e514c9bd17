/* C++ host pipeline over the C ABI (rvsb.h) with the hook points of the
 * reference's Pipeline class (rvs/src/Pipeline.hpp:79-185): a derived class
 * provides the configuration and the input loader and chooses which outputs
 * to save; execute() runs the frame loop of Pipeline::execute /
 * computeView (rvs/src/Pipeline.cpp:76-94, 169-345) on the B200 backend, with
 * the next frame's inputs loaded and the previous frame's outputs saved on
 * worker threads while the current frame is synthesised (the reference's
 * asynchronous loader and writer, Pipeline.cpp:215-245, 283-291).
 *
 * Header-only; link librvsb and the CUDA runtime. */
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <future>
#include <stdexcept>
#include <string>
#include <vector>

#include "rvsb.h"

namespace rvsb {

/* Raw planes of one input view at one frame, as read_color_YUV and
 * read_depth_YUV read them (rvs/src/image_loading.cpp:74-211): Y W*H, U and V
 * (W/2)*(H/2) colour samples, and the W*H luma plane of the depth map
 * (W x H the camera's size; with an input Crop_region, the first W*H
 * samples of the padded depth frame's luma: rvsb_config_input_crop). */
struct InputPlanes {
    std::vector<uint16_t> y, u, v, depth;
};

class Pipeline {
public:
    virtual ~Pipeline() { release(); }

    /* Pipeline::execute (Pipeline.cpp:76-94): output frame f of virtual view
     * 0 from input frame StartFrame + f, mapped into the input files with the
     * ping-pong rule of getExtendedIndex (Pipeline.cpp:157-167), with the pose
     * trace applied (Pipeline.cpp:173-181).  Returns the number of output
     * frames; throws std::runtime_error with the backend's message on failure
     * and std::logic_error where a wanted output has no save function. */
    int execute() {
        const rvsb_config* cfg = getConfig();
        if (rvsb_config_num_virtual(cfg) != 1)
            throw std::runtime_error("exactly one virtual camera is supported");
        int start = 0, n_frames = 1, n_out = 1;
        rvsb_config_frames(cfg, &start, &n_frames, &n_out);
        if (n_frames <= 0) throw std::runtime_error("Cannot extend frame index with zero input frames");
        setup();
        std::future<std::vector<InputPlanes>> next;
        std::future<void> saving;
        auto load_frame = [this, start, n_frames](int virtualFrame) {
            const int frame = extendedIndex(start + virtualFrame, n_frames);
            std::vector<InputPlanes> views(cams_.size());
            for (size_t i = 0; i < cams_.size(); ++i) views[i] = loadInputView(frame, (int)i, cams_[i]);
            return views;
        };
        next = std::async(std::launch::async, load_frame, 0);
        for (int virtualFrame = 0; virtualFrame < n_out; ++virtualFrame) {
            std::vector<InputPlanes> views = next.get();
            if (virtualFrame + 1 < n_out) next = std::async(std::launch::async, load_frame, virtualFrame + 1);
            computeView(start + virtualFrame, virtualFrame, 0, views, saving);
        }
        if (saving.valid()) saving.get();
        return n_out;
    }

protected:
    /* Config (Pipeline.hpp:95): the loaded configuration (rvsb_config_load). */
    virtual const rvsb_config* getConfig() const = 0;

    /* loadInputView (Pipeline.hpp:100): the raw planes of input view
     * `inputView` at file frame `inputFrame`.  Called from a worker thread. */
    virtual InputPlanes loadInputView(int inputFrame, int inputView, const rvsb_camera& parameters) = 0;

    /* wantColor .. wantMaskedDepth (Pipeline.hpp:105-127): which outputs to
     * produce; all off by default, as in the reference. */
    virtual bool wantColor() { return false; }
    virtual bool wantMaskedColor() { return false; }
    virtual bool wantMask() { return false; }
    virtual bool wantDepth() { return false; }
    virtual bool wantMaskedDepth() { return false; }

    /* saveColor .. saveMaskedDepth (Pipeline.hpp:130-152), called from a
     * worker thread with host data valid for the duration of the call:
     *   colour, masked colour: YUV420 samples, Y W*H then U and V (W/2)*(H/2);
     *   mask: W*H bytes, 255 where the blended validity is not above
     *         ValidityThreshold;
     *   depth, masked depth: W*H samples already encoded as write_depth
     *         encodes them (normalised disparity, BitDepthDepth).
     * W, H are the virtual camera's size (after its Crop_region). */
    virtual void saveColor(const uint16_t*, int, int, const rvsb_camera&) { notImplemented("saveColor"); }
    virtual void saveMaskedColor(const uint16_t*, int, int, const rvsb_camera&) { notImplemented("saveMaskedColor"); }
    virtual void saveMask(const uint8_t*, int, int, const rvsb_camera&) { notImplemented("saveMask"); }
    virtual void saveDepth(const uint16_t*, int, int, const rvsb_camera&) { notImplemented("saveDepth"); }
    virtual void saveMaskedDepth(const uint16_t*, int, int, const rvsb_camera&) { notImplemented("saveMaskedDepth"); }

    /* createBlender (Pipeline.hpp:182): the blending options of virtual view
     * `virtualView` (BlendingMethod, factors, Precision); by default those of
     * the configuration. */
    virtual rvsb_synth_params synthesisParameters(int /*virtualView*/) {
        rvsb_synth_params p;
        rvsb_config_synth_params(getConfig(), &p);
        return p;
    }

    /* createSpaceTransformer (Pipeline.hpp:187) with set_targetPosition
     * (Pipeline.cpp:171-181): the virtual camera of an output frame, by
     * default the configured camera with the pose trace entry of `inputFrame`. */
    virtual rvsb_camera virtualCamera(int inputFrame, int virtualView) {
        rvsb_camera c;
        if (rvsb_config_virtual_camera_at(getConfig(), virtualView, inputFrame, &c) != RVSB_OK)
            throw std::runtime_error("pose trace has no entry for frame " + std::to_string(inputFrame));
        return c;
    }

    /* CUDA device the pipeline runs on. */
    virtual int device() { return 0; }

private:
    static int extendedIndex(int outputFrame, int nInput) {
        const int group = outputFrame / nInput, rel = outputFrame % nInput;
        return group % 2 != 0 ? nInput - rel - 1 : rel;
    }
    static void notImplemented(const char* what) { throw std::logic_error(std::string(what) + " not implemented"); }

    void fail(rvsb_status st, const char* what) {
        throw std::runtime_error(std::string(what) + ": " + rvsb_status_string(st) + " (" +
                                 (ctx_ ? rvsb_last_error(ctx_) : "") + ")");
    }

    void setup() {
        if (ctx_) return;
        rvsb_status st = rvsb_create(device(), 0, &ctx_);
        if (st != RVSB_OK) fail(st, "rvsb_create");
        const rvsb_config* cfg = getConfig();
        cams_.resize(rvsb_config_num_inputs(cfg));
        for (size_t i = 0; i < cams_.size(); ++i) rvsb_config_input_camera(cfg, (int)i, &cams_[i]);
        if ((st = rvsb_scene_create(ctx_, cams_.data(), (int)cams_.size(), &scene_)) != RVSB_OK)
            fail(st, "rvsb_scene_create");
        rvsb_camera v0;
        rvsb_config_virtual_camera(cfg, 0, &v0);
        ny_ = (size_t)v0.width * v0.height;
        nc_ = (size_t)(v0.width / 2) * (v0.height / 2);
        auto dev = [](void** p, size_t bytes) {
            if (cudaMalloc(p, bytes) != cudaSuccess) throw std::runtime_error("cudaMalloc of the output buffers failed");
        };
        dev((void**)&d_yuv_, (ny_ + 2 * nc_) * 2);
        if (wantMaskedColor()) dev((void**)&d_masked_, (ny_ + 2 * nc_) * 2);
        if (wantMask()) dev((void**)&d_mask_, ny_);
        if (wantDepth()) dev((void**)&d_depth_, ny_ * 2);
        if (wantMaskedDepth()) dev((void**)&d_mdepth_, ny_ * 2);
    }

    void release() {
        cudaFree(d_yuv_);
        cudaFree(d_masked_);
        cudaFree(d_mask_);
        cudaFree(d_depth_);
        cudaFree(d_mdepth_);
        d_yuv_ = d_masked_ = d_depth_ = d_mdepth_ = nullptr;
        d_mask_ = nullptr;
        if (scene_) rvsb_scene_destroy(scene_);
        if (ctx_) rvsb_destroy(ctx_);
        scene_ = nullptr;
        ctx_ = nullptr;
    }

    struct Outputs {
        std::vector<uint16_t> yuv, masked, depth, mdepth;
        std::vector<uint8_t> mask;
    };

    /* computeView (Pipeline.cpp:169-345): upload, synthesise, then save on a
     * worker thread once the previous frame's saving has finished. */
    void computeView(int inputFrame, int virtualFrame, int virtualView, const std::vector<InputPlanes>& views,
                     std::future<void>& saving) {
        rvsb_status st;
        for (size_t i = 0; i < views.size(); ++i) {
            const InputPlanes& in = views[i];
            const rvsb_view_planes p{in.y.data(), in.u.data(), in.v.data(), in.depth.data()};
            if ((st = rvsb_scene_upload(scene_, (int)i, &p, 0, nullptr)) != RVSB_OK) fail(st, "rvsb_scene_upload");
        }
        const rvsb_camera virt = virtualCamera(inputFrame, virtualView);
        const rvsb_synth_params params = synthesisParameters(virtualView);
        const rvsb_yuv420 out{d_yuv_, d_yuv_ + ny_, d_yuv_ + ny_ + nc_};
        rvsb_aux_out aux{};
        aux.mask = d_mask_;
        if (d_masked_) aux.masked = rvsb_yuv420{d_masked_, d_masked_ + ny_, d_masked_ + ny_ + nc_};
        aux.depth = d_depth_;
        aux.masked_depth = d_mdepth_;
        aux.validity_threshold = rvsb_config_validity_threshold(getConfig());
        if ((st = rvsb_synthesize_aux(scene_, &virt, &params, &out, &aux, nullptr)) != RVSB_OK)
            fail(st, "synthesis");
        // The previous frame's saving must finish before its buffers are reused.
        if (saving.valid()) saving.get();
        Outputs& o = outputs_[virtualFrame % 2];
        auto copy = [](auto& host, const void* dev, size_t count) {
            host.resize(count);
            if (cudaMemcpy(host.data(), dev, count * sizeof(host[0]), cudaMemcpyDeviceToHost) != cudaSuccess)
                throw std::runtime_error("copying the outputs to the host failed");
        };
        if (wantColor()) copy(o.yuv, d_yuv_, ny_ + 2 * nc_);
        if (d_masked_) copy(o.masked, d_masked_, ny_ + 2 * nc_);
        if (wantMask()) copy(o.mask, d_mask_, ny_);
        if (d_depth_) copy(o.depth, d_depth_, ny_);
        if (d_mdepth_) copy(o.mdepth, d_mdepth_, ny_);
        saving = std::async(std::launch::async, [this, &o, virtualFrame, virtualView, virt]() {
            if (wantColor()) saveColor(o.yuv.data(), virtualFrame, virtualView, virt);
            if (wantMask()) saveMask(o.mask.data(), virtualFrame, virtualView, virt);
            if (wantMaskedColor()) saveMaskedColor(o.masked.data(), virtualFrame, virtualView, virt);
            if (wantDepth()) saveDepth(o.depth.data(), virtualFrame, virtualView, virt);
            if (wantMaskedDepth()) saveMaskedDepth(o.mdepth.data(), virtualFrame, virtualView, virt);
        });
    }

    rvsb_context* ctx_ = nullptr;
    rvsb_scene* scene_ = nullptr;
    std::vector<rvsb_camera> cams_;
    size_t ny_ = 0, nc_ = 0;
    uint16_t *d_yuv_ = nullptr, *d_masked_ = nullptr, *d_depth_ = nullptr, *d_mdepth_ = nullptr;
    uint8_t* d_mask_ = nullptr;
    Outputs outputs_[2];
};

}  // namespace rvsb
