// rvsb: command-line drop-in for the reference's `RVS <config.json>`
// (rvs/src/view_synthesis.cpp:64-176) on the B200 backend.
//
// Like the reference's Application (rvs/src/Application.cpp), it derives from
// the pipeline (include/rvsb_pipeline.hpp, the hook points of
// rvs/src/Pipeline.hpp) and supplies the configuration, the YUV file loader
// and the file writers: each output frame is appended to its file
// (truncated on frame 0, image_writing.cpp:72-76).  The loader reads frame
// `frame` at byte offset frame * frame size and wraps to 0 past the end of
// the file (image_loading.cpp:95-98).  Besides OutputFiles, the CPU-mode
// outputs MaskedOutputFiles, OutputMasks, DepthOutputFiles and
// MaskedDepthOutputFiles are written when configured (Pipeline.cpp:303-336).
// A virtual camera's Crop_region gives colour outputs of the region's size
// and depth and mask outputs of the padded resolution whose luma is zero,
// as the reference writes them (image_writing.cpp:262-267, 285-290).  An
// input camera's Crop_region is read as the reference reads it: colour
// frames of the region's size, depth frames of the padded size.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "rvsb.h"
#include "rvsb_pipeline.hpp"

namespace {

// Reads frame `frame` of a raw YUV file.  Errors throw with the reference's
// texts (image_loading.cpp:84-90, 155-161, 66-71); its CLI prints them and
// exits with status 1 (view_synthesis.cpp:171-175).
void read_at(const char* path, const char* kind, long offset_per_frame, int frame, std::vector<uint16_t*> dst,
             std::vector<size_t> counts) {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("Failed to read raw YUV ") + kind + " file \"" + path + "\"");
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    long off = offset_per_frame * frame;
    if (off >= size) off = 0;  // image_loading.cpp:95-98
    std::fseek(f, off, SEEK_SET);
    for (size_t k = 0; k < dst.size(); ++k) {
        if (std::fread(dst[k], 2, counts[k], f) != counts[k]) {
            std::fclose(f);
            throw std::runtime_error("Failed to read the expected amount of data");
        }
    }
    std::fclose(f);
}

void append(const char* path, bool first, const void* data, size_t bytes) {
    FILE* f = std::fopen(path, first ? "wb" : "ab");
    if (!f) throw std::runtime_error("Failed to open YUV output image");
    const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
    std::fclose(f);
    if (!ok) throw std::runtime_error(std::string("Failed to write \"") + path + "\"");
}

class Application : public rvsb::Pipeline {
public:
    Application(rvsb_config* cfg, int chroma_rounding) : cfg_(cfg), chroma_rounding_(chroma_rounding) {
        for (int k = 0; k < 5; ++k) files_[k] = rvsb_config_output_file(cfg, k, 0);
        rvsb_camera v;
        rvsb_config_virtual_camera(cfg, 0, &v);
        crop_[2] = v.width;
        crop_[3] = v.height;
        padded_[0] = v.width;
        padded_[1] = v.height;
        rvsb_config_virtual_crop(cfg, 0, crop_, padded_);
        // Depth and mask files carry constant chroma planes
        // (write_depth_YUV / write_mask_YUV, image_writing.cpp:104-139).
        neutral_ = (uint16_t)std::lround(0.5 * (1.0 + (double)((1u << v.bit_depth_depth) - 1u)));
        depth_chroma_ = v.depth_color_format == RVSB_FMT_YUV420;
        ny_ = (size_t)v.width * v.height;
        nc_ = (size_t)(v.width / 2) * (v.height / 2);
        py_ = (size_t)padded_[0] * padded_[1];
        pc_ = (size_t)(padded_[0] / 2) * (padded_[1] / 2);
    }

protected:
    const rvsb_config* getConfig() const override { return cfg_; }

    rvsb::InputPlanes loadInputView(int frame, int view, const rvsb_camera& c) override {
        nvtxRangePushA("rvsb cli: load input view");
        struct Pop {
            ~Pop() { nvtxRangePop(); }
        } pop;
        rvsb::InputPlanes p;
        const size_t cy = (size_t)c.width * c.height, cc = (size_t)(c.width / 2) * (c.height / 2);
        p.y.resize(cy);
        p.u.resize(cc);
        p.v.resize(cc);
        read_at(rvsb_config_texture_path(cfg_, view), "color", (long)(cy * 2 * 3 / 2), frame,
                {p.y.data(), p.u.data(), p.v.data()}, {cy, cc, cc});
        // Depth frames have the padded size (image_loading.cpp:149); with a
        // Crop_region the view's depth is the first region-area samples of
        // that frame's luma (SynthesizedView.cpp:89-94).
        int32_t region[4], padded[2];
        size_t py = cy;
        if (rvsb_config_input_crop(cfg_, view, region, padded) == RVSB_OK) py = (size_t)padded[0] * padded[1];
        const long depth_frame = c.depth_color_format == RVSB_FMT_YUV420 ? (long)(py * 2 * 3 / 2) : (long)(py * 2);
        p.depth.resize(py);
        read_at(rvsb_config_depth_path(cfg_, view), "depth", depth_frame, frame, {p.depth.data()}, {py});
        p.depth.resize(cy);
        return p;
    }

    bool wantColor() override { return files_[RVSB_OUT_COLOR] != nullptr; }
    bool wantMaskedColor() override { return files_[RVSB_OUT_MASKED_COLOR] != nullptr; }
    bool wantMask() override { return files_[RVSB_OUT_MASK] != nullptr; }
    bool wantDepth() override { return files_[RVSB_OUT_DEPTH] != nullptr; }
    bool wantMaskedDepth() override { return files_[RVSB_OUT_MASKED_DEPTH] != nullptr; }

    void saveColor(const uint16_t* yuv, int frame, int, const rvsb_camera&) override {
        nvtxRangePushA("rvsb cli: save colour");
        append(files_[RVSB_OUT_COLOR], frame == 0, yuv, (ny_ + 2 * nc_) * 2);
        nvtxRangePop();
    }
    void saveMaskedColor(const uint16_t* yuv, int frame, int, const rvsb_camera&) override {
        append(files_[RVSB_OUT_MASKED_COLOR], frame == 0, yuv, (ny_ + 2 * nc_) * 2);
    }
    void saveMask(const uint8_t* mask, int frame, int, const rvsb_camera&) override {
        std::vector<uint8_t> m(py_ + 2 * pc_, 128);
        std::fill(m.begin(), m.begin() + py_, 0);
        pad(m.data(), mask);
        append(files_[RVSB_OUT_MASK], frame == 0, m.data(), m.size());
    }
    void saveDepth(const uint16_t* depth, int frame, int, const rvsb_camera&) override {
        write_depth(files_[RVSB_OUT_DEPTH], frame, depth);
    }
    void saveMaskedDepth(const uint16_t* depth, int frame, int, const rvsb_camera&) override {
        write_depth(files_[RVSB_OUT_MASKED_DEPTH], frame, depth);
    }

    rvsb_synth_params synthesisParameters(int view) override {
        rvsb_synth_params p = rvsb::Pipeline::synthesisParameters(view);
        p.chroma_rounding = chroma_rounding_;
        return p;
    }

private:
    // The luma plane of a depth or mask output.  Without Crop_region it is
    // the output itself.  With one, the reference pads with
    // `padded(region) = image` (image_writing.cpp:262-267, 285-290): an
    // OpenCV header assignment to a temporary region, which copies no data,
    // so its file holds an all-zero luma plane of the padded size.  That is
    // reproduced here.
    template <class T>
    void pad(T* dst, const T* src) const {
        if (crop_[0] != 0 || crop_[1] != 0 || crop_[2] != padded_[0] || crop_[3] != padded_[1]) return;
        std::memcpy(dst, src, (size_t)crop_[2] * crop_[3] * sizeof(T));
    }
    void write_depth(const char* path, int frame, const uint16_t* depth) const {
        std::vector<uint16_t> img(depth_chroma_ ? py_ + 2 * pc_ : py_, neutral_);
        std::fill(img.begin(), img.begin() + py_, 0);
        pad(img.data(), depth);
        append(path, frame == 0, img.data(), img.size() * 2);
    }

    rvsb_config* cfg_;
    int chroma_rounding_;
    const char* files_[5];
    int32_t crop_[4] = {0, 0, 0, 0}, padded_[2] = {0, 0};
    uint16_t neutral_ = 0;
    bool depth_chroma_ = true;
    size_t ny_ = 0, nc_ = 0, py_ = 0, pc_ = 0;
};

}  // namespace

int main(int argc, char** argv) {
    std::string config_path;
    int chroma_rounding = RVSB_CHROMA_TIES_EVEN;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--help")) {
            config_path.clear();
            break;
        }
        if (!std::strcmp(argv[i], "--cuda") || !std::strcmp(argv[i], "--b200")) continue;
        // Output chroma rounding of an OpenCV built without IPP (ties up).
        if (!std::strcmp(argv[i], "--chroma-ties-up")) {
            chroma_rounding = RVSB_CHROMA_TIES_UP;
            continue;
        }
        if (!std::strcmp(argv[i], "--opengl") || !std::strcmp(argv[i], "--analyzer")) {
            std::fprintf(stderr, "%s is not supported by this backend\n", argv[i]);
            return 1;
        }
        if (config_path.empty())
            config_path = argv[i];
        else {
            std::fprintf(stderr, "Too many parameters (try --help)\n");
            return 1;
        }
    }
    if (config_path.empty()) {
        std::fprintf(stderr, "Usage: rvsb CONFIGURATION_FILE [--cuda] [--chroma-ties-up]\n");
        return 1;
    }
    char err[1024] = {0};
    rvsb_config* cfg = nullptr;
    if (rvsb_config_load(config_path.c_str(), &cfg, err, sizeof(err)) != RVSB_OK) {
        std::fprintf(stderr, "%s\n", err);
        return 1;
    }
    int rc = 0;
    const auto t0 = std::chrono::steady_clock::now();
    int n_out = 0;
    try {
        Application app(cfg, chroma_rounding);
        n_out = app.execute();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        rc = 1;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc == 0)
        std::printf("Total time: %.3f sec.\nAv. speed: %.3f fps.\nAv. time per frame: %.3f sec.\n", secs,
                    n_out / secs, secs / n_out);
    rvsb_config_free(cfg);
    return rc;
}
