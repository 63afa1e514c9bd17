// rvsb: command-line drop-in for the reference's `RVS <config.json>`
// (rvs/src/view_synthesis.cpp:64-176) on the B200 backend, written against
// the C ABI only.
//
// Frame loop of Pipeline::execute / computeView (rvs/src/Pipeline.cpp:76-94,
// 157-298): output frame f uses input frame start_frame + f, mapped into the
// input files with the ping-pong rule of getExtendedIndex, the pose trace
// entry of that input frame, and appends its YUV420 planes to each output
// file (truncating on frame 0, image_writing.cpp:72-76).  Like the
// reference's asynchronous loader and writer (Pipeline.cpp:226-245), the
// next frame's input files are read while the current frame is synthesised
// and the previous frame's outputs are written meanwhile.  Besides
// OutputFiles, the CPU-mode outputs MaskedOutputFiles, OutputMasks,
// DepthOutputFiles and MaskedDepthOutputFiles are written when configured
// (Pipeline.cpp:303-336).  A virtual camera's Crop_region gives colour
// outputs of the region's size and depth and mask outputs placed into a zero
// image of the padded resolution (image_writing.cpp:262-267, 285-290).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <string>
#include <vector>

#include "rvsb.h"

namespace {

int extended_index(int output_frame, int n_input_frames) {
    const int group = output_frame / n_input_frames;
    const int rel = output_frame % n_input_frames;
    return group % 2 != 0 ? n_input_frames - rel - 1 : rel;
}

bool read_at(const char* path, long offset_per_frame, int frame, std::vector<uint16_t*> dst,
             std::vector<size_t> counts, std::string& err) {
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        err = std::string("Failed to read raw YUV file \"") + path + "\"";
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    long off = offset_per_frame * frame;
    if (off >= size) off = 0;  // image_loading.cpp:95-98
    std::fseek(f, off, SEEK_SET);
    for (size_t k = 0; k < dst.size(); ++k) {
        if (std::fread(dst[k], 2, counts[k], f) != counts[k]) {
            std::fclose(f);
            err = std::string("Failed to read the expected amount of data from \"") + path + "\"";
            return false;
        }
    }
    std::fclose(f);
    return true;
}

// Host planes of one input frame (all views).
struct InputFrame {
    std::vector<std::vector<uint16_t>> bufs;  // 4 per view: y, u, v, depth
};

// Host copies of one frame's outputs and the files they go to.
struct OutputFrame {
    std::vector<uint16_t> yuv, masked, depth, masked_depth;
    std::vector<uint8_t> mask;
};

bool append(const char* path, bool first, const void* data, size_t bytes, std::string& err) {
    FILE* f = std::fopen(path, first ? "wb" : "ab");
    if (!f) {
        err = "Failed to open YUV output image";
        return false;
    }
    const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
    std::fclose(f);
    if (!ok) err = std::string("Failed to write \"") + path + "\"";
    return ok;
}

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
    rvsb_status st = rvsb_config_load(config_path.c_str(), &cfg, err, sizeof(err));
    if (st != RVSB_OK) {
        std::fprintf(stderr, "%s\n", err);
        return 1;
    }
    const int n_in = rvsb_config_num_inputs(cfg);
    if (rvsb_config_num_virtual(cfg) != 1) {
        std::fprintf(stderr, "exactly one virtual camera is supported\n");
        return 1;
    }
    int start = 0, n_frames = 1, n_out = 1;
    rvsb_config_frames(cfg, &start, &n_frames, &n_out);
    rvsb_synth_params params;
    rvsb_config_synth_params(cfg, &params);
    params.chroma_rounding = chroma_rounding;
    std::vector<rvsb_camera> cams(n_in);
    for (int i = 0; i < n_in; ++i) rvsb_config_input_camera(cfg, i, &cams[i]);
    const char* files[5];
    for (int k = 0; k < 5; ++k) files[k] = rvsb_config_output_file(cfg, k, 0);

    rvsb_context* ctx = nullptr;
    if (rvsb_create(0, 0, &ctx) != RVSB_OK) {
        std::fprintf(stderr, "failed to create a CUDA context on device 0\n");
        return 1;
    }
    rvsb_scene* scene = nullptr;
    if ((st = rvsb_scene_create(ctx, cams.data(), n_in, &scene)) != RVSB_OK) {
        std::fprintf(stderr, "%s\n", rvsb_last_error(ctx));
        return 1;
    }
    rvsb_camera virt0;
    rvsb_config_virtual_camera(cfg, 0, &virt0);
    const size_t ny = (size_t)virt0.width * virt0.height, nc = (size_t)(virt0.width / 2) * (virt0.height / 2);
    // Device outputs.
    uint16_t *d_yuv = nullptr, *d_masked = nullptr, *d_depth = nullptr, *d_mdepth = nullptr;
    uint8_t* d_mask = nullptr;
    cudaMalloc(&d_yuv, (ny + 2 * nc) * 2);
    if (files[RVSB_OUT_MASKED_COLOR]) cudaMalloc(&d_masked, (ny + 2 * nc) * 2);
    if (files[RVSB_OUT_MASK]) cudaMalloc(&d_mask, ny);
    if (files[RVSB_OUT_DEPTH]) cudaMalloc(&d_depth, ny * 2);
    if (files[RVSB_OUT_MASKED_DEPTH]) cudaMalloc(&d_mdepth, ny * 2);
    rvsb_yuv420 out{d_yuv, d_yuv + ny, d_yuv + ny + nc};
    rvsb_aux_out aux{};
    aux.mask = d_mask;
    if (d_masked) aux.masked = rvsb_yuv420{d_masked, d_masked + ny, d_masked + ny + nc};
    aux.depth = d_depth;
    aux.masked_depth = d_mdepth;
    aux.validity_threshold = rvsb_config_validity_threshold(cfg);

    auto load = [&](int vf, InputFrame& fr, std::string& e) -> bool {
        const int frame = extended_index(start + vf, n_frames);
        fr.bufs.resize(n_in * 4);
        for (int i = 0; i < n_in; ++i) {
            const rvsb_camera& c = cams[i];
            const size_t cy = (size_t)c.width * c.height, cc = (size_t)(c.width / 2) * (c.height / 2);
            fr.bufs[i * 4 + 0].resize(cy);
            fr.bufs[i * 4 + 1].resize(cc);
            fr.bufs[i * 4 + 2].resize(cc);
            fr.bufs[i * 4 + 3].resize(cy);
            const long color_frame = (long)(cy * 2 * 3 / 2);
            if (!read_at(rvsb_config_texture_path(cfg, i), color_frame, frame,
                         {fr.bufs[i * 4].data(), fr.bufs[i * 4 + 1].data(), fr.bufs[i * 4 + 2].data()}, {cy, cc, cc},
                         e))
                return false;
            const long depth_frame = c.depth_color_format == RVSB_FMT_YUV420 ? (long)(cy * 2 * 3 / 2) : (long)(cy * 2);
            if (!read_at(rvsb_config_depth_path(cfg, i), depth_frame, frame, {fr.bufs[i * 4 + 3].data()}, {cy}, e))
                return false;
        }
        return true;
    };
    // Depth and mask files carry constant chroma planes
    // (write_depth_YUV / write_mask_YUV, image_writing.cpp:104-139) and the
    // padded resolution of a cropped camera.
    const uint16_t neutral = (uint16_t)std::lround(0.5 * (1.0 + (double)((1u << virt0.bit_depth_depth) - 1u)));
    const bool depth_chroma = virt0.depth_color_format == RVSB_FMT_YUV420;
    int32_t crop[4] = {0, 0, virt0.width, virt0.height}, padded[2] = {virt0.width, virt0.height};
    rvsb_config_virtual_crop(cfg, 0, crop, padded);
    const size_t py = (size_t)padded[0] * padded[1], pc = (size_t)(padded[0] / 2) * (padded[1] / 2);
    // The region's rows placed into a zero luma plane of the padded size.
    auto pad = [&](auto* dst, const auto* src) {
        for (int r = 0; r < crop[3]; ++r)
            std::memcpy(dst + (size_t)(crop[1] + r) * padded[0] + crop[0], src + (size_t)r * crop[2],
                        (size_t)crop[2] * sizeof(*src));
    };
    auto write = [&](int vf, const OutputFrame& o, std::string& e) -> bool {
        const bool first = vf == 0;
        if (files[RVSB_OUT_COLOR] && !append(files[RVSB_OUT_COLOR], first, o.yuv.data(), o.yuv.size() * 2, e))
            return false;
        if (files[RVSB_OUT_MASKED_COLOR] &&
            !append(files[RVSB_OUT_MASKED_COLOR], first, o.masked.data(), o.masked.size() * 2, e))
            return false;
        if (files[RVSB_OUT_MASK]) {
            std::vector<uint8_t> m(py + 2 * pc, 128);
            std::fill(m.begin(), m.begin() + py, 0);
            pad(m.data(), o.mask.data());
            if (!append(files[RVSB_OUT_MASK], first, m.data(), m.size(), e)) return false;
        }
        for (int k : {RVSB_OUT_DEPTH, RVSB_OUT_MASKED_DEPTH}) {
            if (!files[k]) continue;
            const std::vector<uint16_t>& d = k == RVSB_OUT_DEPTH ? o.depth : o.masked_depth;
            std::vector<uint16_t> img(depth_chroma ? py + 2 * pc : py, neutral);
            std::fill(img.begin(), img.begin() + py, 0);
            pad(img.data(), d.data());
            if (!append(files[k], first, img.data(), img.size() * 2, e)) return false;
        }
        return true;
    };

    InputFrame in[2];
    OutputFrame outs[2];
    std::string load_err, write_err;
    std::future<bool> loading = std::async(std::launch::async, [&] { return load(0, in[0], load_err); });
    std::future<bool> writing;
    const auto t0 = std::chrono::steady_clock::now();
    int rc = 0;
    for (int vf = 0; vf < n_out && rc == 0; ++vf) {
        if (!loading.get()) {
            std::fprintf(stderr, "%s\n", load_err.c_str());
            rc = 1;
            break;
        }
        InputFrame& cur = in[vf % 2];
        if (vf + 1 < n_out)
            loading = std::async(std::launch::async, [&, vf] { return load(vf + 1, in[(vf + 1) % 2], load_err); });
        for (int i = 0; i < n_in && rc == 0; ++i) {
            rvsb_view_planes p{cur.bufs[i * 4].data(), cur.bufs[i * 4 + 1].data(), cur.bufs[i * 4 + 2].data(),
                               cur.bufs[i * 4 + 3].data()};
            if ((st = rvsb_scene_upload(scene, i, &p, 0, nullptr)) != RVSB_OK) {
                std::fprintf(stderr, "upload failed: %s\n", rvsb_last_error(ctx));
                rc = 1;
            }
        }
        if (rc) break;
        rvsb_camera virt;
        if (rvsb_config_virtual_camera_at(cfg, 0, start + vf, &virt) != RVSB_OK) {
            std::fprintf(stderr, "pose trace has no entry for frame %d\n", start + vf);
            rc = 1;
            break;
        }
        st = rvsb_synthesize_aux(scene, &virt, &params, &out, &aux, nullptr);
        if (st != RVSB_OK) {
            std::fprintf(stderr, "synthesis failed: %s (%s)\n", rvsb_status_string(st), rvsb_last_error(ctx));
            rc = 1;
            break;
        }
        // The previous frame's write must finish before its buffers are reused.
        if (writing.valid() && !writing.get()) {
            std::fprintf(stderr, "%s\n", write_err.c_str());
            rc = 1;
            break;
        }
        OutputFrame& o = outs[vf % 2];
        o.yuv.resize(ny + 2 * nc);
        cudaMemcpy(o.yuv.data(), d_yuv, o.yuv.size() * 2, cudaMemcpyDeviceToHost);
        if (d_masked) {
            o.masked.resize(ny + 2 * nc);
            cudaMemcpy(o.masked.data(), d_masked, o.masked.size() * 2, cudaMemcpyDeviceToHost);
        }
        if (d_mask) {
            o.mask.resize(ny);
            cudaMemcpy(o.mask.data(), d_mask, ny, cudaMemcpyDeviceToHost);
        }
        if (d_depth) {
            o.depth.resize(ny);
            cudaMemcpy(o.depth.data(), d_depth, ny * 2, cudaMemcpyDeviceToHost);
        }
        if (d_mdepth) {
            o.masked_depth.resize(ny);
            cudaMemcpy(o.masked_depth.data(), d_mdepth, ny * 2, cudaMemcpyDeviceToHost);
        }
        if (cudaGetLastError() != cudaSuccess) {
            std::fprintf(stderr, "copying the outputs failed\n");
            rc = 1;
            break;
        }
        writing = std::async(std::launch::async, [&, vf] { return write(vf, outs[vf % 2], write_err); });
    }
    if (loading.valid()) loading.wait();
    if (writing.valid() && !writing.get() && rc == 0) {
        std::fprintf(stderr, "%s\n", write_err.c_str());
        rc = 1;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc == 0)
        std::printf("Total time: %.3f sec.\nAv. speed: %.3f fps.\nAv. time per frame: %.3f sec.\n", secs,
                    n_out / secs, secs / n_out);
    cudaFree(d_yuv);
    cudaFree(d_masked);
    cudaFree(d_mask);
    cudaFree(d_depth);
    cudaFree(d_mdepth);
    rvsb_scene_destroy(scene);
    rvsb_destroy(ctx);
    rvsb_config_free(cfg);
    return rc;
}
