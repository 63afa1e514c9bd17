// rvsb: command-line drop-in for the reference's `RVS <config.json>`
// (rvs/src/view_synthesis.cpp:64-176) on the B200 backend, written against
// the C ABI only.
//
// Frame loop of Pipeline::execute / computeView (rvs/src/Pipeline.cpp:76-94,
// 157-298): output frame f uses input frame start_frame + f, mapped into the
// input files with the ping-pong rule of getExtendedIndex, the pose trace
// entry of that input frame, and appends its YUV420 planes to each output
// file (truncating on frame 0, image_writing.cpp:72-76).
#include <chrono>
#include <cstdio>
#include <cstring>
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

    rvsb_context* ctx = nullptr;
    if (rvsb_create(0, 0, &ctx) != RVSB_OK) {
        std::fprintf(stderr, "failed to create a CUDA context on device 0\n");
        return 1;
    }
    std::vector<std::vector<uint16_t>> bufs(n_in * 4);
    std::vector<rvsb_view_planes> planes(n_in);
    const auto t0 = std::chrono::steady_clock::now();
    int rc = 0;
    for (int vf = 0; vf < n_out && rc == 0; ++vf) {
        const int input_frame = start + vf;
        const int frame = extended_index(input_frame, n_frames);
        for (int i = 0; i < n_in && rc == 0; ++i) {
            const rvsb_camera& c = cams[i];
            const size_t ny = (size_t)c.width * c.height, nc = (size_t)(c.width / 2) * (c.height / 2);
            bufs[i * 4 + 0].resize(ny);
            bufs[i * 4 + 1].resize(nc);
            bufs[i * 4 + 2].resize(nc);
            bufs[i * 4 + 3].resize(ny);
            std::string e;
            const long color_frame = (long)(ny * 2 * 3 / 2);
            if (!read_at(rvsb_config_texture_path(cfg, i), color_frame, frame,
                         {bufs[i * 4].data(), bufs[i * 4 + 1].data(), bufs[i * 4 + 2].data()}, {ny, nc, nc}, e)) {
                std::fprintf(stderr, "%s\n", e.c_str());
                rc = 1;
                break;
            }
            const long depth_frame = c.depth_color_format == RVSB_FMT_YUV420 ? (long)(ny * 2 * 3 / 2) : (long)(ny * 2);
            if (!read_at(rvsb_config_depth_path(cfg, i), depth_frame, frame, {bufs[i * 4 + 3].data()}, {ny}, e)) {
                std::fprintf(stderr, "%s\n", e.c_str());
                rc = 1;
                break;
            }
            planes[i].y = bufs[i * 4].data();
            planes[i].u = bufs[i * 4 + 1].data();
            planes[i].v = bufs[i * 4 + 2].data();
            planes[i].depth = bufs[i * 4 + 3].data();
        }
        if (rc) break;
        rvsb_camera virt;
        if (rvsb_config_virtual_camera_at(cfg, 0, input_frame, &virt) != RVSB_OK) {
            std::fprintf(stderr, "pose trace has no entry for frame %d\n", input_frame);
            rc = 1;
            break;
        }
        const size_t ny = (size_t)virt.width * virt.height, nc = (size_t)(virt.width / 2) * (virt.height / 2);
        std::vector<uint16_t> oy(ny), ou(nc), ov(nc);
        rvsb_yuv420 out{oy.data(), ou.data(), ov.data()};
        st = rvsb_synthesize_host(ctx, cams.data(), n_in, planes.data(), &virt, &params, &out, nullptr);
        if (st != RVSB_OK) {
            std::fprintf(stderr, "synthesis failed: %s (%s)\n", rvsb_status_string(st), rvsb_last_error(ctx));
            rc = 1;
            break;
        }
        const char* out_path = rvsb_config_output_path(cfg, 0);
        if (out_path) {
            FILE* f = std::fopen(out_path, vf ? "ab" : "wb");
            if (!f) {
                std::fprintf(stderr, "Failed to open YUV output image\n");
                rc = 1;
                break;
            }
            std::fwrite(oy.data(), 2, ny, f);
            std::fwrite(ou.data(), 2, nc, f);
            std::fwrite(ov.data(), 2, nc, f);
            std::fclose(f);
        }
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc == 0)
        std::printf("Total time: %.3f sec.\nAv. speed: %.3f fps.\nAv. time per frame: %.3f sec.\n", secs,
                    n_out / secs, secs / n_out);
    rvsb_destroy(ctx);
    rvsb_config_free(cfg);
    return rc;
}
