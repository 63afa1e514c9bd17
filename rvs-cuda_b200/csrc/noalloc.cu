// rvsb_inpaint_sources_noalloc: the inpainting scans (compute_nearest,
// rvs/src/inpainting.cpp:104-136, as implemented by inpaint.cu) over a
// caller's hole mask, with every scratch buffer taken from one static device
// array instead of allocated memory.
//
// Who needs this: a caller that may not allocate device memory while it
// runs.  Two such callers are a frame loop whose whole device budget is
// reserved up front (there a new cudaMalloc can fail, or push a co-resident
// process out of its share), and a latency-bound loop sharing the device
// with other streams, which cannot afford cudaFree's implicit device-wide
// synchronisation.  The regular synthesis entry points size their workspace
// with cudaMalloc on first use of a shape, so neither caller can use them for
// this step.
//
// Limits and rules:
//  - The scratch holds images of at most kMaxPixels = 524,288 pixels (for
//    example 960x540 or 1024x512): 5 words of 8 bytes per pixel plus a
//    256-byte status block, 20 MiB + 256 bytes per device in all.  Larger
//    images are rejected with RVSB_E_ARG before any device work.
//  - Set-up: the first call on each device, with that device current, looks
//    the array up with cudaGetSymbolAddress (which loads this file's device
//    code on that device).  Make that first call before any stream capture
//    begins; later calls only launch kernels.
//  - Initial contents: nothing in the array needs to start at zero.  The
//    status block (hole count and hole bounding box) must start each call
//    empty, and the first kernel of every call writes it so; every scan word
//    a later kernel reads has been written earlier in the same call.
//  - All calls on one device share the one array: two calls whose kernels
//    overlap in time (different streams, or different host threads without
//    ordering) race on it and give wrong results.  Order such calls, for
//    example on one stream.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <mutex>

#include "../../include/rvsb.h"
#include "device_common.cuh"
#include "kernels.hpp"

namespace rvsb {
namespace {

constexpr size_t kMaxPixels = size_t(1) << 19;
constexpr size_t kStatusBytes = 256;
constexpr size_t kWordsPerPixel = 5;  // codes + 4 scan buffers
constexpr size_t kScratchBytes = kStatusBytes + kWordsPerPixel * sizeof(uint64_t) * kMaxPixels;
constexpr int kMaxDevices = 64;

static_assert(sizeof(DevStatus) <= kStatusBytes, "status block too small");

}  // namespace
}  // namespace rvsb

// The scratch array itself (device memory reserved when this file's device
// code is loaded on a device; no allocation call is involved).
static __device__ __align__(256) unsigned char g_noalloc_scratch[rvsb::kScratchBytes];

namespace rvsb {
namespace {

std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Address of the scratch array on the current device, looked up once per
// device.
cudaError_t scratch_on_current_device(unsigned char** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

// Writes the empty status: no holes, an inverted bounding box.
__global__ void noalloc_reset_kernel(DevStatus* st) {
    if (threadIdx.x == 0) {
        st->bin_total = 0;
        st->bin_overflow = 0;
        st->hole_x0 = INT_MAX;
        st->hole_y0 = INT_MAX;
        st->hole_x1 = INT_MIN;
        st->hole_y1 = INT_MIN;
        st->n_holes = 0;
        st->pad = 0;
    }
}

// Per pixel: the code word the fill copies (only the hole bit: no colour is
// carried), the source of a non-hole (itself; -1 marks a hole until the fill
// writes it) and the hole count and bounding box, one atomic per warp.
__global__ void noalloc_prep_kernel(const uint8_t* __restrict__ holes, int w, int h, DevStatus* st,
                                    uint64_t* __restrict__ codes, int32_t* __restrict__ sources) {
    const size_t n = (size_t)w * h;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const size_t o = base + threadIdx.x;
        int x0 = INT_MAX, y0 = INT_MAX, x1 = INT_MIN, y1 = INT_MIN;
        bool hole = false;
        if (o < n) {
            const int x = (int)(o % (size_t)w), y = (int)(o / (size_t)w);
            hole = holes[o] != 0;
            codes[o] = hole ? dev::kHoleBit : 0ull;
            sources[o * 2 + 0] = hole ? -1 : x;
            sources[o * 2 + 1] = hole ? -1 : y;
            if (hole) {
                x0 = x1 = x;
                y0 = y1 = y;
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, hole);
        if (mask) {
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, s));
                y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, s));
                x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, s));
                y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, s));
            }
            if ((threadIdx.x & 31) == 0) {
                atomicMin(&st->hole_x0, x0);
                atomicMin(&st->hole_y0, y0);
                atomicMax(&st->hole_x1, x1);
                atomicMax(&st->hole_y1, y1);
                atomicAdd(&st->n_holes, __popc(mask));
            }
        }
    }
}

template <typename... Args>
void set_error(char* err, size_t err_len, const char* fmt, Args... args) {
    if (err && err_len) std::snprintf(err, err_len, fmt, args...);
}

}  // namespace
}  // namespace rvsb

extern "C" rvsb_status rvsb_inpaint_sources_noalloc(const uint8_t* holes, int width, int height,
                                                    int32_t* sources, void* stream, char* err, size_t err_len) {
    using namespace rvsb;
    if (err && err_len) err[0] = '\0';
    if (!holes || !sources) {
        set_error(err, err_len, "%s", "null hole mask or source buffer");
        return RVSB_E_ARG;
    }
    // The fill pass works on 2x2 blocks (as the synthesis path's inpainting
    // does), so both sides must be even; the scan words hold 16-bit
    // coordinates, and 32768 is the synthesis path's largest side.
    if (width < 2 || height < 2 || (width & 1) || (height & 1) || width > 32768 || height > 32768) {
        set_error(err, err_len, "image size %d x %d is invalid (each side even, 2..32768)", width, height);
        return RVSB_E_ARG;
    }
    const long long npix = (long long)width * height;
    if ((size_t)npix > kMaxPixels) {
        set_error(err, err_len, "image of %d x %d pixels exceeds the no-allocation scratch limit of %lld pixels",
                  width, height, (long long)kMaxPixels);
        return RVSB_E_ARG;
    }
    unsigned char* base = nullptr;
    cudaError_t e = scratch_on_current_device(&base);
    if (e != cudaSuccess) {
        set_error(err, err_len, "scratch set-up failed: %s", cudaGetErrorString(e));
        return RVSB_E_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevStatus* st = reinterpret_cast<DevStatus*>(base);
    uint64_t* words = reinterpret_cast<uint64_t*>(base + kStatusBytes);
    uint64_t* codes = words;
    uint64_t* scan[4];
    for (int k = 0; k < 4; ++k) scan[k] = words + (size_t)(k + 1) * (size_t)npix;
    noalloc_reset_kernel<<<1, 32, 0, s>>>(st);
    int dev = 0, sms = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || sms <= 0) {
        set_error(err, err_len, "device query failed: %s", cudaGetErrorString(e));
        return RVSB_E_CUDA;
    }
    const int threads = 256;
    const int blocks = (int)std::min<long long>((npix + threads - 1) / threads, (long long)sms * 8);
    noalloc_prep_kernel<<<blocks, threads, 0, s>>>(holes, width, height, st, codes, sources);
    launch_inpaint_scans(st, holes, codes, scan, width, height, sources, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(err, err_len, "kernel launch failed: %s", cudaGetErrorString(e));
        return RVSB_E_CUDA;
    }
    return RVSB_OK;
}
