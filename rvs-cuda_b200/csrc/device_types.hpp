// Parameter blocks shared by the host launch code and the kernels.
#pragma once

#include <cstdint>

namespace rvsb {

// Tiling constants.  A binning block is BLOCK_W x BLOCK_H quads of an input
// view (each quad = two triangles, transform.cpp:159-176); an output tile
// (its size is chosen per batch among the raster variants) holds 64-bit
// z-buffers in shared memory and is processed by one CTA of the variant's
// thread count (TILE_THREADS unless the variant names another).
constexpr int BLOCK_W = 8;
constexpr int BLOCK_H = 4;
// Vertex tile of the warp kernel (WARP_TILE x WARP_TILE input pixels per CTA),
// also the unit of the ERP input culling tables.
constexpr int WARP_TILE = 32;
constexpr int TILE_THREADS = 512;
// Smallest tile of any raster variant (sizes the bin arrays).
constexpr int MIN_TILE_W = 32;
constexpr int MIN_TILE_H = 32;

// Per input view parameters of one synthesis (device copy in a table).
struct DevView {
    int w, h;          // input size
    int proj;          // 0 perspective, 1 equirectangular
    int bits_color;
    float f0, f1, p0, p1;                 // perspective intrinsics
    float near_, far_, depth_scale;       // depth decode (process_input_frame.cu:369-376)
    int has_invalid;
    float color_scale;                    // 1 / (2^bits - 1)
    float chroma_sx, chroma_sy;           // (w/2)/w, (h/2)/h as float
    int cw, ch;                           // chroma plane size
    float R[9], t[3];                     // relative pose (SpaceTransformer.cpp:77-92)
    const uint16_t* py;
    const uint16_t* pu;
    const uint16_t* pv;
    const uint16_t* pd;
    const float4* depth_lut;              // 65536 (d, -d/f0, -d/f1, 0), indexed by the raw sample
    const float* erp_row;                 // ERP: per row (cos theta, sin theta), 2*h floats
    const float* erp_col;                 // ERP: per column (cos phi, sin phi), 2*w floats
    // ERP inputs, per WARP_TILE x WARP_TILE vertex tile grown by one pixel:
    // the unit direction of its centre and an angle bounding every vertex
    // direction from it (x, y, z, radius), and the range of its decoded
    // depths (min, max); used to skip tiles no output pixel can come from.
    const float4* erp_cone;
    const float2* tile_depth;
    const uint64_t* color;                // h*w decoded colour: Y | 4U << 18 | 4V << 36
    float4* vert;                         // h*w warped vertices (u, v, z, 0)
    int4* bbox;                           // per binning block: x0, y0, x1, y1 (x0 > x1: empty)
    int nbx, nby;                         // binning blocks
    int tri_shift;                        // triangle index = i << tri_shift | j << 2 | t
    int pad;
};

// Virtual camera of one synthesis.
struct DevTarget {
    int wo, ho;
    int proj;
    int wrap;                             // horizontal wrap (ERP output, full range)
    // Perspective output: the planes u = -1, u = W + 1, v = -1, v = H + 1 in
    // the virtual camera's frame (a . y > 0 beyond each, for y0 > 0); cull
    // enables skipping ERP input tiles wholly beyond one of them.
    int cull;
    float cull_plane[4][3];
    float f0, f1, p0, p1;                 // perspective
    float u0, v0, du_dphi, dv_dtheta;     // equirectangular
    int bits;                             // output bit depth
    unsigned max_val;                     // 2^bits - 1
    float blend_exp;                      // BlendingFactor
    float inv_blend_exp;                  // 1.0f / BlendingFactor
    int blend_exp_int;                    // BlendingFactor when it is an integer in [2, 16], else 0
    int chroma_ties_up;                   // output chroma mean: 1 rounds ties up, 0 to even
    int blend_max;                        // BlendingFactor < 0: blend by maximum quality
    // Precision P != 1 (SynthesizedView.cpp:325-333): wo x ho is the raster
    // size int(0.5 + W * P) x int(0.5 + H * P); the output W x H is resized
    // from it (image_writing.cpp:188-190).
    int rescale;
    int out_w, out_h;
    float uv_sx, uv_sy;                   // raster size / output size (float)
    float precision;
    int rs_area;                          // the resize is an exact 2x reduction (area mean)
    double rs_scale_x, rs_scale_y;        // raster size / output size (double), bilinear
    int tile_wl, tile_hl;                 // log2 of the tile width and height
    int ntx, nty;                         // output tiles
    int n_views;
    int bin_capacity;
};

// Largest number of input views of one synthesis.
constexpr int MAX_VIEWS = 16;

// Status words written by the kernels (device memory, reset per call).
struct DevStatus {
    int bin_total;      // number of (tile, view, block) entries
    int bin_overflow;   // 1 when bin_total exceeded the list capacity
    int hole_x0, hole_y0, hole_x1, hole_y1;   // bounding box of holes (x0 > x1: none)
    int n_holes;
    int pad;
};

// Optional intermediate outputs (device pointers, may be null).
struct DebugPtrs {
    float* warped_uvz = nullptr;
    float* view_color = nullptr;
    float* view_depth = nullptr;
    float* view_validity = nullptr;
    float* blend_color = nullptr;
    float* blend_quality = nullptr;
    int32_t* inpaint_source = nullptr;
    bool any() const {
        return warped_uvz || view_color || view_depth || view_validity || blend_color ||
               blend_quality || inpaint_source;
    }
};

// Auxiliary outputs of a synthesis (Pipeline.cpp:303-336, CPU mode): any
// pointer may be null.  acc_depth / acc_valid are the slot's per-pixel
// blended depth and validity (workspace buffers, set when any output is on).
struct AuxPtrs {
    uint8_t* mask;            // 255 where the blended validity is not above threshold
    uint16_t* masked_y;       // YUV420 colour with masked pixels set to 0.5
    uint16_t* masked_u;
    uint16_t* masked_v;
    uint16_t* depth;          // encoded blended depth
    uint16_t* masked_depth;   // the same, 0 where masked
    float* acc_depth;
    float* acc_valid;
    float threshold;          // "ValidityThreshold"
    int on;                   // any output requested
    float depth_near, depth_far;  // virtual camera's depth range
    unsigned depth_max;       // 2^BitDepthDepth - 1
    int pad;
};

// Multispectral blending (BlendedViewMultiSpec, BlendedView.cpp:63-88): the
// raster stores every view's resolved colour and quality, the blur kernels
// the masked box mean of each view's luma, and the blend kernel the two
// frequency bands' blends.  Per view, npix = Wo*Ho entries each.
struct MsPtrs {
    float4* view;       // (Y, U, V, quality) per view and pixel
    double* hsum;       // row-window sums of masked luma
    int* hcnt;          // row-window counts of masked pixels
    float* blur;        // blurred luma (0 outside the mask)
    int on;
    int rad;            // window radius: max(Wo, Ho) / 20
    float low_exp, high_exp;
    int low_int, high_int;  // integer exponents in [2, 16] (0 otherwise)
};

// Device buffers of one slot's workspace.
struct SlotBuffers {
    DevStatus* status;   // 1 entry
    int* counts;         // ntiles * n_views
    int* offsets;        // ntiles * n_views
    int* cursor;         // ntiles * n_views
    int* list;           // bin list, `capacity` entries
    int capacity;
    int pad;
    uint64_t* codes;     // Wo*Ho packed output codes + hole bit
    uint8_t* holes;      // Wo*Ho hole mask (1 = no view covers the pixel)
    uint64_t* scan[4];   // Wo*Ho inpainting scratch each
    uint64_t* inpaint_seg;  // column-group and warp-segment minima of the inpainting pre-passes
    int* tile_order;        // output tiles, most bin entries first (raster launch order)
    float4* pcolor;      // Precision != 1: blended colour per raster pixel
    int32_t* psrc;       // Precision != 1: inpainting source of every hole
};

// Most row groups per column strip in the inpainting passes.
constexpr int INPAINT_MAX_GROUPS = 8;

// Everything one synthesis (one virtual view) needs on the device.  A batch
// keeps one table per slot in device memory; every kernel of the batch reads
// the table of its slot (a grid dimension), so the launch sequence of a
// batch is fixed and the per-call data travels in one copy of the tables.
struct SlotTable {
    DevTarget t;
    SlotBuffers b;
    uint16_t* out_y;
    uint16_t* out_u;
    uint16_t* out_v;
    DebugPtrs dbg;
    AuxPtrs aux;
    MsPtrs ms;
    DevView v[MAX_VIEWS];
};

}  // namespace rvsb
