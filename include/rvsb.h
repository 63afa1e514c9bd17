/*
 * rvsb.h - C ABI of the B200 backend for the RVS per-frame view-synthesis path.
 *
 * The reference (RVS, the MPEG Reference View Synthesizer, with its CUDA fork)
 * synthesises one virtual view per frame in Pipeline::computeView
 * (rvs/src/Pipeline.cpp:169-345).  For each input view it calls
 * SynthesizedView::compute (rvs/src/SynthesizedView.cpp:374-380: unproject,
 * R*x+t, project, triangle raster), then BlendedView::blend
 * (rvs/src/BlendedView.cpp:256-262), and after the last view the inpainter
 * (rvs/src/inpainting.cpp:213-235) and the YUV420 writer
 * (rvs/src/image_writing.cpp:182-225).  The CUDA fork exposes the same steps
 * as C++ free functions with OpenCV types (the .cuh headers under rvs_cuda_lib/src).
 *
 * This header replaces both layers with plain C: cameras are plain structs,
 * images are raw plane pointers plus the sizes in the camera struct, streams
 * are passed as void* (a cudaStream_t), and errors are status codes instead
 * of exceptions.  Each entry point names the reference interface it replaces.
 *
 * Threading: a context may be used from one host thread at a time; scenes
 * and servers created from it share its device.  All device work is issued on
 * the stream passed in (NULL = the legacy default stream).
 */
#ifndef RVSB_H
#define RVSB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RVSB_ABI_VERSION 1

/* Status codes.  The reference throws std::runtime_error / std::logic_error
 * (e.g. rvs_cuda_lib/src/transform_triangle.cu:376-379,
 * rvs/src/Parameters.cpp:330-339) and its call sites print and continue
 * (rvs/src/SynthesizedView.cpp:461-464); here every failure is returned. */
typedef enum rvsb_status {
    RVSB_OK = 0,
    RVSB_E_ARG = 1,          /* null pointer, size or index out of range */
    RVSB_E_CONFIG = 2,       /* JSON / camera parameters rejected */
    RVSB_E_IO = 3,           /* file missing or shorter than one frame */
    RVSB_E_OOM_BUDGET = 4,   /* request does not fit the HBM budget */
    RVSB_E_CUDA = 5,         /* CUDA runtime error */
    RVSB_E_TIMEOUT = 6,      /* a bounded wait expired */
    RVSB_E_UNSUPPORTED = 7,  /* a reference option this build does not take */
    RVSB_E_BUSY = 8,         /* queue full */
    RVSB_E_NOT_FOUND = 9     /* unknown ticket / camera name */
} rvsb_status;

typedef enum rvsb_projection {
    RVSB_PROJ_PERSPECTIVE = 0,      /* "Perspective" */
    RVSB_PROJ_EQUIRECTANGULAR = 1   /* "Equirectangular" */
} rvsb_projection;

typedef enum rvsb_color_format {
    RVSB_FMT_YUV420 = 0,            /* "YUV420" */
    RVSB_FMT_YUV400 = 1             /* "YUV400" (depth only) */
} rvsb_color_format;

/* One camera of an RVS camera-parameter file.  Field meanings follow
 * Parameters::readFrom (rvs/src/Parameters.cpp:104-129) and the setters at
 * rvs/src/Parameters.cpp:316-463.  width, height and principle_point are
 * the values after a virtual camera's Crop_region
 * (rvsb_config_virtual_crop). */
typedef struct rvsb_camera {
    int32_t projection;          /* rvsb_projection ("Projection") */
    int32_t width;               /* "Resolution"[0] */
    int32_t height;              /* "Resolution"[1] */
    int32_t bit_depth_color;     /* "BitDepthColor" (1..16) */
    int32_t bit_depth_depth;     /* "BitDepthDepth" (1..16) */
    int32_t depth_color_format;  /* rvsb_color_format ("DepthColorSpace") */
    int32_t has_invalid_depth;   /* "HasInvalidDepth", default 1 */
    int32_t full_hor_range;      /* "Hor_range" equals [-180, 180] as integers */
    float position[3];           /* "Position" (x forward, y left, z up) */
    float rotation[3];           /* "Rotation": yaw, pitch, roll in degrees */
    float depth_range[2];        /* "Depth_range": near, far (far >= 1000 = infinity) */
    float focal[2];              /* "Focal" (perspective) */
    float principle_point[2];    /* "Principle_point" (perspective) */
    float hor_range[2];          /* "Hor_range" in degrees (equirectangular) */
    float ver_range[2];          /* "Ver_range" in degrees (equirectangular) */
} rvsb_camera;

/* Raw planes of one input view, as stored in the reference's .yuv files
 * (read_color_YUV / read_depth_YUV, rvs/src/image_loading.cpp:74-211):
 * samples are little-endian uint16 for bit depths 9..16.
 *   y:     width*height colour luma samples
 *   u, v:  (width/2)*(height/2) chroma samples each
 *   depth: width*height samples of the depth map's luma plane */
typedef struct rvsb_view_planes {
    const uint16_t* y;
    const uint16_t* u;
    const uint16_t* v;
    const uint16_t* depth;
} rvsb_view_planes;

/* YUV420 output planes (write_color, rvs/src/image_writing.cpp:182-225):
 * y: width*height, u and v: (width/2)*(height/2) uint16 samples each. */
typedef struct rvsb_yuv420 {
    uint16_t* y;
    uint16_t* u;
    uint16_t* v;
} rvsb_yuv420;

/* Rounding of the output chroma 2x2 mean.  write_color_YUV
 * (rvs/src/image_writing.cpp:83-84) halves U and V with OpenCV's
 * cv::resize(0.5, 0.5, INTER_LINEAR) on uint16 samples, whose ties depend on
 * how OpenCV was built: with Intel IPP (the default of a source build on
 * x86-64, and the opencv-python wheel) a 2x2 sum s gives round-half-even(s/4);
 * without IPP it gives (s + 2) >> 2. */
typedef enum rvsb_chroma_rounding {
    RVSB_CHROMA_TIES_EVEN = 0, /* OpenCV built with IPP (default) */
    RVSB_CHROMA_TIES_UP = 1    /* OpenCV built without IPP */
} rvsb_chroma_rounding;

/* "BlendingMethod" (Pipeline::createBlender, rvs/src/Pipeline.cpp:347-361). */
typedef enum rvsb_blending_method {
    RVSB_BLEND_SIMPLE = 0,        /* BlendedViewSimple: quality^BlendingFactor weights */
    RVSB_BLEND_MULTISPECTRAL = 1  /* BlendedViewMultiSpec: low and high frequencies
                                     blended with their own factors */
} rvsb_blending_method;

/* Synthesis options (Config, rvs/src/Config.hpp:157-205). */
typedef struct rvsb_synth_params {
    float blending_factor;    /* "BlendingFactor" (default 5); < 0 blends by maximum quality */
    float precision;          /* "Precision" P > 0 (Config.cpp:389-399): rasterise at
                                 int(0.5 + W*P) x int(0.5 + H*P), which must be even,
                                 and resize to W x H when written; 1 unless set */
    int32_t chroma_rounding;  /* rvsb_chroma_rounding; 0 unless set */
    int32_t blending_method;  /* rvsb_blending_method; 0 unless set */
    float low_freq_factor;    /* "BlendingLowFreqFactor" (Multispectral) */
    float high_freq_factor;   /* "BlendingHighFreqFactor" (Multispectral) */
    int32_t reserved[2];      /* must be 0 */
} rvsb_synth_params;

/* ----------------------------------------------------------------------- */
/* Context                                                                  */
/* ----------------------------------------------------------------------- */

typedef struct rvsb_context rvsb_context;

/* Creates a context on CUDA device `device`.  `hbm_budget_bytes` caps the
 * device memory the context's scenes and work buffers may hold (0 = 60 GB).
 * Replaces the per-call cudaMalloc/cudaFree of the reference wrappers
 * (e.g. rvs_cuda_lib/src/transform_triangle.cu:327-380) with arenas owned
 * by the context. */
rvsb_status rvsb_create(int device, size_t hbm_budget_bytes, rvsb_context** out);
void rvsb_destroy(rvsb_context* ctx);

/* Last error message of the context (never NULL). */
const char* rvsb_last_error(const rvsb_context* ctx);
const char* rvsb_status_string(rvsb_status status);

/* Bytes of device memory currently held by the context. */
size_t rvsb_memory_in_use(const rvsb_context* ctx);

/* ----------------------------------------------------------------------- */
/* Front end: RVS JSON, camera JSON, pose trace                             */
/* ----------------------------------------------------------------------- */

/* Parses one camera object of a camera-parameter file (JSON text of the
 * object itself).  Replaces Parameters::readFrom
 * (rvs/src/Parameters.cpp:104-129) including its validation
 * (Depth_range order and far <= 1000, Depthmap == 1, ColorSpace YUV420).
 * On failure returns RVSB_E_CONFIG and writes a message into err. */
rvsb_status rvsb_camera_from_json(const char* json_object_text, rvsb_camera* out,
                                  char* err, size_t err_len);

typedef struct rvsb_config rvsb_config;

/* Loads an RVS configuration file and the camera files it names.  Replaces
 * Config::loadFromFile (rvs/src/Config.cpp:72-120) with
 * loadCamerasParametersFromFile (rvs/src/Config.cpp:122-175), the
 * InputOverrides/VirtualOverrides rule (rvs/src/JsonParser.cpp:199-219) and
 * the pose trace (rvs/src/PoseTraces.cpp:54-109).  Relative paths are
 * resolved against the working directory, as the reference does. */
rvsb_status rvsb_config_load(const char* rvs_json_path, rvsb_config** out,
                             char* err, size_t err_len);
void rvsb_config_free(rvsb_config* cfg);

int rvsb_config_num_inputs(const rvsb_config* cfg);
int rvsb_config_num_virtual(const rvsb_config* cfg);
rvsb_status rvsb_config_input_camera(const rvsb_config* cfg, int i, rvsb_camera* out);
rvsb_status rvsb_config_virtual_camera(const rvsb_config* cfg, int i, rvsb_camera* out);
/* Texture and depth file paths of input i; output path of virtual view i. */
const char* rvsb_config_texture_path(const rvsb_config* cfg, int i);
const char* rvsb_config_depth_path(const rvsb_config* cfg, int i);
const char* rvsb_config_output_path(const rvsb_config* cfg, int i);
/* StartFrame, NumberOfFrames, NumberOfOutputFrames, BlendingFactor, Precision. */
void rvsb_config_frames(const rvsb_config* cfg, int* start_frame, int* number_of_frames,
                        int* number_of_output_frames);
void rvsb_config_synth_params(const rvsb_config* cfg, rvsb_synth_params* out);
/* Output file i of one kind (NULL when the configuration has none):
 * OutputFiles, MaskedOutputFiles, OutputMasks, DepthOutputFiles,
 * MaskedDepthOutputFiles (Config.cpp:88-98). */
typedef enum rvsb_output_kind {
    RVSB_OUT_COLOR = 0,
    RVSB_OUT_MASKED_COLOR = 1,
    RVSB_OUT_MASK = 2,
    RVSB_OUT_DEPTH = 3,
    RVSB_OUT_MASKED_DEPTH = 4
} rvsb_output_kind;
const char* rvsb_config_output_file(const rvsb_config* cfg, int kind, int i);
/* "ValidityThreshold" (default 5000, Config.hpp:157). */
float rvsb_config_validity_threshold(const rvsb_config* cfg);
/* Virtual camera i for output frame `frame` after applying the pose trace
 * the way Pipeline::computeView does (rvs/src/Pipeline.cpp:173-181:
 * position += trace position, rotation = trace rotation). */
rvsb_status rvsb_config_virtual_camera_at(const rvsb_config* cfg, int i, int frame, rvsb_camera* out);
/* "Crop_region" of virtual camera i (Parameters::setCropRegionFrom,
 * Parameters.cpp:424-434): region = x, y, width, height inside the padded
 * "Resolution" padded_size = width, height.  The camera returned by
 * rvsb_config_virtual_camera has the region's size and, for a perspective
 * camera, its principal point moved by (-x, -y) (Parameters.cpp:187-190,
 * 245-249).  Colour outputs have the region's size; depth and mask outputs
 * are placed into a zero image of the padded size (write_maskedDepth /
 * write_mask, image_writing.cpp:262-267, 285-290).  Without the key the
 * region is the whole resolution. */
rvsb_status rvsb_config_virtual_crop(const rvsb_config* cfg, int i, int32_t region[4], int32_t padded_size[2]);
/* "Crop_region" of input camera i, as rvsb_config_virtual_crop.  The camera
 * returned by rvsb_config_input_camera has the region's size (and moved
 * principal point).  The reference reads such a view's colour frames at the
 * region's size (image_loading.cpp:76) and its depth frames at the padded
 * size (image_loading.cpp:149), decodes the padded depth and then takes its
 * first width x height samples in memory order as the region-sized depth
 * map (SynthesizedView.cpp:89-94).  The depth plane to pass for the view is
 * therefore the first width * height samples of the padded frame's luma
 * plane, which is what the rvsb CLI loads. */
rvsb_status rvsb_config_input_crop(const rvsb_config* cfg, int i, int32_t region[4], int32_t padded_size[2]);

/* Relative pose of an input camera seen from the virtual camera:
 * R = R_virt^T * R_in, t = -R_virt^T * (t_virt - t_in), in float with the
 * reference's operation order.  Replaces SpaceTransformer::get_rotation /
 * get_translation (rvs/src/SpaceTransformer.cpp:77-92) and
 * Parameters::getRotationMatrix (rvs/src/Parameters.cpp:151-155). */
rvsb_status rvsb_relative_pose(const rvsb_camera* input, const rvsb_camera* virt,
                               float R[9], float t[3]);

/* ----------------------------------------------------------------------- */
/* Scenes: input views resident in device memory                           */
/* ----------------------------------------------------------------------- */

typedef struct rvsb_scene rvsb_scene;

/* Creates a scene of n_inputs input cameras (the InputCameraNames order,
 * which is also the blend order, rvs/src/Pipeline.cpp:202-266) and reserves
 * device memory for their raw planes under the context's HBM budget. */
rvsb_status rvsb_scene_create(rvsb_context* ctx, const rvsb_camera* inputs, int n_inputs,
                              rvsb_scene** out);
void rvsb_scene_destroy(rvsb_scene* scene);

/* Uploads (host pointers, planes_on_device = 0) or copies (device pointers,
 * planes_on_device = 1) the raw planes of input view `view` into the scene.
 * Replaces InputView::load -> read_color / read_depth and their loader
 * kernels (rvs/src/View.cpp:233-257, rvs/src/image_loading.cpp:74-211,
 * rvs_cuda_lib/src/process_input_frame.cu:95-467); the decode itself is
 * fused into the synthesis kernels.  Planes that follow each other in the
 * caller's memory in the order y, u, v, depth (a view's colour frame and
 * depth frame read into one buffer) are copied in one transfer. */
rvsb_status rvsb_scene_upload(rvsb_scene* scene, int view, const rvsb_view_planes* planes,
                              int planes_on_device, void* stream);

/* ----------------------------------------------------------------------- */
/* Synthesis                                                                */
/* ----------------------------------------------------------------------- */

/* Synthesises the virtual camera `virt` from all views of `scene` into the
 * device planes `out` (YUV420, virt->bit_depth_color bits in uint16).
 * Replaces one pass of Pipeline::computeView (rvs/src/Pipeline.cpp:169-298):
 * SynthesizedView::compute + BlendedView::blend per input view, inpainting,
 * then the quantisation of write_color.  Asynchronous on `stream`. */
rvsb_status rvsb_synthesize(rvsb_scene* scene, const rvsb_camera* virt,
                            const rvsb_synth_params* params, const rvsb_yuv420* out,
                            void* stream);

/* One frame of the reference's per-frame path with the raw input planes
 * already in device memory (the InputView::load + computeView pair of
 * rvs/src/Pipeline.cpp:215-285): decodes every view's colour from
 * `device_planes` (n = the scene's view count) into the scene, reads their
 * depth planes in place and synthesises `virt` into `out`.  No plane is
 * copied; the planes must stay valid until the work on `stream` is done. */
rvsb_status rvsb_synthesize_frame(rvsb_scene* scene, const rvsb_view_planes* device_planes,
                                  const rvsb_camera* virt, const rvsb_synth_params* params,
                                  const rvsb_yuv420* out, void* stream);

/* The same call with host buffers on both sides (the reference's plain
 * per-frame path): uploads the n raw input views from host memory,
 * synthesises, and copies the YUV420 result back into host memory.  Blocks
 * until the result is in `out_host`.  Planes adjacent in host memory move
 * in one transfer, as in rvsb_scene_upload; so does an `out_host` whose U
 * plane follows Y and V follows U (one YUV420 frame buffer). */
rvsb_status rvsb_synthesize_host(rvsb_context* ctx, const rvsb_camera* inputs, int n_inputs,
                                 const rvsb_view_planes* host_planes, const rvsb_camera* virt,
                                 const rvsb_synth_params* params, const rvsb_yuv420* out_host,
                                 void* stream);

/* Frames with host buffers, pipelined: the reference's per-frame loop
 * (Pipeline.cpp:76-94 with its asynchronous loader and writer,
 * Pipeline.cpp:226-245) over one input camera set, with the upload of frame
 * k+1 on its own stream while frame k synthesises and the download of frame
 * k-1 on a third.  Up to three frames are in flight; a submit that would
 * start a fourth first waits for the oldest.  Host buffers are best pinned (else
 * the copies are synchronous) and best laid out as one buffer per frame: the
 * planes of all views back to back (per view y, u, v, depth, views in order)
 * go up in one transfer, and a YUV420 output buffer comes back in one; one
 * large transfer runs at the host link's full rate, sixteen plane-sized ones
 * about 12% below it.  They must stay untouched until the frame's
 * rvsb_host_stream_wait returns.  Each frame's uploads are ordered after
 * the work queued on `stream` before the submit (NULL: the legacy default
 * stream); rvsb_host_stream_join makes `stream` wait for every frame
 * submitted so far without blocking the host.  Results are the same as
 * rvsb_synthesize_host's. */
typedef struct rvsb_host_stream rvsb_host_stream;
rvsb_status rvsb_host_stream_create(rvsb_context* ctx, const rvsb_camera* inputs, int n_inputs,
                                    rvsb_host_stream** out);
void rvsb_host_stream_destroy(rvsb_host_stream* hs);
rvsb_status rvsb_host_stream_submit(rvsb_host_stream* hs, const rvsb_view_planes* host_planes,
                                    const rvsb_camera* virt, const rvsb_synth_params* params,
                                    const rvsb_yuv420* out_host, void* stream, uint64_t* ticket);
/* Blocks until frame `ticket` is in its host output buffers. */
rvsb_status rvsb_host_stream_wait(rvsb_host_stream* hs, uint64_t ticket);
rvsb_status rvsb_host_stream_join(rvsb_host_stream* hs, void* stream);

/* Intermediate results of one synthesis, for stage-by-stage checks against
 * the reference's CPU path.  Every pointer is a device pointer and may be
 * NULL; n = number of input views, W,H = input size, Wo,Ho = raster size (the
 * output size, or int(0.5 + Wout*P) x int(0.5 + Hout*P) for Precision P != 1).
 *   warped_uvz:    n*H*W*4 floats, (u, v, virtual depth, 0) per input pixel
 *                  (SynthesizedView::computeBasicMode, SynthesizedView.cpp:320-331)
 *   view_color:    n*Ho*Wo*3 floats, raster colour of each view
 *   view_depth:    n*Ho*Wo floats (+inf where uncovered)
 *   view_validity: n*Ho*Wo floats (triangle quality, 0 where uncovered)
 *                  (transform_trianglesMethod, rvs/src/transform.cpp:148-181)
 *   blend_color:   Ho*Wo*3 floats, blended colour before inpainting
 *   blend_quality: Ho*Wo floats, blended quality (BlendedView.cpp:180-212)
 *   inpaint_source: Ho*Wo int32 pairs (x, y) of the pixel each hole copies
 *                  (compute_nearest, rvs/src/inpainting.cpp:104-136) */
typedef struct rvsb_debug_out {
    float* warped_uvz;
    float* view_color;
    float* view_depth;
    float* view_validity;
    float* blend_color;
    float* blend_quality;
    int32_t* inpaint_source;
} rvsb_debug_out;

rvsb_status rvsb_synthesize_debug(rvsb_scene* scene, const rvsb_camera* virt,
                                  const rvsb_synth_params* params, const rvsb_yuv420* out,
                                  const rvsb_debug_out* dbg, void* stream);

/* Auxiliary outputs of one synthesis: the extra files the reference writes
 * in CPU mode (Pipeline.cpp:303-336; its CUDA mode skips them).  Device
 * pointers; any may be NULL.
 *   mask:          width*height bytes, 255 where the blended validity (the
 *                  maximum over the views of the winning triangle's quality)
 *                  is not above validity_threshold, else 0
 *                  (View::get_validity_mask, View.cpp:206-211; OutputMasks)
 *   masked:        YUV420 of the inpainted colour with masked pixels set to
 *                  0.5 (MaskedOutputFiles)
 *   depth:         width*height samples of the blended depth (the first
 *                  view's depth, replaced by a later view's where its quality
 *                  is larger, BlendedView.cpp:205-208) encoded as normalised
 *                  disparity with the virtual camera's Depth_range and
 *                  BitDepthDepth (write_depth, image_writing.cpp:232-268;
 *                  DepthOutputFiles)
 *   masked_depth:  the same, 0 where masked (MaskedDepthOutputFiles) */
typedef struct rvsb_aux_out {
    uint8_t* mask;
    rvsb_yuv420 masked;
    uint16_t* depth;
    uint16_t* masked_depth;
    float validity_threshold;  /* "ValidityThreshold" (default 5000) */
    int32_t reserved;
} rvsb_aux_out;

/* rvsb_synthesize plus the auxiliary outputs; Precision 1 only
 * (RVSB_E_UNSUPPORTED otherwise). */
rvsb_status rvsb_synthesize_aux(rvsb_scene* scene, const rvsb_camera* virt, const rvsb_synth_params* params,
                                const rvsb_yuv420* out, const rvsb_aux_out* aux, void* stream);

/* Kernel launches issued by the most recent synthesis call of the scene
 * (for launch accounting). */
int rvsb_scene_last_launch_count(const rvsb_scene* scene);
/* The raster autotuner (see rvsb_batch_set_autotune) for the per-view calls
 * of this scene (default off). */
rvsb_status rvsb_scene_set_autotune(rvsb_scene* scene, int enable);
/* Pins the raster variant of the scene's per-view calls (0 .. 7), or -1 for
 * the default or the tuner's choice; as rvsb_batch_set_raster_variant. */
rvsb_status rvsb_scene_set_raster_variant(rvsb_scene* scene, int variant);

/* ----------------------------------------------------------------------- */
/* Batches: many virtual views of one resident scene                       */
/* ----------------------------------------------------------------------- */

/* The reference synthesises one virtual view per Pipeline::computeView call
 * (rvs/src/Pipeline.cpp:169-345), frame after frame.  A batch runs up to
 * `max_slots` virtual views of the same uploaded input views together: each
 * kernel covers every slot in one launch, so a group of views costs the
 * launches of one view, and with graphs enabled the group's launch sequence
 * is captured once per shape and replayed.  Outputs are identical to one
 * rvsb_synthesize call per view.  Each slot holds its own workspace (grown
 * on first use, or up front with rvsb_batch_reserve).  Calls on one batch
 * must be ordered (one stream, or the caller waits between them). */
typedef struct rvsb_batch rvsb_batch;

rvsb_status rvsb_batch_create(rvsb_scene* scene, int max_slots, rvsb_batch** out);
void rvsb_batch_destroy(rvsb_batch* batch);
/* Allocates every slot's workspace for outputs up to max_width x max_height
 * now, so later calls of that size do not allocate. */
rvsb_status rvsb_batch_reserve(rvsb_batch* batch, int max_width, int max_height);
/* Capture each batch shape into a CUDA graph and replay it (default off). */
rvsb_status rvsb_batch_set_graphs(rvsb_batch* batch, int enable);
/* Raster autotuner (default off): the first batch of each new shape (batch
 * size bucket, largest input set and output, projections) is run once with
 * every raster variant -- tile size 32x32 or 64x32, views per shared
 * z-buffer group, the stretched-triangle threshold, threads per tile (512 or
 * 1024) and whether triangles whose candidate box holds up to 32 pixels
 * take the one-lane-per-pixel medium path -- and the fastest is kept for that shape.
 * All variants give identical outputs. */
rvsb_status rvsb_batch_set_autotune(rvsb_batch* batch, int enable);
/* Use one raster variant (0 .. 7) for every call, or -1 for the default or
 * tuned one; the variant used by the last call. */
rvsb_status rvsb_batch_set_raster_variant(rvsb_batch* batch, int variant);
int rvsb_batch_last_raster_variant(const rvsb_batch* batch);
/* n virtual views (outputs may differ in size and projection), processed in
 * groups of max_slots on `stream`. */
rvsb_status rvsb_synthesize_batch(rvsb_batch* batch, const rvsb_camera* virts, int n,
                                  const rvsb_synth_params* params, const rvsb_yuv420* outs, void* stream);
int rvsb_batch_last_launch_count(const rvsb_batch* batch);
rvsb_status rvsb_batch_set_profiling(rvsb_batch* batch, int enable);
int rvsb_batch_stage_times(rvsb_batch* batch, float* ms, int max_stages);

/* ----------------------------------------------------------------------- */
/* Serving: requests on resident scenes, continuous batching               */
/* ----------------------------------------------------------------------- */

/* No counterpart in the reference, which renders the frames of one
 * configuration in sequence (rvs/src/Application.cpp:53-65).  A server
 * accepts virtual-camera requests at any time on scenes whose input views
 * are resident, and a worker thread runs them on `lanes` independent batch
 * slots groups (one stream each): whenever a lane is free it launches every
 * waiting request that fits, up to `max_batch`, in arrival order, while the
 * workspace bytes of the requests in flight stay within `hbm_budget_bytes`
 * (0 = the context's budget).  Requests may mix scenes, output sizes and
 * projections; each output is identical to the same request alone. */
typedef struct rvsb_server rvsb_server;

typedef struct rvsb_request_result {
    uint64_t id;
    int32_t status;      /* rvsb_status of the request */
    int32_t batch_size;  /* requests launched together with it */
    double submit_s;     /* times on the server's clock (seconds) */
    double start_s;
    double done_s;
} rvsb_request_result;

rvsb_status rvsb_server_create(rvsb_context* ctx, int lanes, int max_batch, size_t hbm_budget_bytes,
                               rvsb_server** out);
/* Registers a scene (all views uploaded); its id goes to *scene_id. */
rvsb_status rvsb_server_add_scene(rvsb_server* server, rvsb_scene* scene, int* scene_id);
/* Allocates every slot's workspace for this scene at outputs up to
 * max_width x max_height, so serving does not allocate.  Only while idle. */
rvsb_status rvsb_server_reserve(rvsb_server* server, int scene_id, int max_width, int max_height);
/* Queues one request; `out` holds device planes the caller keeps valid
 * until the request's result has been polled. */
rvsb_status rvsb_server_submit(rvsb_server* server, int scene_id, const rvsb_camera* virt,
                               const rvsb_synth_params* params, const rvsb_yuv420* out, uint64_t* request_id);
/* Moves up to max_results finished requests into results; returns the count. */
int rvsb_server_poll(rvsb_server* server, rvsb_request_result* results, int max_results);
/* Waits until no request is waiting or running (RVSB_E_TIMEOUT otherwise). */
rvsb_status rvsb_server_drain(rvsb_server* server, int timeout_ms);
/* Seconds on the server's clock (the clock of the result times). */
double rvsb_server_clock(const rvsb_server* server);
void rvsb_server_destroy(rvsb_server* server);

/* Per-stage timing with CUDA events recorded on the launch stream (the
 * per-stage timers that replace the reference's whole-run clock(),
 * rvs/src/view_synthesis.cpp:149-166).  Stages: 0 warp, 1 bin, 2 raster
 * (with the resolve, blend and quantisation of every tile), 3 inpaint,
 * 4 whole synthesis. */
#define RVSB_NUM_STAGES 5
rvsb_status rvsb_scene_set_profiling(rvsb_scene* scene, int enable);
/* Milliseconds per stage of the most recent profiled synthesis; call after
 * its stream has completed.  Returns the number of values written, or -1. */
int rvsb_scene_stage_times(rvsb_scene* scene, float* ms, int max_stages);
const char* rvsb_stage_name(int stage);

/* Inpainting sources of a hole mask, computed without allocating memory.
 * This entry point has no counterpart in the reference.  It runs the
 * nearest-pixel inpainting scans of the synthesis (compute_nearest,
 * rvs/src/inpainting.cpp:104-136) over `holes` (width*height bytes in device
 * memory, nonzero = hole) and writes, for every pixel, the (x, y) of the
 * pixel whose colour the reference's inpainting copies into it (a non-hole
 * gets itself) to `sources` (width*height pairs of int32 in device memory).
 * It is for callers that must not allocate device memory while running;
 * its scratch is one static device array of 20 MiB, so images are limited
 * to 524,288 pixels (e.g. 960x540) and larger ones fail with RVSB_E_ARG and
 * a message in `err`; so do sides that are odd or outside 2..32768 (the
 * fill works on 2x2 blocks).  The first call on each device (with it current) does
 * a one-time set-up and should precede any stream capture.  Calls on one
 * device share the scratch: calls that overlap in time race, so order them
 * (for example on one stream).  Work is issued on `stream`. */
rvsb_status rvsb_inpaint_sources_noalloc(const uint8_t* holes, int width, int height, int32_t* sources,
                                         void* stream, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* RVSB_H */
