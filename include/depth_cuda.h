/* depth_cuda: B200 (sm_100a) stereo-depth hot path behind a plain C ABI.
 *
 * The stages: rectification remap of a raw IR pair -> 5x5 (configurable) census -> Hamming matching
 * cost -> multi-path SGM with P1/P2 -> winner-takes-all with subpixel fit -> left/right check ->
 * 3x3 median -> disparity-to-depth. It is a drop-in for the reference's GPU stereo matcher
 * (libs/depth_metal/include/einstar/depth_metal/metal_stereo.hpp:67-107, class MetalStereo), which
 * implements libs/depth's matcher interface (libs/depth/include/einstar/depth/stereo.hpp:96-115).
 *
 * Conventions
 * - Every entry point returns an int status with the values of einstar::Errc
 *   (libs/core/include/einstar/core/error.hpp:8-19); the message of the last failure is available from
 *   ds_last_error() (per handle) or ds_last_global_error() (create failures, per thread).
 * - Host images are u8 rows `stride` bytes apart (stride >= width); outputs are tightly packed.
 * - A handle is not thread-safe (as MetalStereo: callers serialise per handle). It owns all its device
 *   buffers and one CUDA stream.
 * - Disparities follow the reference: d = x_left - x_right, float, -1e9 where invalid
 *   (stereo.hpp:23-24). The u16 output is round((d - min_disparity) * 64), 0xFFFF where invalid.
 */
#ifndef DEPTH_CUDA_H
#define DEPTH_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DS_API __attribute__((visibility("default")))
#else
#define DS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* einstar::Errc (libs/core/include/einstar/core/error.hpp:8-19), same values. */
enum ds_status {
    DS_OK = 0,
    DS_NOT_FOUND = 1,
    DS_IO = 2,
    DS_TIMEOUT = 3,
    DS_PROTOCOL = 4,
    DS_INVALID_ARGUMENT = 5,
    DS_BLOCKED = 6,
    DS_UNSUPPORTED = 7,
    DS_BUSY = 8,
    DS_DISCONNECTED = 9
};

/* depth::SgmParams (libs/depth/include/einstar/depth/stereo.hpp:26-40); ints for bools. */
typedef struct ds_sgm_params {
    int min_disparity;
    int num_disparities; /* 1..512 */
    int census_radius_x; /* window (2rx+1) <= 9 */
    int census_radius_y; /* window (2ry+1) <= 7 */
    int p1;
    int p2;
    int adaptive_p2;
    int eight_paths;
    int slant_steps;
    float uniqueness;
    int lr_max_diff;
} ds_sgm_params;

/* depth::StereoParams (libs/depth/include/einstar/depth/stereo.hpp:41-88). With pyramid_levels = 0 and
 * the later stages off (ds_default_params) a frame is the hot path: SGM, L-R check and, with `median`,
 * a 3x3 median. Any of pyramid_levels > 0, detail_enabled, filter_occlusion, filter_spikes or
 * speckle_max_region_size > 1 selects depth::compute_disparity (stereo.cpp:501-536) instead: SGM at the
 * pyramid's coarsest level, slanted-window ZNCC refinement up to the stereo resolution, detail refinement
 * on the full-resolution pair (ds_compute_raw with remap tables at twice the stereo size), occlusion and
 * spike filters, speckle removal; the confidence is then the ZNCC score and `median` is not applied.
 * Those frames run through ds_compute* only (not in batches or the request server). */
typedef struct ds_stereo_params {
    int pyramid_levels;          /* 0..4: SGM at 1/2^levels of the stereo resolution */
    ds_sgm_params sgm;
    int subpixel;                /* parabola fit in the WTA (stereo.cpp:430-431) and the refinements */
    int median;                  /* hot path: 3x3 median of valid neighbours after the L-R check (stereo.cpp:129-147) */
    int detail_enabled;          /* depth::DetailParams::enabled */
    int filter_occlusion;        /* depth::FilterParams::occlusion */
    int filter_spikes;           /* depth::FilterParams::spikes */
    int speckle_max_region_size; /* depth::SpeckleParams::max_region_size (reference default 200) */
    int wide_costs;              /* 1: 16-bit path values even when census window + P2 <= 255 */
    /* depth::RefineParams (stereo.hpp:41-47) */
    int refine_search_radius;    /* 2 */
    int refine_zncc_radius;      /* 3 (7 x 7 window) */
    float refine_min_zncc;       /* 0.5 */
    int refine_reject_edge_winners; /* 1 */
    /* depth::DetailParams (stereo.hpp:53-61) */
    int detail_radius;           /* 5 (10 x 10 full-resolution window) */
    float detail_search;         /* 1 */
    float detail_step;           /* 0.5 */
    float detail_min_zncc;       /* 0.5 */
    /* depth::FilterParams, depth::SpeckleParams (stereo.hpp:66-79) */
    float occlusion_tolerance;   /* 1 */
    float spike_threshold;       /* 1 */
    float speckle_max_diff;      /* 1 */
} ds_stereo_params;

/* depth::RectifiedGeometry (libs/depth/include/einstar/depth/point_image.hpp:12-26). */
typedef struct ds_geometry {
    double f;
    double cx, cy;
    double baseline;
    double cx_offset;
} ds_geometry;

/* depth_metal::StereoTimings (metal_stereo.hpp:61-65). */
typedef struct ds_timings {
    double gpu_ms;     /* device time of the frame's work (CUDA events on the handle's stream) */
    double speckle_ms; /* always 0: no CPU speckle stage */
    double total_ms;   /* host wall time of the call */
} ds_timings;

/* Output slots of one frame; every pointer may be NULL (not produced). Host memory for
 * ds_compute / ds_compute_raw, device memory for the *_device variants. */
typedef struct ds_outputs {
    float* disparity;        /* W*H f32, after L-R check (+ median when enabled) */
    float* confidence;       /* W*H f32, 1 where the disparity is valid, else 0 (stereo.cpp:515-519) */
    uint16_t* disparity_u16; /* W*H u16 (see above) */
    float* depth;            /* W*H f32 mm, 0 where invalid or outside [min_depth, max_depth]; needs ds_set_point_params */
    uint8_t* rect_left;      /* W*H u8 rectified images (compute_raw only) */
    uint8_t* rect_right;
} ds_outputs;

typedef struct ds_handle ds_handle;

/* Hot-path defaults: depth::SgmParams defaults, pyramid 0, subpixel and median on, the later stages off
 * (their parameters at the reference's defaults). */
DS_API void ds_default_params(ds_stereo_params* params);

/* MetalStereo::create (metal_stereo.hpp:70-71; validation as metal_stereo.cpp:115-120). */
DS_API int ds_create(const ds_stereo_params* params, int width, int height, ds_handle** out);
DS_API void ds_destroy(ds_handle* handle);

/* MetalStereo::set_rectification (metal_stereo.hpp:75): float32 remap tables (map_x, map_y per camera,
 * map_width x map_height, tightly packed) copied to the device once and kept resident. The tables
 * are either at the stereo resolution (full-resolution SGM) or twice it, in which case the rectified
 * image is box-downsampled 2x2 as calib::remap + depth::downsample2 would give. */
DS_API int ds_set_rectification(ds_handle* handle, const float* map_left_x, const float* map_left_y,
                                 const float* map_right_x, const float* map_right_y, int map_width, int map_height,
                                 int raw_width, int raw_height);

/* MetalStereo::set_point_params (metal_stereo.hpp:84-85). */
DS_API int ds_set_point_params(ds_handle* handle, const ds_geometry* geometry, float min_depth_mm, float max_depth_mm,
                               float max_depth_jump_mm);

/* MetalStereo::compute (metal_stereo.hpp:78): already rectified pair, host memory. */
DS_API int ds_compute(ds_handle* handle, const uint8_t* left, const uint8_t* right, ptrdiff_t stride,
                      const ds_outputs* out);

/* MetalStereo::compute_raw (metal_stereo.hpp:80-81): raw pair (raw_width x raw_height), host memory. */
DS_API int ds_compute_raw(ds_handle* handle, const uint8_t* raw_left, const uint8_t* raw_right, ptrdiff_t stride,
                          const ds_outputs* out);

/* Device-resident variants (no counterpart in the reference, whose buffers live in unified memory):
 * inputs and outputs are device pointers (tightly packed), the work is enqueued on `stream`
 * (a cudaStream_t; NULL = the handle's own stream, cudaStreamLegacy for the legacy default stream) and
 * the call returns without waiting. */
DS_API int ds_compute_device(ds_handle* handle, const uint8_t* left, const uint8_t* right, const ds_outputs* out,
                             void* stream);
DS_API int ds_compute_raw_device(ds_handle* handle, const uint8_t* raw_left, const uint8_t* raw_right,
                                 const ds_outputs* out, void* stream);

/* MetalStereo::last_timings (metal_stereo.hpp:97). */
DS_API int ds_last_timings(const ds_handle* handle, ds_timings* out);
DS_API const char* ds_last_error(const ds_handle* handle);
DS_API const char* ds_last_global_error(void);

/* Intermediate results of the last frame, for stage-by-stage parity tests (host memory, may be NULL):
 * census words (u64, W*H each) and the summed path costs (u16, H*W*num_disparities, [y][x][d]). */
DS_API int ds_debug_read(ds_handle* handle, uint64_t* census_left, uint64_t* census_right, uint16_t* path_sums);

/* Device bytes the handle holds (all buffers). */
DS_API size_t ds_device_bytes(const ds_handle* handle);

/* Per-stage device times, the counterpart of the reference's per-stage GPU profile
 * (libs/gpu/include/einstar/gpu/profile.hpp:14-32; stage labels metal_stereo.cpp:480-652). When enabled,
 * every frame records CUDA events between its stages on the stream it runs on; nothing is serialised.
 * Stages: 0 rectify, 1 census, 2 costs (0 when the path kernels recompute them), 3 SGM paths,
 * 4 WTA + L-R check, 5 median + outputs (DS_STAGES). Up to 4096 frames may be pending between two
 * ds_profile_collect calls; a frame beyond that fails with DS_IO. */
#define DS_STAGES 6
DS_API int ds_profile_enable(ds_handle* handle, int on);
/* Waits for the profiled frames since the last call and writes up to `max_frames` rows of DS_STAGES
 * milliseconds each to `stage_ms` (row = frame, oldest first); `*frames` = rows written. */
DS_API int ds_profile_collect(ds_handle* handle, double* stage_ms, int max_frames, int* frames);

/* Number of kernels this library has launched since it was loaded (all handles). */
DS_API uint64_t ds_kernel_launches(void);

/* Kernel configuration (no counterpart in the reference; the Metal port picks its SIMD variant at
 * create, metal_stereo.cpp:178-189). A scanline is run by `lanes_per_line` lanes (8, 16 or 32) holding
 * 2*regs_per_lane disparities each, so lanes_per_line * 2 * regs_per_lane >= num_disparities (the WTA
 * picks its own split of the same disparities). Supported: 8 lanes with regs 4, 6, 8; 16 lanes with
 * regs 1..4; 32 lanes with regs 1, 2, 3, 4, 6, 8. materialize_costs: write the matching-cost volume once
 * instead of recomputing costs from the census in every direction. fused_pairs selects the sweep kernels
 * instead: the vertical path pair, then the horizontal pair with the WTA and the L-R check (two launches
 * per frame, 8 bytes of volume traffic per pixel and disparity). They need 4 paths, census windows of at
 * most 32 neighbours, 2 (window + P2) <= 255, and 4 or 8 lanes per line with regs 6 or 8 (D <= 128).
 * Otherwise, frames with 4 paths, byte path values (2 (window + P2) <= 255) and a slab of 64, 96 or 128
 * disparities take the row-sweep WTA, whose block shape is fixed (wta_threads applies to the others).
 * Results are identical for every configuration; only speed differs (the autotuner chooses). */
typedef struct ds_kernel_config {
    int regs_per_lane;
    int lanes_per_line;
    int materialize_costs;
    int path_warps_per_block; /* 1..8 */
    int wta_threads;          /* multiple of 32, 32..256 */
    int prefetch_steps;       /* 4 or 8: steps of inputs each scanline keeps in flight */
    int fused_pairs;          /* the sweep kernels (see above); block shapes are fixed */
    int horz_warps_per_block; /* unused by the sweep kernels (kept for layout) */
} ds_kernel_config;
DS_API int ds_set_kernel_config(ds_handle* handle, const ds_kernel_config* config);
DS_API int ds_get_kernel_config(const ds_handle* handle, ds_kernel_config* config);

/* ---- Batched path (no counterpart in the reference, which processes one frame per call) ----------
 * Many pairs of uneven size and disparity range run together: every stage is one persistent launch
 * per kernel variant that walks the blocks of all its pairs, and the whole batch is captured once into
 * a CUDA graph that ds_batch_run replays. Results are identical to per-pair ds_compute* calls. */
typedef struct ds_pair_desc {
    int width, height;         /* stereo resolution */
    ds_stereo_params params;
    int raw;                   /* 1: inputs are raw and rectified with calibration `calib` */
    int calib;                 /* 0 .. n_calib-1 */
    int have_geometry;         /* 1: depth output with `geometry` and the depth gates */
    ds_geometry geometry;
    float min_depth_mm, max_depth_mm;
    ds_kernel_config kernel;   /* regs_per_lane 0: the library's default */
} ds_pair_desc;

typedef struct ds_batch ds_batch;

/* Scheduling of a batch: pairs (heaviest first) are cut into micro-batches of `micro_batch` pairs that go
 * through all stages back to back (so a pair's volumes are consumed while still in L2), and the
 * micro-batches run round-robin on `branches` parallel branches of the graph. 0 = defaults (1, 8).
 * Micro-batches on one branch run one after another, so they share cost and path-value volumes: the
 * batch holds branches x micro_batch volumes (each sized for the largest pair it serves), not one per
 * pair. */
typedef struct ds_batch_options {
    int micro_batch;
    int branches;
} ds_batch_options;

DS_API int ds_batch_create(const ds_pair_desc* pairs, int n, int n_calib, const ds_batch_options* options,
                           ds_batch** out);
DS_API void ds_batch_destroy(ds_batch* batch);
DS_API const char* ds_batch_last_error(const ds_batch* batch);
/* Resident remap tables of calibration `calib` (as ds_set_rectification; tables of every raw pair using
 * it must be at its stereo resolution or twice it). */
DS_API int ds_batch_set_rectification(ds_batch* batch, int calib, const float* map_left_x, const float* map_left_y,
                                      const float* map_right_x, const float* map_right_y, int map_width,
                                      int map_height, int raw_width, int raw_height);
/* Device pointers of pair `pair`: inputs (raw or rectified, tightly packed) and outputs (NULL entries
 * go to the batch's internal buffers). Re-binding does not re-capture the graph. */
DS_API int ds_batch_bind(ds_batch* batch, int pair, const uint8_t* left, const uint8_t* right, const ds_outputs* out);
/* Enqueues the whole batch on `stream` (NULL: the batch's own stream) as one CUDA graph launch; the
 * graph is captured on the first call. */
DS_API int ds_batch_run(ds_batch* batch, void* stream);
/* The same launches without a graph (for comparison and debugging). */
DS_API int ds_batch_run_eager(ds_batch* batch, void* stream);
DS_API size_t ds_batch_device_bytes(const ds_batch* batch);
/* Kernel launches per run (persistent launches: one per stage and kernel variant). */
DS_API int ds_batch_launches_per_run(const ds_batch* batch);
/* The schedule in effect (defaults resolved). */
DS_API int ds_batch_get_options(const ds_batch* batch, ds_batch_options* out);
/* Stage timing of the last run, measured on the first micro-batch (CUDA events captured into the graph
 * between its stages, while the other branches run beside it):
 * 0 rectify, 1 census, 2 costs, 3 SGM paths, 4 WTA + L-R, 5 median + outputs (DS_BATCH_STAGES).
 * Enabling or disabling it captures the graph again on the next run. */
#define DS_BATCH_STAGES 6
DS_API int ds_batch_profile(ds_batch* batch, int on);
DS_API int ds_batch_stage_ms(ds_batch* batch, double* ms);

/* ---- Points, normals, weights (the hand-off to tracking) and the recording layout of depth ----------------
 * depth::PointImageParams (libs/depth/include/einstar/depth/point_image.hpp:41-47). */
typedef struct ds_point_params {
    float min_depth_mm;              /* 150 */
    float max_depth_mm;              /* 700 */
    float max_depth_jump_mm;         /* 4: neighbours used for normals */
    float edge_weight;               /* 0.25: view term of a point without a normal */
    float weight_reference_depth_mm; /* 0: no depth-noise term */
} ds_point_params;
DS_API void ds_default_point_params(ds_point_params* params);

/* depth::disparity_to_points (libs/depth/src/point_image.cpp:10-54) on device buffers, enqueued on
 * `stream` (a cudaStream_t; NULL = the default stream): organised points in the rectified left frame
 * (float4 x, y, z, w = 1 where valid, 0 elsewhere), unit normals towards the camera (float4, w = 0; zero
 * where unknown) and weights (confidence x view term x depth-noise term). `confidence` may be NULL
 * (weight 1). points_xyzw and normals_xyzw hold width * height float4, 16-byte aligned. Allocates
 * nothing. The Metal port's counterpart: disparity_points / point_normals
 * (libs/depth_metal/src/stereo_kernels.metal.inc:719-766). */
DS_API int ds_disparity_to_points(const float* disparity, const float* confidence, int width, int height,
                                  const ds_geometry* geometry, const ds_point_params* params, float* points_xyzw,
                                  float* normals_xyzw, float* weights, void* stream);

/* depth_metal::DepthPacker::pack (libs/depth_metal/src/depth_packer.cpp:10-21): the session file's
 * uncompressed depth layout, width * height * 3 bytes on the device: u16 depth in 1/50 mm delta-coded
 * along each row (value minus its left neighbour's, mod 2^16; 0 = no depth), then u8 confidence
 * round(weight * 255). `packed` must be 2-byte aligned. */
DS_API int ds_pack_depth(const float* points_xyzw, const float* weights, int width, int height, uint8_t* packed,
                         void* stream);

/* Raw IR images of a session recording (the RAWI record, libs/session/src/session.cpp:248-272, read back at
 * :815-836): after zstd decompression each row holds its bytes delta-coded from the left neighbour (mod 256).
 * Undoes that on the device, `coded` -> `image` (width x height, rows `*_stride` bytes apart), enqueued on
 * `stream`. In place when coded == image (equal strides); otherwise the buffers must not overlap. */
DS_API int ds_undelta_rows(const uint8_t* coded, ptrdiff_t coded_stride, uint8_t* image, ptrdiff_t image_stride, int width, int height,
                           void* stream);

/* ---- Marker blob search on the raw images -------------------------------------------------------------
 * depth_metal::BlobParams / BlobBox (metal_stereo.hpp:21-39) and MetalStereo::set_blob_params /
 * FrameRequest::marker_blobs (metal_stereo.hpp:41-58, 94-95): connected pixels above `threshold`
 * (4-neighbourhood, markers::find_blobs, libs/markers/src/detect.cpp:14-45), gated by box size, aspect,
 * fill and border, then a dark-ring pre-check on the blob's moment ellipse (the reference's GPU search,
 * stereo_kernels.metal.inc:770-901). The ring test uses exact half-angle formulas and a table of the 16
 * ring directions instead of atan2/cos/sin, so candidates are reproducible bit for bit. Candidates come
 * back ordered by their first pixel in raster order (the order of the CPU detector); when more than
 * max_blobs pass, `found` counts them all and which max_blobs are kept is unspecified. */
typedef struct ds_blob_params {
    uint32_t threshold;      /* 150: grey level a blob pixel exceeds */
    uint32_t min_diameter;   /* 3: box width and height limits (px) */
    uint32_t max_diameter;   /* 60 */
    float max_aspect;        /* 4: box aspect */
    float min_fill;          /* 0.5: pixels / (box area * pi / 4) */
    uint32_t border;         /* 4: room for the background ring */
    float max_axis_ratio;    /* 3: moment-ellipse axis ratio (x 1.2 leeway) */
    float ring_scale;        /* 1.4: the dark ring at this multiple of the moment ellipse */
    float ring_contrast;     /* 0.5: ring level between background and peak */
    float ring_max_bright;   /* 0.3: fraction of the 16 ring samples allowed above that level */
    uint32_t max_blobs;      /* 1024: candidates returned per image (1..65536) */
} ds_blob_params;

typedef struct ds_blob_box {
    uint32_t x0, y0, x1, y1; /* inclusive box */
    uint32_t pixels, peak;
} ds_blob_box;

/* Candidates of both raw images of a frame; `left`/`right` hold `capacity` boxes each (host memory). */
typedef struct ds_blob_boxes {
    ds_blob_box* left;
    ds_blob_box* right;
    uint32_t capacity;
    uint32_t found[2];       /* out: candidates that passed (before any cap) */
    uint32_t kept[2];        /* out: boxes written */
} ds_blob_boxes;

DS_API void ds_default_blob_params(ds_blob_params* params);
/* MetalStereo::set_blob_params: enables the blob search of ds_compute_raw_blobs; buffers are sized on
 * first use. */
DS_API int ds_set_blob_params(ds_handle* handle, const ds_blob_params* params);
/* ds_compute_raw plus the blob search on both raw images, run on a second stream concurrently with the
 * stereo (MetalStereo::compute_frame with FrameRequest::marker_blobs). */
DS_API int ds_compute_raw_blobs(ds_handle* handle, const uint8_t* raw_left, const uint8_t* raw_right, ptrdiff_t stride,
                                const ds_outputs* out, ds_blob_boxes* blobs);
/* MetalStereo::compute_frame (metal_stereo.hpp:92-95 with FrameRequest / FrameOutputs, :41-58), the call the
 * scanner frontend makes per frame (libs/pipeline/src/stereo_frontend.cpp:302-328): raw pair in; the
 * frame's points, normals and weights (ds_disparity_to_points with the handle's point parameters and the
 * default ds_point_params otherwise) written to the caller's device buffers and left there; optional host
 * copies (`host`: disparity, confidence, u16, depth, rectified pair); with `marker_blobs`, the blob
 * candidates of both raw images in `blobs`, handed to `on_blobs` (when set) on the calling thread as soon as
 * the blob search has finished, while the stereo may still run on the GPU. */
typedef void (*ds_blob_callback)(const ds_blob_boxes* blobs, void* user);
typedef struct ds_frame_request {
    int marker_blobs;          /* needs ds_set_blob_params */
    ds_blob_callback on_blobs; /* may be NULL */
    void* user;
} ds_frame_request;
typedef struct ds_frame_outputs {
    float* points_xyzw;        /* device, W*H float4 (16-byte aligned); with normals and weights, or all NULL */
    float* normals_xyzw;       /* device, W*H float4 */
    float* weights;            /* device, W*H */
    ds_outputs host;           /* host copies; entries may be NULL */
    ds_blob_boxes* blobs;      /* host; needed with marker_blobs */
} ds_frame_outputs;
DS_API int ds_compute_frame(ds_handle* handle, const uint8_t* raw_left, const uint8_t* raw_right, ptrdiff_t stride,
                            const ds_frame_request* request, ds_frame_outputs* out);
/* MetalStereo::compute_frame_raw (metal_stereo.hpp:86-90, metal_stereo.cpp:251-275): raw pair (host, rows `stride`
 * bytes apart) -> rectified -> stereo (with the handle's filters) -> points, normals and weights written to the
 * caller's device buffers (W*H float4, float4, float; required) and left there. rect_left / rect_right: host
 * W x H buffers for the rectified pair, or NULL. Needs ds_set_rectification and ds_set_point_params (the
 * reference's errors). Returns when the frame has finished. */
DS_API int ds_compute_frame_raw(ds_handle* handle, const uint8_t* raw_left, const uint8_t* raw_right, ptrdiff_t stride,
                                float* points_xyzw, float* normals_xyzw, float* weights, uint8_t* rect_left,
                                uint8_t* rect_right);

/* The blob search alone on one host image of any size (width x height, rows `stride` bytes apart):
 * up to `capacity` boxes, `found` = candidates that passed. Needs ds_set_blob_params. */
DS_API int ds_find_blobs(ds_handle* handle, const uint8_t* image, int width, int height, ptrdiff_t stride, ds_blob_box* out,
                         uint32_t capacity, uint32_t* found, uint32_t* kept);

/* ---- Request server: continuous batching of frames as they arrive (no counterpart in the reference,
 * whose frontend runs one camera pair synchronously, libs/pipeline/src/stereo_frontend.cpp:302-330) ------
 * A worker thread admits submitted frames in arrival order as soon as a slot (a CUDA stream with its own
 * frame buffers) is free and the cost / path-value volumes stay within `volume_budget_bytes`; admitted
 * frames run concurrently on their slots' streams. Volume memory is owned by the slots and reused: the
 * sum of all slots' volume buffers never exceeds the budget. Calibrations (remap tables, geometry) stay
 * resident on the device. Inputs are copied from and results to the caller's host buffers, which must
 * stay valid until the frame's completion has been polled; pinned host memory lets the copies overlap
 * other frames' work. */
typedef struct ds_server ds_server;

typedef struct ds_server_options {
    size_t volume_budget_bytes; /* 0: 40 GB */
    int max_slots;              /* frames on the GPU at once; 0: 8 */
    int max_pending;            /* queued frames before ds_server_submit returns DS_BUSY; 0: 4096 */
} ds_server_options;

typedef struct ds_request {
    int calib;                /* resident calibration of a raw pair; -1: the pair is already rectified */
    int width, height;        /* stereo (rectified) size */
    ds_stereo_params params;
    const uint8_t* left;      /* host; raw_width x raw_height (calib >= 0) or width x height */
    const uint8_t* right;
    ptrdiff_t stride;         /* bytes between rows of left and right */
    ds_outputs out;           /* host buffers, width x height (rect_left / rect_right unused) */
    uint64_t tag;             /* returned with the completion */
} ds_request;

typedef struct ds_completion {
    uint64_t ticket;
    uint64_t tag;
    int status;               /* DS_OK, or the failure's code (text: ds_server_last_error) */
    double queue_ms;          /* submit -> admission to a slot */
    double gpu_ms;            /* device time of the frame on its slot, copies included */
    double latency_ms;        /* submit -> results in host memory */
} ds_completion;

typedef struct ds_server_stats {
    uint64_t submitted, completed, failed;
    int pending, running, peak_running, slots;
    size_t running_volume_bytes, peak_running_volume_bytes;
    size_t volume_bytes;      /* volume memory held by the slots (<= the budget) */
    size_t device_bytes;      /* all device memory of the server */
} ds_server_stats;

/* Creates the server and its worker thread on the current device. */
DS_API int ds_server_create(const ds_server_options* options, ds_server** out);
/* Finishes the frames on the GPU, drops the pending ones and frees everything. */
DS_API void ds_server_destroy(ds_server* server);
DS_API const char* ds_server_last_error(const ds_server* server);
/* Resident calibration `calib` (>= 0): remap tables as ds_set_rectification, and the geometry used for
 * depth (NULL: frames of this calibration produce no depth). Replacing a calibration waits for the
 * frames in flight. */
DS_API int ds_server_add_calibration(ds_server* server, int calib, const float* map_left_x, const float* map_left_y,
                                     const float* map_right_x, const float* map_right_y, int map_width, int map_height,
                                     int raw_width, int raw_height, const ds_geometry* geometry, float min_depth_mm,
                                     float max_depth_mm);
/* Allocates, ahead of time, the buffers of `count` slots for frames of this size, parameters and
 * calibration (-1: rectified), so that serving them allocates nothing. */
DS_API int ds_server_reserve(ds_server* server, int width, int height, const ds_stereo_params* params, int calib,
                             int count);
/* Queues a frame (validated here) and returns at once; *ticket identifies its completion. */
DS_API int ds_server_submit(ds_server* server, const ds_request* request, uint64_t* ticket);
/* Waits up to timeout_ms (0: no wait, < 0: no limit) for at least one completion and returns up to `max`
 * of them, oldest first; *n = the number written. */
DS_API int ds_server_poll(ds_server* server, ds_completion* out, int max, int* n, int timeout_ms);
DS_API int ds_server_get_stats(ds_server* server, ds_server_stats* out);

/* ---- Disparity without device allocation (no counterpart in the reference) -----------------------
 * For callers that cannot allocate device memory when they need a disparity map: processes with a fixed
 * device-memory budget that forbid allocations after start-up, real-time loops where an allocation may
 * block or fail, frameworks whose own allocator owns the device. Computes what ds_compute_device computes
 * before its median (census, path aggregation, WTA, left/right check; the reference's sgm_disparity,
 * libs/depth/src/stereo.cpp:361-463) from `left`/`right` (device, tightly packed width x height u8) into
 * `disparity` (device, width x height f32), enqueued on `stream` (a cudaStream_t; NULL = the default
 * stream). Allocates nothing: all intermediates live in one static 16 MiB device array that every GPU
 * loading the library keeps until the process exits. A request whose intermediates exceed it
 * (two W x H census images of 4- or 8-byte words, plus P paths x W x H x disparities of 1- or 2-byte path
 * values; about 320 x 240 at 32 disparities and 4 paths fits) is rejected with DS_INVALID_ARGUMENT and a
 * message giving the bytes needed. The first call on each device looks up the array's device address
 * (with that device current) and should come before any stream capture. The address is kept per device
 * for the life of the process: calls must run in the device's primary context (the CUDA runtime's, which
 * is what cudaSetDevice makes current), and not after a cudaDeviceReset. Calls share the array: calls
 * whose work overlaps on the GPU (other streams, other threads) race and must be serialised by the
 * caller. Errors: ds_last_global_error(). */
DS_API int ds_sgm_disparity_noalloc(const uint8_t* left, const uint8_t* right, int width, int height,
                                    const ds_sgm_params* sgm, int subpixel, float* disparity, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DEPTH_CUDA_H */
