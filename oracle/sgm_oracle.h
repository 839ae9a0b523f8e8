/* CPU restatement ("port") of the reference's stereo-depth hot path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle: only tests/, the smoke check and the bench's
 * CPU-baseline leg may load it, and only as the checker or the timed CPU arm. The product path
 * (open_source_einstar_b200, libdepth_cuda.so) never calls it and has no CPU fallback.
 *
 * Each function cites the reference file:line it restates. Parity is pinned against the
 * reference itself: oracle/_ref (built from the reference's unmodified libs/depth/src/stereo.cpp)
 * and the golden fixtures under tests/golden/ generated from it.
 */
#ifndef SGM_ORACLE_H
#define SGM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirror of depth::SgmParams (libs/depth/include/einstar/depth/stereo.hpp:26-40). */
typedef struct orc_sgm_params {
    int min_disparity;
    int num_disparities;
    int census_radius_x;
    int census_radius_y;
    int p1;
    int p2;
    int adaptive_p2;
    int eight_paths;
    int slant_steps;
    float uniqueness;
    int lr_max_diff;
} orc_sgm_params;

/* kInvalidDisparity (stereo.hpp:23) and the integer kNoMatch of sgm_disparity (stereo.cpp:413). */
#define ORC_INVALID_DISPARITY (-1.0e9f)
#define ORC_NO_MATCH ((int32_t)0x80000000)

void orc_census(const uint8_t* img, int w, int h, int rx, int ry, uint64_t* out);
void orc_cost_volume(const uint64_t* cl, const uint64_t* cr, int w, int h, const orc_sgm_params* p, uint16_t* cost);
void orc_aggregate(const uint16_t* cost, const uint8_t* guide, int w, int h, const orc_sgm_params* p, uint16_t* sum);
void orc_wta(const uint16_t* sum, int w, int h, const orc_sgm_params* p, int subpixel, float* disp, int32_t* right_disp);
void orc_lr_check(float* disp, const int32_t* right_disp, int w, int h, int lr_max_diff);
int orc_sgm_disparity(const uint8_t* left, const uint8_t* right, int w, int h, const orc_sgm_params* p, int subpixel,
                      float* out);
void orc_median3(const float* in, int w, int h, float* out);
void orc_remap(const uint8_t* src, int src_w, int src_h, const float* map_x, const float* map_y, int w, int h, uint8_t* dst);
void orc_depth(const float* disp, int w, int h, double f, double baseline, double cx_offset, float min_depth, float max_depth,
               float* depth);
void orc_encode_u16(const float* disp, long n, int min_disparity, uint16_t* out);

/* depth::disparity_to_points (libs/depth/src/point_image.cpp:10-54; params point_image.hpp:41-54):
 * organised points in the rectified left frame (xyzw, w = 1 where valid), unit normals towards the camera
 * (xyzw, w = 0) from central differences, and weights = confidence x view term x depth-noise term.
 * `conf` may be NULL (weight 1). */
void orc_points(const float* disp, const float* conf, int w, int h, double f, double cx, double cy, double baseline,
                double cx_offset, float min_depth, float max_depth, float max_jump, float edge_weight,
                float weight_reference_depth, float* points, float* normals, float* weights);

/* depth_metal::DepthPacker (libs/depth_metal/src/depth_packer.cpp:10-21): u16 depth in 1/50 mm,
 * delta-coded along rows (q - q_left, mod 2^16), then u8 confidence round(w * 255); out = w*h*3 bytes. */
void orc_pack_depth(const float* points_xyzw, const float* weights, int w, int h, uint8_t* out);

/* Marker blob search. orc_find_blobs: connected pixels above `threshold` (4-neighbourhood), in the order
 * and with the statistics of markers::find_blobs (libs/markers/src/detect.cpp:14-45), plus each blob's
 * first pixel and its second moments relative to that pixel (32-bit two's complement sums). Returns the
 * number of blobs; at most `cap` are written. orc_blob_candidates: the gates and dark-ring pre-check of
 * the GPU search (stereo_kernels.metal.inc:846-900, restated with half-angle formulas and a table of the
 * 16 ring directions) over those blobs, in the same order; returns the number that pass, at most `cap`
 * written as (x0, y0, x1, y1, pixels, peak). */
typedef struct orc_blob {
    int32_t x0, y0, x1, y1, pixels, peak, root;
    int32_t mom[5];
} orc_blob;
typedef struct orc_blob_params {
    uint32_t threshold, min_diameter, max_diameter;
    float max_aspect, min_fill;
    uint32_t border;
    float max_axis_ratio, ring_scale, ring_contrast, ring_max_bright;
    uint32_t max_blobs;
} orc_blob_params;
int orc_find_blobs(const uint8_t* img, int w, int h, int threshold, orc_blob* out, int cap);
int orc_blob_candidates(const uint8_t* img, int w, int h, const orc_blob_params* p, uint32_t* boxes, int cap);

#ifdef __cplusplus
}
#endif

#endif
