/* CPU restatement of the reference stereo hot path. TEST INFRASTRUCTURE ONLY (see sgm_oracle.h):
 * the checker for the CUDA kernels, never part of the product path.
 *
 * Build flags must keep float arithmetic un-contracted (-ffp-contract=off): the rectification remap
 * and the subpixel fit are compared bit-for-bit with the reference, which evaluates every float
 * operation separately.
 */
#include "sgm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define COST_MAX 0xFFFFu

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* Census transform, libs/depth/src/stereo.cpp:328-346. For every pixel at least (rx, ry) away from
 * the border, one bit per window neighbour in row-major order (centre skipped), first neighbour in the
 * most significant used bit; the bit is set when the neighbour is darker than the centre. Pixels
 * nearer the border get 0. */
void orc_census(const uint8_t* img, int w, int h, int rx, int ry, uint64_t* out) {
    memset(out, 0, (size_t)w * (size_t)h * sizeof(uint64_t));
    for (int y = ry; y < h - ry; ++y) {
        for (int x = rx; x < w - rx; ++x) {
            const uint8_t c = img[(size_t)y * w + x];
            uint64_t word = 0;
            for (int v = -ry; v <= ry; ++v)
                for (int u = -rx; u <= rx; ++u) {
                    if (u == 0 && v == 0) continue;
                    word = (word << 1) | (uint64_t)(img[(size_t)(y + v) * w + (x + u)] < c);
                }
            out[(size_t)y * w + x] = word;
        }
    }
}

/* Hamming cost volume [y][x][k], libs/depth/src/stereo.cpp:364-380: cost(x, y, k) is the popcount of
 * the two census words when the right pixel x - (min_disparity + k) is inside the row, else the
 * window area (2rx+1)(2ry+1). */
void orc_cost_volume(const uint64_t* cl, const uint64_t* cr, int w, int h, const orc_sgm_params* p, uint16_t* cost) {
    const int nd = p->num_disparities;
    const uint16_t invalid = (uint16_t)((2 * p->census_radius_x + 1) * (2 * p->census_radius_y + 1));
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            uint16_t* c = cost + ((size_t)y * w + x) * (size_t)nd;
            const uint64_t a = cl[(size_t)y * w + x];
            for (int k = 0; k < nd; ++k) {
                const int xr = x - (p->min_disparity + k);
                c[k] = (xr >= 0 && xr < w) ? (uint16_t)__builtin_popcountll(a ^ cr[(size_t)y * w + xr]) : invalid;
            }
        }
}

/* One scanline of the path recurrence, libs/depth/src/stereo.cpp:44-89. The first pixel takes its
 * costs unchanged; each following pixel adds, per disparity, the cheapest of: staying (prev[k]),
 * a one-step change (prev[k+-1] + P1), with slant steps a two-step change (prev[k+-2] + P1), or any
 * jump (min(prev) + P2'); minus min(prev). P2' shrinks across intensity edges of the left image:
 * max(P1 + 1, P2 / (|I - I_prev| / 8 + 1)). Values are 16-bit and added into `sum` with 16-bit
 * wrap-around, as the reference's uint16 volume does. */
static void run_line(const uint16_t* cost, const uint8_t* guide, int w, int h, const orc_sgm_params* p, int x, int y, int dx,
                     int dy, uint16_t* prev, uint16_t* cur, uint16_t* sum) {
    const int nd = p->num_disparities;
    const uint16_t* c = cost + ((size_t)y * w + x) * (size_t)nd;
    uint16_t* s = sum + ((size_t)y * w + x) * (size_t)nd;
    int pmin = COST_MAX;
    for (int k = 0; k < nd; ++k) {
        prev[k] = c[k];
        pmin = imin(pmin, c[k]);
        s[k] = (uint16_t)(s[k] + prev[k]);
    }
    int last_i = guide[(size_t)y * w + x];
    for (x += dx, y += dy; x >= 0 && y >= 0 && x < w && y < h; x += dx, y += dy) {
        const int I = guide[(size_t)y * w + x];
        const int p2 = p->adaptive_p2 ? imax(p->p1 + 1, p->p2 / (abs(I - last_i) / 8 + 1)) : p->p2;
        last_i = I;
        c = cost + ((size_t)y * w + x) * (size_t)nd;
        s = sum + ((size_t)y * w + x) * (size_t)nd;
        const int jump = pmin + p2;
        int cmin = COST_MAX;
        for (int k = 0; k < nd; ++k) {
            int b = imin(prev[k], jump);
            if (k >= 1) b = imin(b, prev[k - 1] + p->p1);
            if (k + 1 < nd) b = imin(b, prev[k + 1] + p->p1);
            if (p->slant_steps) {
                if (k >= 2) b = imin(b, prev[k - 2] + p->p1);
                if (k + 2 < nd) b = imin(b, prev[k + 2] + p->p1);
            }
            cur[k] = (uint16_t)(c[k] + b - pmin);
            cmin = imin(cmin, cur[k]);
        }
        for (int k = 0; k < nd; ++k) s[k] = (uint16_t)(s[k] + cur[k]);
        memcpy(prev, cur, (size_t)nd * sizeof(uint16_t));
        pmin = cmin;
    }
}

/* Sum of the 4 (or 8) path directions, libs/depth/src/stereo.cpp:382-409. A direction's lines start
 * at every pixel of its entry border(s); the lines of one direction are disjoint and together visit
 * every pixel once, so the order they run in does not matter. */
void orc_aggregate(const uint16_t* cost, const uint8_t* guide, int w, int h, const orc_sgm_params* p, uint16_t* sum) {
    static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {1, -1}, {-1, 1}};
    const int ndirs = p->eight_paths ? 8 : 4;
    const int nd = p->num_disparities;
    uint16_t* prev = (uint16_t*)malloc((size_t)nd * sizeof(uint16_t));
    uint16_t* cur = (uint16_t*)malloc((size_t)nd * sizeof(uint16_t));
    memset(sum, 0, (size_t)w * (size_t)h * (size_t)nd * sizeof(uint16_t));
    for (int di = 0; di < ndirs; ++di) {
        const int dx = dirs[di][0], dy = dirs[di][1];
        if (dx != 0) {
            const int sx = dx > 0 ? 0 : w - 1;
            for (int y = 0; y < h; ++y) run_line(cost, guide, w, h, p, sx, y, dx, dy, prev, cur, sum);
        }
        if (dy != 0) {
            const int sy = dy > 0 ? 0 : h - 1;
            const int corner = dx > 0 ? 0 : w - 1;
            for (int x = 0; x < w; ++x) {
                if (dx != 0 && x == corner) continue;
                run_line(cost, guide, w, h, p, x, sy, dx, dy, prev, cur, sum);
            }
        }
    }
    free(prev);
    free(cur);
}

/* Parabola through three costs, clamped to [-0.5, 0.5]; libs/depth/src/stereo.cpp:92-96. */
static float parabola(float cm, float c0, float cp) {
    const float denom = cm - 2.0f * c0 + cp;
    if (denom <= 0.0f) return 0.0f;
    float t = 0.5f * (cm - cp) / denom;
    if (t < -0.5f) t = -0.5f;
    if (t > 0.5f) t = 0.5f;
    return t;
}

/* Winner-takes-all, libs/depth/src/stereo.cpp:411-448.
 * Left: over the candidates whose right pixel is inside the image, the first strict minimum; rejected
 * when the best non-adjacent cost `second` exists and best >= uniqueness * second (float compare);
 * parabola subpixel when both neighbours are candidates.
 * Right: for each right pixel xr, the first strict minimum along the diagonal sum(xr + min + k)[k]. */
void orc_wta(const uint16_t* sum, int w, int h, const orc_sgm_params* p, int subpixel, float* disp, int32_t* right_disp) {
    const int nd = p->num_disparities, mind = p->min_disparity;
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const uint16_t* s = sum + ((size_t)y * w + x) * (size_t)nd;
            float* out = &disp[(size_t)y * w + x];
            *out = ORC_INVALID_DISPARITY;
            const int lo = imax(0, x - mind - (w - 1));
            const int hi = imin(nd, x - mind + 1);
            if (hi <= lo) continue;
            int best = lo;
            for (int k = lo + 1; k < hi; ++k)
                if (s[k] < s[best]) best = k;
            unsigned second = COST_MAX;
            for (int k = lo; k < hi; ++k)
                if ((k - best > 1 || best - k > 1) && s[k] < second) second = s[k];
            if (second != COST_MAX && (float)s[best] >= p->uniqueness * (float)second) continue;
            float d = (float)(mind + best);
            if (subpixel && best > lo && best + 1 < hi) d += parabola((float)s[best - 1], (float)s[best], (float)s[best + 1]);
            *out = d;
        }
        for (int xr = 0; xr < w; ++xr) {
            int best = -1;
            unsigned bv = COST_MAX;
            for (int k = imax(0, -(xr + mind)); k < nd; ++k) {
                const int xl = xr + mind + k;
                if (xl >= w) break;
                const uint16_t v = sum[((size_t)y * w + xl) * (size_t)nd + k];
                if (v < bv) {
                    bv = v;
                    best = k;
                }
            }
            right_disp[(size_t)y * w + xr] = best < 0 ? ORC_NO_MATCH : mind + best;
        }
    }
}

/* Left/right consistency, libs/depth/src/stereo.cpp:450-461: the matched right pixel is
 * lround(x - d) (halves away from zero); invalid when it leaves the row, has no right match, or its
 * right disparity differs from d by more than lr_max_diff. */
void orc_lr_check(float* disp, const int32_t* right_disp, int w, int h, int lr_max_diff) {
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            float* d = &disp[(size_t)y * w + x];
            if (!(*d > -1.0e8f)) continue;
            const long xr = lroundf((float)x - *d);
            if (xr < 0 || xr >= w) {
                *d = ORC_INVALID_DISPARITY;
                continue;
            }
            const int32_t r = right_disp[(size_t)y * w + xr];
            if (r == ORC_NO_MATCH || fabsf((float)r - *d) > (float)lr_max_diff) *d = ORC_INVALID_DISPARITY;
        }
}

/* depth::sgm_disparity, libs/depth/src/stereo.cpp:361-463, composed from the stages above. */
int orc_sgm_disparity(const uint8_t* left, const uint8_t* right, int w, int h, const orc_sgm_params* p, int subpixel,
                      float* out) {
    const size_t n = (size_t)w * (size_t)h, vol = n * (size_t)p->num_disparities;
    uint64_t* cl = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint64_t* cr = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint16_t* cost = (uint16_t*)malloc(vol * sizeof(uint16_t));
    uint16_t* sum = (uint16_t*)malloc(vol * sizeof(uint16_t));
    int32_t* rd = (int32_t*)malloc(n * sizeof(int32_t));
    if (!cl || !cr || !cost || !sum || !rd) {
        free(cl), free(cr), free(cost), free(sum), free(rd);
        return -1;
    }
    orc_census(left, w, h, p->census_radius_x, p->census_radius_y, cl);
    orc_census(right, w, h, p->census_radius_x, p->census_radius_y, cr);
    orc_cost_volume(cl, cr, w, h, p, cost);
    orc_aggregate(cost, left, w, h, p, sum);
    orc_wta(sum, w, h, p, subpixel, out, rd);
    orc_lr_check(out, rd, w, h, p->lr_max_diff);
    free(cl), free(cr), free(cost), free(sum), free(rd);
    return 0;
}

/* 3x3 median of the valid neighbours (centre included, image-bounded) of every valid pixel; invalid
 * pixels stay invalid. libs/depth/src/stereo.cpp:129-147 selects element n/2 with nth_element; the
 * same order statistic is taken here by insertion sort. */
void orc_median3(const float* in, int w, int h, float* out) {
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const float c = in[(size_t)y * w + x];
            out[(size_t)y * w + x] = ORC_INVALID_DISPARITY;
            if (!(c > -1.0e8f)) continue;
            float v[9];
            int n = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int xx = x + dx, yy = y + dy;
                    if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                    const float q = in[(size_t)yy * w + xx];
                    if (!(q > -1.0e8f)) continue;
                    int i = n++;
                    while (i > 0 && v[i - 1] > q) {
                        v[i] = v[i - 1];
                        --i;
                    }
                    v[i] = q;
                }
            out[(size_t)y * w + x] = v[n / 2];
        }
}

/* Bilinear remap, libs/calib/src/rectify.cpp:133-148: the 2x2 neighbourhood at floor(map) must be
 * inside the source, else 0; value ((a(1-fx) + b fx)(1-fy) + (c(1-fx) + d fx) fy), every float
 * operation rounded separately, then clamp(v + 0.5, 0, 255) truncated to u8. */
void orc_remap(const uint8_t* src, int src_w, int src_h, const float* map_x, const float* map_y, int w, int h, uint8_t* dst) {
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            const float sx = map_x[i], sy = map_y[i];
            const int x0 = (int)floorf(sx), y0 = (int)floorf(sy);
            if (x0 < 0 || y0 < 0 || x0 + 1 >= src_w || y0 + 1 >= src_h) {
                dst[i] = 0;
                continue;
            }
            const float fx = sx - (float)x0, fy = sy - (float)y0;
            const uint8_t* r0 = src + (size_t)y0 * src_w + x0;
            const uint8_t* r1 = r0 + src_w;
            const float a = r0[0], b = r0[1], c = r1[0], d = r1[1];
            const float gx = 1.0f - fx, gy = 1.0f - fy;
            const float top = a * gx + b * fx;
            const float bot = c * gx + d * fx;
            float v = top * gy + bot * fy;
            v = v + 0.5f;
            if (v < 0.0f) v = 0.0f;
            if (v > 255.0f) v = 255.0f;
            dst[i] = (uint8_t)v;
        }
}

/* Disparity to depth, libs/depth/include/einstar/depth/point_image.hpp:19 (z = f B / (d + cx_offset),
 * in double) with the gates of libs/depth/src/point_image.cpp:18-20: 0 where the disparity is invalid,
 * d + cx_offset <= 0, or z is outside [min_depth, max_depth]. */
void orc_depth(const float* disp, int w, int h, double f, double baseline, double cx_offset, float min_depth, float max_depth,
               float* depth) {
    const size_t n = (size_t)w * (size_t)h;
    for (size_t i = 0; i < n; ++i) {
        const float d = disp[i];
        depth[i] = 0.0f;
        if (!(d > -1.0e8f) || (double)d + cx_offset <= 0.0) continue;
        const double z = f * baseline / ((double)d + cx_offset);
        if (z < (double)min_depth || z > (double)max_depth) continue;
        depth[i] = (float)z;
    }
}

/* The u16 disparity format of this library (the reference keeps f32): round((d - min_disparity) * 64)
 * with ties to even, i.e. 1/64 px steps above the search's lower end, clamped to [0, 0xFFFE];
 * 0xFFFF where invalid. */
void orc_encode_u16(const float* disp, long n, int min_disparity, uint16_t* out) {
    for (long i = 0; i < n; ++i) {
        const float d = disp[i];
        if (!(d > -1.0e8f)) {
            out[i] = 0xFFFF;
            continue;
        }
        const float q = (d - (float)min_disparity) * 64.0f;
        long v = lrintf(q);
        if (v < 0) v = 0;
        if (v > 0xFFFE) v = 0xFFFE;
        out[i] = (uint16_t)v;
    }
}

/* Vec3f arithmetic as Eigen evaluates it for 3 floats (no fused multiply-add: built with
 * -ffp-contract=off): dot = (x*x' + y*y') + z*z', cross component-wise, norm = sqrt(dot(v, v)). */
static float dot3(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

void orc_points(const float* disp, const float* conf, int w, int h, double f, double cx, double cy, double baseline,
                double cx_offset, float min_depth, float max_depth, float max_jump, float edge_weight,
                float weight_reference_depth, float* points, float* normals, float* weights) {
    const size_t n = (size_t)w * (size_t)h;
    for (size_t i = 0; i < n; ++i) {
        for (int c = 0; c < 4; ++c) points[4 * i + c] = normals[4 * i + c] = 0.0f;
        weights[i] = 0.0f;
    }
    /* point_image.cpp:15-25 */
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            const float d = disp[i];
            if (!(d > -1.0e8f) || (double)d + cx_offset <= 0.0) continue;
            const double z = f * baseline / ((double)d + cx_offset);
            if (z < (double)min_depth || z > (double)max_depth) continue;
            points[4 * i + 0] = (float)(((double)x - cx) * z / f);
            points[4 * i + 1] = (float)(((double)y - cy) * z / f);
            points[4 * i + 2] = (float)z;
            points[4 * i + 3] = 1.0f;
            weights[i] = conf ? conf[i] : 1.0f;
        }
    /* point_image.cpp:27-51 */
    const float rc[3] = {(float)baseline, 0.0f, 0.0f};
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            const float* p = points + 4 * i;
            if (p[2] == 0.0f) continue;
            float view = edge_weight;
            if (x > 0 && y > 0 && x + 1 < w && y + 1 < h) {
                const float* l = points + 4 * (i - 1);
                const float* r = points + 4 * (i + 1);
                const float* u = points + 4 * (i - (size_t)w);
                const float* dn = points + 4 * (i + (size_t)w);
                if (l[2] != 0 && r[2] != 0 && u[2] != 0 && dn[2] != 0 && fabsf(l[2] - r[2]) <= max_jump &&
                    fabsf(u[2] - dn[2]) <= max_jump) {
                    const float a[3] = {r[0] - l[0], r[1] - l[1], r[2] - l[2]};
                    const float b[3] = {dn[0] - u[0], dn[1] - u[1], dn[2] - u[2]};
                    float nn[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
                    const float len = sqrtf(dot3(nn, nn));
                    if (len >= 1e-9f) {
                        for (int c = 0; c < 3; ++c) nn[c] = nn[c] / len;
                        if (dot3(nn, p) > 0) for (int c = 0; c < 3; ++c) nn[c] = -nn[c];
                        for (int c = 0; c < 3; ++c) normals[4 * i + c] = nn[c];
                        const float pl = sqrtf(dot3(p, p));
                        const float pn[3] = {p[0] / pl, p[1] / pl, p[2] / pl};
                        const float q[3] = {p[0] - rc[0], p[1] - rc[1], p[2] - rc[2]};
                        const float ql = sqrtf(dot3(q, q));
                        const float qn[3] = {q[0] / ql, q[1] / ql, q[2] / ql};
                        const float v1 = -dot3(nn, pn), v2 = -dot3(nn, qn);
                        const float m = v1 < v2 ? v1 : v2;
                        view = 0.0f > m ? 0.0f : m;
                    }
                }
            }
            float dw = 1.0f; /* depth_noise_weight, point_image.hpp:56-60 */
            if (weight_reference_depth > 0.0f) {
                const float rr = weight_reference_depth / p[2];
                const float r2 = rr * rr;
                dw = r2 > 1.0f ? 1.0f : (r2 < 0.1f ? 0.1f : r2);
            }
            weights[i] *= view * dw;
        }
}

static uint32_t quantize_mm50(float z) {
    if (!(z > 0.0f)) return 0u;
    float q = roundf(z * 50.0f);
    if (q < 1.0f) q = 1.0f;
    if (q > 65535.0f) q = 65535.0f;
    return (uint32_t)q;
}

void orc_pack_depth(const float* points_xyzw, const float* weights, int w, int h, uint8_t* out) {
    const size_t n = (size_t)w * (size_t)h;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            const uint32_t q = quantize_mm50(points_xyzw[4 * i + 2]);
            const uint32_t left = x > 0 ? quantize_mm50(points_xyzw[4 * (i - 1) + 2]) : 0u;
            const uint16_t dq = (uint16_t)((q - left) & 0xFFFFu);
            out[2 * i] = (uint8_t)(dq & 0xFF);
            out[2 * i + 1] = (uint8_t)(dq >> 8);
            float c = roundf(weights[i] * 255.0f);
            if (c < 0.0f) c = 0.0f;
            if (c > 255.0f) c = 255.0f;
            out[2 * n + i] = (uint8_t)c;
        }
}

/* ---- marker blob search ---------------------------------------------------------------------------------- */

/* Connected components above the threshold, libs/markers/src/detect.cpp:14-45: scan in raster order, flood
 * fill each unlabelled foreground pixel with an explicit stack. */
int orc_find_blobs(const uint8_t* img, int w, int h, int threshold, orc_blob* out, int cap) {
    const size_t n = (size_t)w * (size_t)h;
    int32_t* label = (int32_t*)malloc(n * sizeof(int32_t));
    int* stack = (int*)malloc(n * sizeof(int));
    if (!label || !stack) {
        free(label);
        free(stack);
        return -1;
    }
    for (size_t i = 0; i < n; ++i) label[i] = -1;
    int nb = 0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            if (img[i] <= threshold || label[i] >= 0) continue;
            orc_blob b;
            memset(&b, 0, sizeof(b));
            b.x0 = b.x1 = x;
            b.y0 = b.y1 = y;
            b.root = (int32_t)i;
            uint32_t m[5] = {0, 0, 0, 0, 0};
            int top = 0;
            stack[top++] = (int)i;
            label[i] = nb;
            while (top > 0) {
                const int p = stack[--top];
                const int px = p % w, py = p / w;
                ++b.pixels;
                if (img[p] > b.peak) b.peak = img[p];
                b.x0 = imin(b.x0, px), b.x1 = imax(b.x1, px), b.y0 = imin(b.y0, py), b.y1 = imax(b.y1, py);
                const int dx = px - x, dy = py - y;
                m[0] += (uint32_t)dx, m[1] += (uint32_t)dy, m[2] += (uint32_t)(dx * dx), m[3] += (uint32_t)(dx * dy),
                    m[4] += (uint32_t)(dy * dy);
                const int nbr[4][2] = {{px - 1, py}, {px + 1, py}, {px, py - 1}, {px, py + 1}};
                for (int k = 0; k < 4; ++k) {
                    const int qx = nbr[k][0], qy = nbr[k][1];
                    if (qx < 0 || qy < 0 || qx >= w || qy >= h) continue;
                    const size_t j = (size_t)qy * w + qx;
                    if (label[j] >= 0 || img[j] <= threshold) continue;
                    label[j] = nb;
                    stack[top++] = (int)j;
                }
            }
            for (int k = 0; k < 5; ++k) b.mom[k] = (int32_t)m[k];
            if (nb < cap) out[nb] = b;
            ++nb;
        }
    free(label);
    free(stack);
    return nb;
}

static const float k_ring_cos[16] = {1.0f, 0.923879533f, 0.707106781f, 0.382683432f, 0.0f, -0.382683432f, -0.707106781f, -0.923879533f,
                                     -1.0f, -0.923879533f, -0.707106781f, -0.382683432f, 0.0f, 0.382683432f, 0.707106781f, 0.923879533f};
static const float k_ring_sin[16] = {0.0f, 0.382683432f, 0.707106781f, 0.923879533f, 1.0f, 0.923879533f, 0.707106781f, 0.382683432f,
                                     0.0f, -0.382683432f, -0.707106781f, -0.923879533f, -1.0f, -0.923879533f, -0.707106781f, -0.382683432f};

/* Grey level at the nearest pixel (round half away from zero), coordinates clamped before the conversion. */
static float blob_sample(const uint8_t* img, int w, int h, float x, float y) {
    x = fminf(fmaxf(x, -1.0f), (float)w);
    y = fminf(fmaxf(y, -1.0f), (float)h);
    const int sx = imin(imax((int)roundf(x), 0), w - 1), sy = imin(imax((int)roundf(y), 0), h - 1);
    return (float)img[(size_t)sy * w + sx];
}

static float blob_ring(const uint8_t* img, int w, int h, int k, float su, float sv, float ct, float st, float cx, float cy) {
    const float u = su * k_ring_cos[k], v = sv * k_ring_sin[k];
    return blob_sample(img, w, h, (cx + ct * u) - st * v, (cy + st * u) + ct * v);
}

/* 1 when blob b passes the size, aspect, fill and border gates and the dark-ring pre-check. */
static int blob_passes(const uint8_t* img, int w, int h, const orc_blob_params* p, const orc_blob* b) {
    const float bw = (float)(b->x1 - b->x0 + 1), bh = (float)(b->y1 - b->y0 + 1);
    const float dmin = (float)p->min_diameter, dmax = (float)p->max_diameter;
    if (bw < dmin || bh < dmin || bw > dmax || bh > dmax) return 0;
    if (fmaxf(bw, bh) > p->max_aspect * fminf(bw, bh)) return 0;
    const float pi = 3.14159265358979f;
    if ((float)b->pixels < (((p->min_fill * bw) * bh) * pi) / 4.0f) return 0;
    const int m = imax(3, (int)fmaxf(bw, bh) / 2);
    const int bd = (int)p->border;
    if (b->x0 - m < bd || b->y0 - m < bd || b->x1 + m >= w - bd || b->y1 + m >= h - bd) return 0;
    const float fn = (float)b->pixels;
    const float mx = (float)b->mom[0] / fn, my = (float)b->mom[1] / fn;
    const float cxx = (float)b->mom[2] / fn - mx * mx;
    const float cxy = (float)b->mom[3] / fn - mx * my;
    const float cyy = (float)b->mom[4] / fn - my * my;
    const float dxy = cxx - cyy;
    const float tr = 0.5f * (cxx + cyy);
    const float det = sqrtf(fmaxf(0.0f, (0.25f * dxy) * dxy + cxy * cxy));
    const float l1 = tr + det, l2 = fmaxf(tr - det, 0.0625f);
    const float ea = 2.0f * sqrtf(fmaxf(l1, 0.0f)) + 0.5f, eb = 2.0f * sqrtf(l2) + 0.5f;
    if (ea / eb > p->max_axis_ratio * 1.2f) return 0;
    const float s2 = 2.0f * cxy;
    const float r2 = sqrtf(dxy * dxy + s2 * s2);
    float ct = 1.0f, st = 0.0f;
    if (r2 > 0.0f) {
        const float c2 = fminf(fmaxf(dxy / r2, -1.0f), 1.0f);
        ct = sqrtf(0.5f * (1.0f + c2));
        st = sqrtf(0.5f * (1.0f - c2));
        if (s2 < 0.0f) st = -st;
    }
    const float cx = (float)(b->root % w) + mx, cy = (float)(b->root / w) + my;
    float bg[16];
    const float bu = 2.2f * ea, bv = 2.2f * eb;
    for (int k = 0; k < 16; ++k) bg[k] = blob_ring(img, w, h, k, bu, bv, ct, st, cx, cy);
    for (int a = 0; a < 4; ++a)
        for (int q = a + 1; q < 16; ++q)
            if (bg[q] < bg[a]) {
                const float t = bg[a];
                bg[a] = bg[q];
                bg[q] = t;
            }
    const float level = bg[3] + p->ring_contrast * ((float)b->peak - bg[3]);
    const float ru = p->ring_scale * ea, rv = p->ring_scale * eb;
    int bright = 0;
    for (int k = 0; k < 16; ++k) bright += blob_ring(img, w, h, k, ru, rv, ct, st, cx, cy) > level ? 1 : 0;
    return (float)bright > p->ring_max_bright * 16.0f ? 0 : 1;
}

int orc_blob_candidates(const uint8_t* img, int w, int h, const orc_blob_params* p, uint32_t* boxes, int cap) {
    const int nb = orc_find_blobs(img, w, h, (int)p->threshold, NULL, 0);
    if (nb < 0) return -1;
    orc_blob* blobs = (orc_blob*)malloc((size_t)(nb > 0 ? nb : 1) * sizeof(orc_blob));
    if (!blobs) return -1;
    orc_find_blobs(img, w, h, (int)p->threshold, blobs, nb);
    int found = 0;
    for (int i = 0; i < nb; ++i) {
        if (!blob_passes(img, w, h, p, &blobs[i])) continue;
        if (found < cap) {
            uint32_t* o = boxes + 6 * (size_t)found;
            o[0] = (uint32_t)blobs[i].x0, o[1] = (uint32_t)blobs[i].y0, o[2] = (uint32_t)blobs[i].x1, o[3] = (uint32_t)blobs[i].y1;
            o[4] = (uint32_t)blobs[i].pixels, o[5] = (uint32_t)blobs[i].peak;
        }
        ++found;
    }
    free(blobs);
    return found;
}
