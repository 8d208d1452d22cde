/*
 * es_oracle.h -- TEST INFRASTRUCTURE, not product code.
 *
 * A plain-C, single-threaded CPU restatement of encode-score's per-frame measurement path: frame unpacking, CAMBI
 * (preprocessing, zero-derivative mask, decimation, mode filter, c-values, top-k pooling and score), the per-window
 * detail / structure-tensor statistics, the lasting-texture statistics, PSNR squared errors and color sums.
 *
 * It is the checker for the CUDA path and the timed CPU baseline. Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it; the product library never links or calls it.
 *
 * Each function names the reference lines it restates (paths inside the encode-score project). Where the reference
 * computes in FP32 (window_stats, persist_stats) this restatement computes the exact values (integer numerators, one
 * final rounding), i.e. it is the FP64 oracle the product is held to; where the reference adds doubles in an
 * unspecified atomic order (CAMBI sums) this restatement adds the exact fixed-point values.
 */
#ifndef ES_ORACLE_H
#define ES_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A decoded frame as the reference's kernels read it: src/kernels.cu:284-287 (struct Frame), src/main.cpp:99-102. */
typedef struct {
    const void *y, *u, *v;
    int ypitch, cpitch, semi, bytes, shift, depth;
} eso_frame_view;

/* CAMBI's derived parameters: src/cambi.cpp:39-53 and src/kernels.cu:65-69 (CambiParams). tvi[] is in the "+4"
 * adjusted space of cambi.c, as the reference's kernels take it. */
typedef struct {
    int w, h, window, pad, mask_index, band_base, band_size, vlt;
    int tvi[4];
    int weight[4];
    double topk;
} eso_cambi_params;

#define ESO_SCALES 5

/* src/kernels.cu:297-310 frame_planes: crop at (x0, y0) to w x h and unpack to planes at pipeline depth pd. */
void eso_frame_planes(const eso_frame_view *f, int x0, int y0, int pd, int w, int h, uint16_t *y16, uint16_t *u16,
                      uint16_t *v16);

/* src/cambi.cpp:39-53 (window, mask index, TVI/VLT/band) with the luminance model restated from its published
 * definitions (BT.1886 EOTF, 10-bit limited range, Weber threshold 0.019). */
void eso_cambi_params_derive(int w, int h, eso_cambi_params *p);
/* The TVI luma (raw, not +4 adjusted) for a luma step of `diff` codes, and the visibility luma threshold. */
int eso_tvi_for_diff(int diff, double tvi_threshold);
int eso_vlt_luma(double threshold);

/* src/kernels.cu:524-535 cambi_from8 (depth 8) or the plain copy of src/cambi.cpp:93-102 (depth 10). */
void eso_cambi_preprocess(const uint16_t *img, int pitch, int w, int h, int depth, uint16_t *out);
/* src/kernels.cu:14-40 cambi_mask. */
void eso_cambi_mask(const uint16_t *img, int w, int h, int index, uint8_t *mask);
/* src/kernels.cu:43-53 cambi_decimate16 / cambi_decimate8: dst (w, h) = src[2y][2x], src row pitch spitch. */
void eso_decimate16(const uint16_t *src, int spitch, uint16_t *dst, int w, int h);
void eso_decimate8(const uint8_t *src, int spitch, uint8_t *dst, int w, int h);
/* src/kernels.cu:488-500 cambi_mode with mode3 of 55-60. */
void eso_cambi_mode(const uint16_t *img, int w, int h, uint16_t *out);
/* src/kernels.cu:113-278 cambi_cvalues for one scale: out[n] gets every pixel's c-value (0 where none), and the
 * exact sum of the positive c-values in units of 2^-24 and their count. */
void eso_cambi_cvalues(const uint16_t *img, const uint8_t *mask, int w, int h, const eso_cambi_params *p, float *out,
                       uint64_t *sum_fx, uint64_t *count);
/* src/cambi.cpp:29 topk_count. */
size_t eso_topk_count(size_t n, double topk);
/* src/cambi.cpp:137-170 (topk_exact) and 179: the mean of the k largest of n c-values. */
double eso_cambi_pool(const float *c, size_t n, double topk);
/* src/cambi.cpp:88-184 launch + finish for one plane (pitch in pixels). Optional outputs, each may be NULL:
 * per-scale images, masks and c-values (caller-sized: scale s is ((w + 2^s - 1) >> s) x ((h + 2^s - 1) >> s)), the
 * pooled value of each scale, and the exact sums/counts of positive c-values. */
double eso_cambi_score(const uint16_t *img, int pitch, int w, int h, int depth, const eso_cambi_params *p,
                       uint16_t *const *images, uint8_t *const *masks, float *const *cvalues, double *pooled,
                       uint64_t *sums_fx, uint64_t *counts);

/* src/kernels.cu:346-428 window_stats, exact: per 16x16 window the 8 figures [src fine^2, src mid^2, enc fine^2,
 * enc mid^2, fine x, mid x, src oriented, enc oriented] in double (out64) and rounded to float (out32), either may
 * be NULL; `up` shifts the planes to a 10-bit scale. */
void eso_window_stats(const uint16_t *yr, const uint16_t *yd, int up, int w, int h, double *out64, float *out32);
/* The exact mid detail of a plane times 81 (9 * 3x3 sum - 9x9 sum, edges repeated), on the 10-bit scale. */
void eso_mid81(const uint16_t *y, int up, int w, int h, int32_t *mid81);
/* src/kernels.cu:435-451 persist_stats, exact: `ring` holds the 13 source luma planes of frames centre-6..centre+6
 * in order, `yd` the encode's luma at the centre. Per window [sum src*T, sum enc*T, sum A*B, sum A^2, sum B^2]. */
void eso_persist_stats(const uint16_t *const *ring, const uint16_t *yd, int up, int w, int h, double *out64,
                       float *out32);
/* src/kernels.cu:454-464 plane_sse: exact sum of squared differences. */
uint64_t eso_plane_sse(const uint16_t *a, const uint16_t *b, size_t n);
/* src/kernels.cu:470-484 color_sums: [sum U, sum V] exact on the 10-bit scale, and the sum of the color strength
 * sqrt(du^2 + dv^2), each term rounded to units of 2^-30 (the product's fixed-point definition). */
void eso_color_sums(const uint16_t *u, const uint16_t *v, size_t n, int up, double sums[3]);
/* src/main.cpp:339-348 find_offset's search, in its order of operations (float differences added in double, frame by
 * frame and pixel by pixel, a lag abandoned once its partial total reaches the best so far): the lag of least mean
 * difference of the n_probe thumbnails (2304 floats each) against n_ref reference thumbnails; returns that least mean
 * and writes the lag. */
double eso_find_offset_lag(const float *ref, int n_ref, const float *probe, int n_probe, int *lag);

#ifdef __cplusplus
}
#endif
#endif
