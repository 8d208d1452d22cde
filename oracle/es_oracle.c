/*
 * es_oracle.c -- TEST INFRASTRUCTURE, not product code (see es_oracle.h).
 *
 * Single-threaded, straightforward CPU restatement of the reference's per-frame measurement path. It favours obvious
 * correctness over speed: CAMBI windows are counted with a running histogram per row, the detail figures from exact
 * integer box sums. Build with -ffp-contract=off so that float and double arithmetic is rounded step by step.
 */
#include "es_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NONE (-1)

static int clampi(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

/* ---------------------------------------------------------------------------------------------------------------
 * Frame unpacking: src/kernels.cu:289-310 (sample, frame_planes).
 * --------------------------------------------------------------------------------------------------------------- */
static unsigned sample_at(const void *plane, int pitch, int x, int y, const eso_frame_view *f)
{
    const uint8_t *row = (const uint8_t *)plane + (size_t)y * pitch;
    const unsigned v = f->bytes == 1 ? row[x] : ((const uint16_t *)row)[x];
    return v >> f->shift;
}

void eso_frame_planes(const eso_frame_view *f, int x0, int y0, int pd, int w, int h, uint16_t *y16, uint16_t *u16,
                      uint16_t *v16)
{
    const int up = pd - f->depth;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) y16[(size_t)y * w + x] = (uint16_t)(sample_at(f->y, f->ypitch, x + x0, y + y0, f) << up);
    for (int y = 0; y < h; y += 2)
        for (int x = 0; x < w; x += 2) {
            const int cx = (x + x0) / 2, cy = (y + y0) / 2;
            const size_t ci = (size_t)(y / 2) * (w / 2) + x / 2;
            const unsigned u = f->semi ? sample_at(f->u, f->cpitch, 2 * cx, cy, f) : sample_at(f->u, f->cpitch, cx, cy, f);
            const unsigned v = f->semi ? sample_at(f->u, f->cpitch, 2 * cx + 1, cy, f) : sample_at(f->v, f->cpitch, cx, cy, f);
            u16[ci] = (uint16_t)(u << up);
            v16[ci] = (uint16_t)(v << up);
        }
}

/* ---------------------------------------------------------------------------------------------------------------
 * CAMBI parameters: src/cambi.cpp:21-53. The luminance model is restated from its published definitions:
 * ITU-R BT.1886 Annex 1 EOTF L = a * max(V + b, 0)^2.4 with a reference display of 300 cd/m2 white and 0.01 cd/m2
 * black, on 10-bit limited-range codes (64 black, 940 white), and CAMBI's Weber threshold of 0.019 for a visible
 * step (Tandon et al., "CAMBI: Contrast-aware Multiscale Banding Index", PCS 2021).
 * --------------------------------------------------------------------------------------------------------------- */
static const double kGamma = 2.4, kWhite = 300.0, kBlack = 0.01;
static const int kFoot = 64, kHead = 940;

static double luminance(int code)
{
    const double lw = pow(kWhite, 1.0 / kGamma), lb = pow(kBlack, 1.0 / kGamma);
    const double a = pow(lw - lb, kGamma), b = lb / (lw - lb);
    double v = (double)(code - kFoot) / (double)(kHead - kFoot);
    v = v < 0 ? 0 : v > 1 ? 1 : v;
    const double base = v + b > 0 ? v + b : 0;
    return a * pow(base, kGamma);
}

int eso_tvi_for_diff(int diff, double tvi_threshold)
{
    /* the largest code whose step up by `diff` codes is still visible: L(code + diff) - L(code) > t * L(code) */
    int last = kFoot;
    for (int code = kFoot; code + diff <= kHead; code++) {
        const double l = luminance(code);
        if (luminance(code + diff) - l > tvi_threshold * l) last = code;
    }
    return last;
}

int eso_vlt_luma(double threshold)
{
    /* the largest code whose luminance does not exceed the threshold; the black code when none does */
    int last = kFoot;
    for (int code = kFoot; code <= kHead; code++)
        if (luminance(code) <= threshold) last = code;
    return last;
}

static int ceil_log2(uint32_t n)
{
    int s = 0;
    for (uint32_t t = n ? n - 1 : 0; t; t >>= 1) s++;
    return s;
}

void eso_cambi_params_derive(int w, int h, eso_cambi_params *p)
{
    const int diffs = 4;
    memset(p, 0, sizeof *p);
    p->w = w;
    p->h = h;
    p->window = ((65 * (w + h) / 375) >> 4) | 1;
    p->pad = p->window >> 1;
    p->mask_index = (49 + 3 * (ceil_log2((uint32_t)((w >> 6) * (h >> 6))) - 11) - 1) >> 1;
    for (int d = 0; d < diffs; d++) {
        p->tvi[d] = eso_tvi_for_diff(d + 1, 0.019) + diffs;
        p->weight[d] = d + 1;
    }
    p->vlt = eso_vlt_luma(0.0);
    p->band_base = p->vlt - 3 * diffs + 1 > 0 ? p->vlt - 3 * diffs + 1 : 0;
    p->band_size = p->tvi[diffs - 1] + 1 - p->band_base;
    p->topk = 0.6;
}

/* ---------------------------------------------------------------------------------------------------------------
 * CAMBI per-scale steps.
 * --------------------------------------------------------------------------------------------------------------- */
void eso_cambi_preprocess(const uint16_t *img, int pitch, int w, int h, int depth, uint16_t *out)
{
    if (depth != 8) {
        for (int y = 0; y < h; y++) memcpy(out + (size_t)y * w, img + (size_t)y * pitch, (size_t)w * 2);
        return;
    }
    /* src/kernels.cu:524-535: shift to 10 bits, then the mean of the 2x2 block to the lower right (pairs on the last
     * row and column, the corner kept) */
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
#define AT(xx, yy) ((unsigned)img[(size_t)(yy) * pitch + (xx)] << 2)
            unsigned v;
            if (x < w - 1 && y < h - 1) v = (AT(x, y) + AT(x + 1, y) + AT(x, y + 1) + AT(x + 1, y + 1)) >> 2;
            else if (y < h - 1) v = (AT(x, y) + AT(x, y + 1)) >> 1;
            else if (x < w - 1) v = (AT(x, y) + AT(x + 1, y)) >> 1;
            else v = AT(x, y);
#undef AT
            out[(size_t)y * w + x] = (uint16_t)v;
        }
}

void eso_cambi_mask(const uint16_t *img, int w, int h, int index, uint8_t *mask)
{
    /* flat: equal to the right and lower neighbour, the last column / row counting as equal (cambi.c's zero
     * derivative); the mask counts flat pixels in the 7x7 square, nothing outside the picture */
    const size_t n = (size_t)w * h;
    uint8_t *flat = malloc(n);
    int *rows = malloc(n * sizeof(int));
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const size_t i = (size_t)y * w + x;
            flat[i] = (x == w - 1 || img[i] == img[i + 1]) && (y == h - 1 || img[i] == img[i + w]);
        }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int s = 0;
            for (int dx = -3; dx <= 3; dx++)
                if (x + dx >= 0 && x + dx < w) s += flat[(size_t)y * w + x + dx];
            rows[(size_t)y * w + x] = s;
        }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int s = 0;
            for (int dy = -3; dy <= 3; dy++)
                if (y + dy >= 0 && y + dy < h) s += rows[(size_t)(y + dy) * w + x];
            mask[(size_t)y * w + x] = s > index;
        }
    free(flat);
    free(rows);
}

void eso_decimate16(const uint16_t *src, int spitch, uint16_t *dst, int w, int h)
{
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) dst[(size_t)y * w + x] = src[(size_t)(2 * y) * spitch + 2 * x];
}

void eso_decimate8(const uint8_t *src, int spitch, uint8_t *dst, int w, int h)
{
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) dst[(size_t)y * w + x] = src[(size_t)(2 * y) * spitch + 2 * x];
}

static uint16_t mode3(uint16_t a, uint16_t b, uint16_t c)
{
    if (a == b || a == c) return a;
    if (b == c) return b;
    uint16_t m = a < b ? a : b;
    return m < c ? m : c;
}

void eso_cambi_mode(const uint16_t *img, int w, int h, uint16_t *out)
{
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const size_t i = (size_t)y * w + x;
            if (y == 0 || y == h - 1) { out[i] = img[i]; continue; }
            uint16_t m[3];
            for (int k = 0; k < 3; k++) {
                const uint16_t *row = img + (size_t)(y - 1 + k) * w;
                m[k] = (x == 0 || x == w - 1) ? row[x] : mode3(row[x - 1], row[x], row[x + 1]);
            }
            out[i] = mode3(m[0], m[1], m[2]);
        }
}

/* The c-value of a pixel whose number in the band is u, from the counts `hist` of every number in its window:
 * src/kernels.cu:188-205 (cambi.c's c_value_pixel with the reciprocal table, reciprocal_lut[i] = 1/i as float). */
static float cvalue_of(int u, const uint32_t *hist, const eso_cambi_params *p)
{
    const int value = u + p->band_base + 4;
    const unsigned p0 = hist[u];
    float c = 0.0f;
    for (int d = 0; d < 4; d++) {
        if (value <= p->tvi[d] && value + d + 1 > p->vlt) {
            const int q1 = u + d + 1, q2 = u - d - 1;
            const unsigned p1 = q1 < p->band_size ? hist[q1] : 0u, p2 = q2 >= 0 ? hist[q2] : 0u;
            const unsigned pm = p1 > p2 ? p1 : p2;
            const float recip = (float)(1.0 / (double)(p0 + pm));
            const float val = (float)(unsigned)((unsigned)p->weight[d] * p0 * pm) * recip;
            if (val > c) c = val;
        }
    }
    return c;
}

static int needs_cvalue(int u, const eso_cambi_params *p)
{
    if (u < 0) return 0;
    const int value = u + p->band_base + 4;
    for (int d = 0; d < 4; d++)
        if (value <= p->tvi[d] && value + d + 1 > p->vlt) return 1;
    return 0;
}

void eso_cambi_cvalues(const uint16_t *img, const uint8_t *mask, int w, int h, const eso_cambi_params *p, float *out,
                       uint64_t *sum_fx, uint64_t *count)
{
    const size_t n = (size_t)w * h;
    const int pad = p->pad;
    int *code = malloc(n * sizeof(int));
    uint32_t *hist = calloc((size_t)p->band_size + 1, sizeof(uint32_t));
    for (size_t i = 0; i < n; i++) {
        const unsigned u = (unsigned)img[i] - (unsigned)p->band_base;
        code[i] = mask[i] && u < (unsigned)p->band_size ? (int)u : NONE;
    }
    uint64_t s = 0, c = 0;
    for (int y = 0; y < h; y++) {
        float *row = out + (size_t)y * w;
        int any = 0;
        for (int x = 0; x < w && !any; x++) any = needs_cvalue(code[(size_t)y * w + x], p);
        memset(row, 0, (size_t)w * sizeof(float));
        if (!any) continue;
        const int y0 = y - pad < 0 ? 0 : y - pad, y1 = y + pad > h - 1 ? h - 1 : y + pad;
        memset(hist, 0, ((size_t)p->band_size + 1) * sizeof(uint32_t));
#define COLUMN(cx, delta)                                                                                             \
        for (int yy = y0; yy <= y1; yy++) {                                                                           \
            const int k = code[(size_t)yy * w + (cx)];                                                                \
            if (k != NONE) hist[k] += (delta);                                                                        \
        }
        for (int cx = 0; cx <= pad && cx < w; cx++) COLUMN(cx, 1u)
        for (int x = 0; x < w; x++) {
            if (x > 0) {
                if (x + pad < w) COLUMN(x + pad, 1u)
                if (x - pad - 1 >= 0) COLUMN(x - pad - 1, (uint32_t)-1)
            }
            const int u = code[(size_t)y * w + x];
            if (!needs_cvalue(u, p)) continue;
            const float v = cvalue_of(u, hist, p);
            row[x] = v;
            if (v > 0) {
                s += (uint64_t)(v * 16777216.0f);
                c++;
            }
        }
#undef COLUMN
    }
    free(code);
    free(hist);
    if (sum_fx) *sum_fx = s;
    if (count) *count = c;
}

size_t eso_topk_count(size_t n, double topk)
{
    const size_t k = (size_t)(int)(topk * (double)n);
    return k < 1 ? 1 : k > n ? n : k;
}

static int desc_float(const void *a, const void *b)
{
    const float x = *(const float *)a, y = *(const float *)b;
    return x < y ? 1 : x > y ? -1 : 0;
}

double eso_cambi_pool(const float *c, size_t n, double topk)
{
    const size_t k = eso_topk_count(n, topk);
    size_t m = 0;
    uint64_t sum = 0;
    for (size_t i = 0; i < n; i++)
        if (c[i] > 0) { m++; sum += (uint64_t)(c[i] * 16777216.0f); }
    if (m <= k) return (double)sum * (1.0 / 16777216.0) / (double)k;
    float *v = malloc(m * sizeof(float));
    size_t j = 0;
    for (size_t i = 0; i < n; i++)
        if (c[i] > 0) v[j++] = c[i];
    qsort(v, m, sizeof(float), desc_float);
    const float threshold = v[k - 1];
    uint64_t above_sum = 0;
    size_t above = 0;
    while (above < m && v[above] > threshold) above_sum += (uint64_t)(v[above++] * 16777216.0f);
    free(v);
    const double total = (double)above_sum * (1.0 / 16777216.0);
    return (total + (double)(k - above) * (double)threshold) / (double)k;
}

double eso_cambi_score(const uint16_t *img, int pitch, int w, int h, int depth, const eso_cambi_params *p,
                       uint16_t *const *images, uint8_t *const *masks, float *const *cvalues, double *pooled,
                       uint64_t *sums_fx, uint64_t *counts)
{
    static const int scale_weight[ESO_SCALES] = {16, 8, 4, 2, 1};
    const size_t n = (size_t)w * h;
    uint16_t *scratch = malloc(n * 2), *image = malloc(n * 2);
    uint8_t *mask = malloc(n), *mask_next = malloc(n);
    float *cv = malloc(n * sizeof(float));
    eso_cambi_preprocess(img, pitch, w, h, depth, scratch);
    eso_cambi_mask(scratch, w, h, p->mask_index, mask);
    double total = 0;
    int sw = w, sh = h;
    for (int s = 0; s < ESO_SCALES; s++) {
        if (s > 0) {
            const int pw = sw;
            sw = (sw + 1) >> 1;
            sh = (sh + 1) >> 1;
            eso_decimate16(image, pw, scratch, sw, sh);
            eso_decimate8(mask, pw, mask_next, sw, sh);
            memcpy(mask, mask_next, (size_t)sw * sh);
        }
        eso_cambi_mode(scratch, sw, sh, image);
        eso_cambi_params q = *p;
        q.w = sw;
        q.h = sh;
        uint64_t sfx, cnt;
        eso_cambi_cvalues(image, mask, sw, sh, &q, cv, &sfx, &cnt);
        const double pool = eso_cambi_pool(cv, (size_t)sw * sh, p->topk);
        if (images && images[s]) memcpy(images[s], image, (size_t)sw * sh * 2);
        if (masks && masks[s]) memcpy(masks[s], mask, (size_t)sw * sh);
        if (cvalues && cvalues[s]) memcpy(cvalues[s], cv, (size_t)sw * sh * sizeof(float));
        if (pooled) pooled[s] = pool;
        if (sums_fx) sums_fx[s] = sfx;
        if (counts) counts[s] = cnt;
        total += pool * (double)scale_weight[s];
    }
    free(scratch);
    free(image);
    free(mask);
    free(mask_next);
    free(cv);
    const int odd = 2 * (p->window >> 1) + 1;
    const double score = total / (double)(odd * odd);
    return score < 1000.0 ? score : 1000.0;
}

/* ---------------------------------------------------------------------------------------------------------------
 * Detail and texture figures, exact. With the luma Y on a 10-bit scale and S3 / S9 its 3x3 / 9x9 sums (edge pixels
 * repeated): fine = Y - S3/9, mid = S3/9 - S9/81, gx = (S3(x+1) - S3(x-1)) / 9 inside the picture, 0 on its border
 * columns, gy likewise; src/kernels.cu:346-428 and reference/encode_score/compare.py:77-108.
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct {
    int32_t *s3, *s9;
} box_sums;

static void box_of(const uint16_t *y, int up, int w, int h, box_sums *b)
{
    const size_t n = (size_t)w * h;
    int32_t *h3 = malloc(n * 4), *h9 = malloc(n * 4);
    b->s3 = malloc(n * 4);
    b->s9 = malloc(n * 4);
    for (int r = 0; r < h; r++)
        for (int x = 0; x < w; x++) {
            int32_t a = 0, c = 0;
            for (int d = -4; d <= 4; d++) {
                const int32_t v = (int32_t)y[(size_t)r * w + clampi(x + d, 0, w - 1)] << up;
                c += v;
                if (d >= -1 && d <= 1) a += v;
            }
            h3[(size_t)r * w + x] = a;
            h9[(size_t)r * w + x] = c;
        }
    for (int r = 0; r < h; r++)
        for (int x = 0; x < w; x++) {
            int32_t a = 0, c = 0;
            for (int d = -4; d <= 4; d++) {
                const size_t i = (size_t)clampi(r + d, 0, h - 1) * w + x;
                c += h9[i];
                if (d >= -1 && d <= 1) a += h3[i];
            }
            b->s3[(size_t)r * w + x] = a;
            b->s9[(size_t)r * w + x] = c;
        }
    free(h3);
    free(h9);
}

void eso_mid81(const uint16_t *y, int up, int w, int h, int32_t *mid81)
{
    box_sums b;
    box_of(y, up, w, h, &b);
    for (size_t i = 0; i < (size_t)w * h; i++) mid81[i] = 9 * b.s3[i] - b.s9[i];
    free(b.s3);
    free(b.s9);
}

static double oriented_of(int64_t jxx, int64_t jyy, int64_t jxy)
{
    /* sqrt((Jxx - Jyy)^2 + 4 Jxy^2) of the tensor summed from gradients times 9, then / 81; each double step rounded */
    const double d = (double)(jxx - jyy), x = (double)jxy;
    const double dd = d * d, xx = x * x;
    const double s = dd + 4.0 * xx;
    return sqrt(s) / 81.0;
}

void eso_window_stats(const uint16_t *yr, const uint16_t *yd, int up, int w, int h, double *out64, float *out32)
{
    const int ww = w / 16, wh = h / 16;
    box_sums br, bd;
    box_of(yr, up, w, h, &br);
    box_of(yd, up, w, h, &bd);
    for (int wy = 0; wy < wh; wy++)
        for (int wx = 0; wx < ww; wx++) {
            int64_t f_r = 0, m_r = 0, f_d = 0, m_d = 0, f_x = 0, m_x = 0;
            int64_t jr[3] = {0, 0, 0}, jd[3] = {0, 0, 0};
            for (int y = wy * 16; y < wy * 16 + 16; y++)
                for (int x = wx * 16; x < wx * 16 + 16; x++) {
                    const size_t i = (size_t)y * w + x;
                    const int64_t fr = 9 * ((int64_t)yr[i] << up) - br.s3[i], fd = 9 * ((int64_t)yd[i] << up) - bd.s3[i];
                    const int64_t mr = 9 * (int64_t)br.s3[i] - br.s9[i], md = 9 * (int64_t)bd.s3[i] - bd.s9[i];
                    f_r += fr * fr; m_r += mr * mr; f_d += fd * fd; m_d += md * md; f_x += fr * fd; m_x += mr * md;
                    int64_t gxr = 0, gyr = 0, gxd = 0, gyd = 0;
                    if (x > 0 && x < w - 1) { gxr = br.s3[i + 1] - br.s3[i - 1]; gxd = bd.s3[i + 1] - bd.s3[i - 1]; }
                    if (y > 0 && y < h - 1) { gyr = br.s3[i + w] - br.s3[i - w]; gyd = bd.s3[i + w] - bd.s3[i - w]; }
                    jr[0] += gxr * gxr; jr[1] += gyr * gyr; jr[2] += gxr * gyr;
                    jd[0] += gxd * gxd; jd[1] += gyd * gyd; jd[2] += gxd * gyd;
                }
            const double v[8] = {(double)f_r / 81.0, (double)m_r / 6561.0, (double)f_d / 81.0, (double)m_d / 6561.0,
                                 (double)f_x / 81.0, (double)m_x / 6561.0, oriented_of(jr[0], jr[1], jr[2]),
                                 oriented_of(jd[0], jd[1], jd[2])};
            const size_t o = ((size_t)wy * ww + wx) * 8;
            for (int k = 0; k < 8; k++) {
                if (out64) out64[o + k] = v[k];
                if (out32) out32[o + k] = (float)v[k];
            }
        }
    free(br.s3); free(br.s9); free(bd.s3); free(bd.s9);
}

void eso_persist_stats(const uint16_t *const *ring, const uint16_t *yd, int up, int w, int h, double *out64,
                       float *out32)
{
    const int ww = w / 16, wh = h / 16;
    const size_t n = (size_t)w * h;
    int32_t *mid[13], *md = malloc(n * 4);
    for (int k = 0; k < 13; k++) {
        mid[k] = malloc(n * 4);
        eso_mid81(ring[k], up, w, h, mid[k]);
    }
    eso_mid81(yd, up, w, h, md);
    for (int wy = 0; wy < wh; wy++)
        for (int wx = 0; wx < ww; wx++) {
            int64_t s[5] = {0, 0, 0, 0, 0};
            for (int y = wy * 16; y < wy * 16 + 16; y++)
                for (int x = wx * 16; x < wx * 16 + 16; x++) {
                    const size_t i = (size_t)y * w + x;
                    /* ring[k] is frame centre + k - 6: A from offsets +-2, 4, 6 and B from +-1, 3, 5, each times 486 */
                    const int64_t a = (int64_t)mid[0][i] + mid[2][i] + mid[4][i] + mid[8][i] + mid[10][i] + mid[12][i];
                    const int64_t b = (int64_t)mid[1][i] + mid[3][i] + mid[5][i] + mid[7][i] + mid[9][i] + mid[11][i];
                    const int64_t t = a + b; /* T times 972 */
                    s[0] += (int64_t)mid[6][i] * t;
                    s[1] += (int64_t)md[i] * t;
                    s[2] += a * b;
                    s[3] += a * a;
                    s[4] += b * b;
                }
            const double v[5] = {(double)s[0] / 78732.0, (double)s[1] / 78732.0, (double)s[2] / 236196.0,
                                 (double)s[3] / 236196.0, (double)s[4] / 236196.0};
            const size_t o = ((size_t)wy * ww + wx) * 5;
            for (int k = 0; k < 5; k++) {
                if (out64) out64[o + k] = v[k];
                if (out32) out32[o + k] = (float)v[k];
            }
        }
    for (int k = 0; k < 13; k++) free(mid[k]);
    free(md);
}

uint64_t eso_plane_sse(const uint16_t *a, const uint16_t *b, size_t n)
{
    uint64_t s = 0;
    for (size_t i = 0; i < n; i++) {
        const int64_t d = (int64_t)a[i] - (int64_t)b[i];
        s += (uint64_t)(d * d);
    }
    return s;
}

void eso_color_sums(const uint16_t *u, const uint16_t *v, size_t n, int up, double sums[3])
{
    uint64_t su = 0, sv = 0, ss = 0;
    for (size_t i = 0; i < n; i++) {
        const int uu = u[i] << up, vv = v[i] << up, du = uu - 512, dv = vv - 512;
        su += (uint64_t)uu;
        sv += (uint64_t)vv;
        ss += (uint64_t)llrint(sqrt((double)(du * du + dv * dv)) * 1073741824.0);
    }
    sums[0] = (double)su;
    sums[1] = (double)sv;
    sums[2] = (double)ss * (1.0 / 1073741824.0);
}

double eso_find_offset_lag(const float *ref, int n_ref, const float *probe, int n_probe, int *lag)
{
    const size_t n = (size_t)n_probe;
    double best = 1e30;
    int found = 0;
    for (int l = 0; l + n_probe <= n_ref; l++) {
        double total = 0;
        for (size_t i = 0; i < n && total < best * n * 2304; i++) {
            const float *r = ref + ((size_t)l + i) * 2304, *q = probe + i * 2304;
            for (int p = 0; p < 2304; p++) total += fabsf(r[p] - q[p]);
        }
        const double mean = total / (n * 2304.0);
        if (mean < best) {
            best = mean;
            found = l;
        }
    }
    *lag = found;
    return best;
}
