// Texture window energies on larger windows, in three arithmetics, for the precision study (no counterpart in the
// reference, which sums FP32 box means on fixed 16 x 16 windows, src/kernels.cu:331-428).
//
// The box sums behind the figures (3 x 3 and 9 x 9 sums of luma, with the picture's edge pixels repeated) come from a
// summed-area table of each picture, kept three ways: int64 (exact), FP32 with two-sum compensation (a (hi, lo) pair
// per entry; Knuth's TwoSum), and plain FP32. From them each pixel's fine detail y - S3/9, mid detail S3/9 - S9/81 and
// box-3 gradients are formed: as exact integer numerators in the int64 form; in the compensated form as the same
// numerators in FP32 (9 y - S3, 9 S3 - S9 and differences of S3 are integers below 2^24, so exact) divided once; in the
// plain form as FP32 code usually does, from FP32 box means (y - S3/9, S3/9 - S9/81), which cancel. Their products are
// summed per 16 x 16 block (int64; FP32 with Neumaier's compensation; plain FP32). Windows of 16 k pixels sum k x k
// blocks in the same arithmetic and give the 8 figures of src/kernels.cu:340-341 as doubles.
#include "es_kernels.h"

namespace es {
namespace {

constexpr int kQ = 12;  // per block: fine_r^2, mid_r^2, fine_d^2, mid_d^2, fine_r fine_d, mid_r mid_d, Jxx_r, Jyy_r, Jxy_r, Jxx_d, Jyy_d, Jxy_d

__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e)
{
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// Neumaier's compensated accumulator
struct Comp {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float x)
    {
        float t, e;
        two_sum(s, x, t, e);
        s = t;
        c = __fadd_rn(c, e);
    }
    __device__ __forceinline__ float value() const { return __fadd_rn(s, c); }
};

// Column then row prefix sums of one picture (values << up): thread per column, then thread per row.
__global__ void sat_cols_kernel(const uint16_t *y, int w, int h, int up, long long *si, float *shi, float *slo, float *sp)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= w) return;
    long long a = 0;
    float hi = 0.0f, lo = 0.0f, p = 0.0f;
    for (int r = 0; r < h; r++) {
        const size_t k = (size_t)r * w + x;
        const int v = (int)y[k] << up;
        a += v;
        float t, e;
        two_sum(hi, (float)v, t, e);
        hi = t;
        lo = __fadd_rn(lo, e);
        p = __fadd_rn(p, (float)v);
        si[k] = a;
        shi[k] = hi;
        slo[k] = lo;
        sp[k] = p;
    }
}

__global__ void sat_rows_kernel(int w, int h, long long *si, float *shi, float *slo, float *sp)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= h) return;
    long long a = 0;
    float hi = 0.0f, lo = 0.0f, p = 0.0f;
    for (int x = 0; x < w; x++) {
        const size_t k = (size_t)r * w + x;
        a += si[k];
        float t, e;
        two_sum(hi, shi[k], t, e);
        hi = t;
        lo = __fadd_rn(__fadd_rn(lo, e), slo[k]);
        p = __fadd_rn(p, sp[k]);
        si[k] = a;
        shi[k] = hi;
        slo[k] = lo;
        sp[k] = p;
    }
}

struct SatView {
    const long long *si;
    const float *shi, *slo, *sp;
    const uint16_t *y;
    int w, h, up;
};

// Box sum of side 2r + 1 centred at (x, y) with the edge pixels repeated, in the three arithmetics. Inside the
// picture it is the table's 4-corner difference; near an edge it is summed directly over clamped coordinates.
__device__ void box_sum(const SatView &V, int x, int y, int r, long long &bi, float &bc, float &bp)
{
    if (x - r >= 0 && y - r >= 0 && x + r < V.w && y + r < V.h) {
        const int x1 = x + r, y1 = y + r, x0 = x - r - 1, y0 = y - r - 1;
        auto at = [&](int xx, int yy) { return (size_t)yy * V.w + xx; };
        long long a = V.si[at(x1, y1)];
        float h = V.shi[at(x1, y1)], l = V.slo[at(x1, y1)], p = V.sp[at(x1, y1)];
        auto sub = [&](int xx, int yy, float sign) {
            const size_t k = at(xx, yy);
            a += sign > 0 ? V.si[k] : -V.si[k];
            float t, e;
            two_sum(h, sign * V.shi[k], t, e);
            h = t;
            l = __fadd_rn(__fadd_rn(l, e), sign * V.slo[k]);
            p = __fadd_rn(p, sign * V.sp[k]);
        };
        if (x0 >= 0) sub(x0, y1, -1.0f);
        if (y0 >= 0) sub(x1, y0, -1.0f);
        if (x0 >= 0 && y0 >= 0) sub(x0, y0, 1.0f);
        bi = a;
        bc = __fadd_rn(h, l);
        bp = p;
        return;
    }
    long long a = 0;
    Comp c;
    float p = 0.0f;
    for (int dy = -r; dy <= r; dy++)
        for (int dx = -r; dx <= r; dx++) {
            const int xx = min(max(x + dx, 0), V.w - 1), yy = min(max(y + dy, 0), V.h - 1);
            const int v = (int)V.y[(size_t)yy * V.w + xx] << V.up;
            a += v;
            c.add((float)v);
            p = __fadd_rn(p, (float)v);
        }
    bi = a;
    bc = c.value();
    bp = p;
}

struct PixelTerms {
    long long f, m, gx, gy;  // exact numerators: fine x 9, mid x 81, gradients x 9
    float fc, mc, gxc, gyc;  // FP32 from the compensated table (gradients as their exact numerators, x 9)
    float fp, mp, gxp, gyp;  // FP32 from the plain table
};

__device__ PixelTerms pixel_terms(const SatView &V, int x, int y)
{
    PixelTerms t;
    long long s3, s9;
    float c3, c9, p3, p9;
    box_sum(V, x, y, 1, s3, c3, p3);
    box_sum(V, x, y, 4, s9, c9, p9);
    const int v = (int)V.y[(size_t)y * V.w + x] << V.up;
    t.f = 9 * (long long)v - s3;
    t.m = 9 * s3 - s9;
    t.fc = __fdiv_rn(__fsub_rn(__fmul_rn(9.0f, (float)v), c3), 9.0f);
    t.mc = __fdiv_rn(__fsub_rn(__fmul_rn(9.0f, c3), c9), 81.0f);
    t.fp = __fsub_rn((float)v, __fdiv_rn(p3, 9.0f));
    t.mp = __fsub_rn(__fdiv_rn(p3, 9.0f), __fdiv_rn(p9, 81.0f));
    t.gx = t.gy = 0;
    t.gxc = t.gyc = t.gxp = t.gyp = 0.0f;
    if (x > 0 && x < V.w - 1) {
        long long l, r;
        float lc, rc, lp, rp;
        box_sum(V, x - 1, y, 1, l, lc, lp);
        box_sum(V, x + 1, y, 1, r, rc, rp);
        t.gx = r - l;
        t.gxc = __fsub_rn(rc, lc);
        t.gxp = __fsub_rn(__fdiv_rn(rp, 9.0f), __fdiv_rn(lp, 9.0f));
    }
    if (y > 0 && y < V.h - 1) {
        long long u, d;
        float uc, dc, up, dp;
        box_sum(V, x, y - 1, 1, u, uc, up);
        box_sum(V, x, y + 1, 1, d, dc, dp);
        t.gy = d - u;
        t.gyc = __fsub_rn(dc, uc);
        t.gyp = __fsub_rn(__fdiv_rn(dp, 9.0f), __fdiv_rn(up, 9.0f));
    }
    return t;
}

// One block of 256 threads per 16 x 16 block: the 12 sums in the three arithmetics. The exact sums are in units of
// the numerators (fine and gradients x 9, mid x 81).
__global__ void __launch_bounds__(256) block_sums_kernel(SatView R, SatView D, int bw, long long *qi, float *qc, float *qp)
{
    __shared__ long long si[kQ][8];
    __shared__ float sc[kQ][8], sp[kQ][8];
    const int b = blockIdx.x, bx = b % bw, by = b / bw;
    const int x = 16 * bx + (threadIdx.x & 15), y = 16 * by + (threadIdx.x >> 4);
    const PixelTerms r = pixel_terms(R, x, y), d = pixel_terms(D, x, y);
    const long long vi[kQ] = {r.f * r.f, r.m * r.m, d.f * d.f, d.m * d.m, r.f * d.f, r.m * d.m,
                              r.gx * r.gx, r.gy * r.gy, r.gx * r.gy, d.gx * d.gx, d.gy * d.gy, d.gx * d.gy};
    // compensated form: the tensor's Jxx - Jyy summed per pixel as (gx - gy)(gx + gy) from the exact numerators, so
    // the cancellation of an isotropic texture happens before the sum; Jyy's slot is unused (0)
    auto dxy = [](float gx, float gy) { return __fdiv_rn(__fmul_rn(__fsub_rn(gx, gy), __fadd_rn(gx, gy)), 81.0f); };
    auto pxy = [](float gx, float gy) { return __fdiv_rn(__fmul_rn(gx, gy), 81.0f); };
    const float vc[kQ] = {r.fc * r.fc, r.mc * r.mc, d.fc * d.fc, d.mc * d.mc, r.fc * d.fc, r.mc * d.mc,
                          dxy(r.gxc, r.gyc), 0.0f, pxy(r.gxc, r.gyc), dxy(d.gxc, d.gyc), 0.0f, pxy(d.gxc, d.gyc)};
    const float vp[kQ] = {r.fp * r.fp, r.mp * r.mp, d.fp * d.fp, d.mp * d.mp, r.fp * d.fp, r.mp * d.mp,
                          r.gxp * r.gxp, r.gyp * r.gyp, r.gxp * r.gyp, d.gxp * d.gxp, d.gyp * d.gyp, d.gxp * d.gyp};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kQ; q++) {
        long long a = vi[q];
        float cs = vc[q], ce = 0.0f, p = vp[q];
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            const float os = __shfl_xor_sync(0xffffffffu, cs, o), oe = __shfl_xor_sync(0xffffffffu, ce, o);
            float t, e;
            two_sum(cs, os, t, e);
            cs = t;
            ce = __fadd_rn(__fadd_rn(ce, oe), e);
            p = __fadd_rn(p, __shfl_xor_sync(0xffffffffu, p, o));
        }
        if (lane == 0) {
            si[q][warp] = a;
            sc[q][warp] = __fadd_rn(cs, ce);
            sp[q][warp] = p;
        }
    }
    __syncthreads();
    if (threadIdx.x < kQ) {
        const int q = threadIdx.x;
        long long a = 0;
        Comp c;
        float p = 0.0f;
        for (int k = 0; k < 8; k++) {
            a += si[q][k];
            c.add(sc[q][k]);
            p = __fadd_rn(p, sp[q][k]);
        }
        qi[(size_t)b * kQ + q] = a;
        qc[(size_t)b * kQ + q] = c.value();
        qp[(size_t)b * kQ + q] = p;
    }
}

// Figures of each window of k x k blocks; mode 0 exact (int64, one rounding to double), 1 compensated FP32, 2 FP32.
__global__ void window_figures_kernel(const long long *qi, const float *qc, const float *qp, int bw, int bh, int k, int mode,
                                      double *out)
{
    const int ww = bw / k, wh = bh / k, i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ww * wh) return;
    const int wx = i % ww, wy = i / ww;
    double fig[8];
    if (mode == 0) {
        long long s[kQ] = {};
        for (int by = wy * k; by < wy * k + k; by++)
            for (int bx = wx * k; bx < wx * k + k; bx++)
                for (int q = 0; q < kQ; q++) s[q] += qi[((size_t)by * bw + bx) * kQ + q];
        fig[0] = (double)s[0] / 81.0;
        fig[1] = (double)s[1] / 6561.0;
        fig[2] = (double)s[2] / 81.0;
        fig[3] = (double)s[3] / 6561.0;
        fig[4] = (double)s[4] / 81.0;
        fig[5] = (double)s[5] / 6561.0;
        const double dr = (double)(s[6] - s[7]), xr = (double)s[8], dd = (double)(s[9] - s[10]), xd = (double)s[11];
        fig[6] = sqrt(dr * dr + 4.0 * xr * xr) / 81.0;
        fig[7] = sqrt(dd * dd + 4.0 * xd * xd) / 81.0;
    } else {
        float s[kQ];
        for (int q = 0; q < kQ; q++) {
            Comp c;
            float p = 0.0f;
            for (int by = wy * k; by < wy * k + k; by++)
                for (int bx = wx * k; bx < wx * k + k; bx++) {
                    const size_t at = ((size_t)by * bw + bx) * kQ + q;
                    if (mode == 1) c.add(qc[at]);
                    else p = __fadd_rn(p, qp[at]);
                }
            s[q] = mode == 1 ? c.value() : p;
        }
        for (int q = 0; q < 6; q++) fig[q] = (double)s[q];
        // compensated form: slots 6 and 9 already hold Jxx - Jyy
        const float dr = mode == 1 ? s[6] : __fsub_rn(s[6], s[7]), dd = mode == 1 ? s[9] : __fsub_rn(s[9], s[10]);
        fig[6] = (double)__fsqrt_rn(__fadd_rn(__fmul_rn(dr, dr), __fmul_rn(4.0f, __fmul_rn(s[8], s[8]))));
        fig[7] = (double)__fsqrt_rn(__fadd_rn(__fmul_rn(dd, dd), __fmul_rn(4.0f, __fmul_rn(s[11], s[11]))));
    }
    for (int q = 0; q < 8; q++) out[(size_t)i * 8 + q] = fig[q];
}

}  // namespace

int precision_quantities() { return kQ; }

cudaError_t launch_precision_sat(const uint16_t *y, int w, int h, int up, long long *si, float *shi, float *slo, float *sp,
                                 cudaStream_t s)
{
    {
        LaunchTimer t("precision_sat", s);
        sat_cols_kernel<<<(w + 127) / 128, 128, 0, s>>>(y, w, h, up, si, shi, slo, sp);
    }
    cudaError_t e = after_launch();
    if (e != cudaSuccess) return e;
    LaunchTimer t("precision_sat", s);
    sat_rows_kernel<<<(h + 127) / 128, 128, 0, s>>>(w, h, si, shi, slo, sp);
    return after_launch();
}

cudaError_t launch_precision_blocks(const uint16_t *yr, const uint16_t *yd, int w, int h, int up, const long long *const si[2],
                                    const float *const shi[2], const float *const slo[2], const float *const sp[2], long long *qi,
                                    float *qc, float *qp, cudaStream_t s)
{
    const int bw = w / 16, bh = h / 16;
    if (bw <= 0 || bh <= 0) return cudaSuccess;
    SatView R{si[0], shi[0], slo[0], sp[0], yr, w, h, up}, D{si[1], shi[1], slo[1], sp[1], yd, w, h, up};
    LaunchTimer t("precision_blocks", s);
    block_sums_kernel<<<bw * bh, 256, 0, s>>>(R, D, bw, qi, qc, qp);
    return after_launch();
}

cudaError_t launch_precision_windows(const long long *qi, const float *qc, const float *qp, int bw, int bh, int k, int mode,
                                     double *out, cudaStream_t s)
{
    const int n = (bw / k) * (bh / k);
    if (n <= 0) return cudaSuccess;
    LaunchTimer t("precision_windows", s);
    window_figures_kernel<<<(n + 127) / 128, 128, 0, s>>>(qi, qc, qp, bw, bh, k, mode, out);
    return after_launch();
}

}  // namespace es
