// Per-frame measures other than CAMBI, for sm_100a: frame unpacking, the detail / structure-tensor window energies,
// the lasting-texture statistics, PSNR squared errors, color sums and the per-frame reduction into segment figures.
//
// The reference (src/kernels.cu:297-484, src/main.cpp:518-643) computes the window energies in FP32 from exact box
// sums, writes two full FP32 mid-detail planes per encode, re-reads 13 of them per encode for the lasting texture and
// reduces the windows on the host. Here every figure is computed from integer numerators (fine x 9, mid x 81,
// gradients x 9) summed exactly in int64 and rounded once; the lasting texture keeps running integer sums of the
// source's luma over the even and odd frame offsets (mid detail is linear in luma), so a frame step reads a few
// 16-bit planes once for all encodes; and the per-frame reduction (structure threshold as an exact order statistic,
// masks, sums, histogram bins) runs on the device.
#include "es_kernels.h"

namespace es {
namespace {

// ---------------------------------------------------------------------------------------------------------------
// Frame unpacking: src/kernels.cu:289-310.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned sample_at(const void *plane, int pitch, int x, int y, const FrameViewDev &f)
{
    const unsigned char *row = (const unsigned char *)plane + (size_t)y * pitch;
    const unsigned v = f.bytes == 1 ? row[x] : ((const uint16_t *)row)[x];
    return v >> f.shift;
}

// Thread i takes 4 consecutive 2 x 2 groups of one chroma row (2 rows x 8 luma columns, 4 samples of U and of V).
// Planar frames whose rows and crop allow it are moved with 16- / 8-byte loads and stores; every other layout
// (semi-planar, shifted samples such as P010, odd alignments) one sample at a time.
__global__ void __launch_bounds__(256) unpack_kernel(const __grid_constant__ UnpackBatch b)
{
    const int j = find_job(b.njobs, (int)blockIdx.x, [&](int k) { return b.job[k].first_block; });
    const UnpackJob &J = b.job[j];
    const FrameViewDev f = b.views ? b.views[j].f : J.f;
    const int x0 = b.views ? b.views[j].x0 : J.x0, y0 = b.views ? b.views[j].y0 : J.y0;
    const int cw = J.w / 2, ch = J.h / 2, qw = (cw + 3) / 4;
    const int i = (blockIdx.x - J.first_block) * 256 + threadIdx.x;
    if (i >= qw * ch) return;
    const int cy = i / qw, cx0 = 4 * (i - cy * qw), up = J.pd - f.depth;
    const bool full = cx0 + 4 <= cw && !f.semi && f.shift == 0 && (x0 & 7) == 0;
    if (full && f.bytes == 2 && (f.ypitch & 15) == 0 && (f.cpitch & 7) == 0 && (((uintptr_t)f.y & 15) | ((uintptr_t)f.u & 7) | ((uintptr_t)f.v & 7)) == 0 &&
        (J.w & 7) == 0) {
        auto sh4 = [&](uint4 q) { return make_uint4(q.x << up, q.y << up, q.z << up, q.w << up); };  // samples < 2^10
#pragma unroll
        for (int dy = 0; dy < 2; dy++) {
            const uint4 q = __ldg((const uint4 *)((const unsigned char *)f.y + (size_t)(2 * cy + dy + y0) * f.ypitch) + (2 * cx0 + x0) / 8);
            *(uint4 *)(J.y16 + (size_t)(2 * cy + dy) * J.w + 2 * cx0) = sh4(q);
        }
        const size_t co = (size_t)(cy + y0 / 2) * f.cpitch;
        const uint2 u = __ldg((const uint2 *)((const unsigned char *)f.u + co) + (cx0 + x0 / 2) / 4);
        const uint2 v = __ldg((const uint2 *)((const unsigned char *)f.v + co) + (cx0 + x0 / 2) / 4);
        *(uint2 *)(J.u16 + (size_t)cy * cw + cx0) = make_uint2(u.x << up, u.y << up);
        *(uint2 *)(J.v16 + (size_t)cy * cw + cx0) = make_uint2(v.x << up, v.y << up);
        return;
    }
    if (full && f.bytes == 1 && (f.ypitch & 7) == 0 && (f.cpitch & 3) == 0 && (((uintptr_t)f.y & 7) | ((uintptr_t)f.u & 3) | ((uintptr_t)f.v & 3)) == 0 &&
        (J.w & 7) == 0) {
        auto widen2 = [&](unsigned q) {  // 4 bytes -> 4 16-bit samples, shifted
            return make_uint2(__byte_perm(q, 0, 0x4140) << up, __byte_perm(q, 0, 0x4342) << up);
        };
#pragma unroll
        for (int dy = 0; dy < 2; dy++) {
            const uint2 q = __ldg((const uint2 *)((const unsigned char *)f.y + (size_t)(2 * cy + dy + y0) * f.ypitch) + (2 * cx0 + x0) / 8);
            const uint2 lo = widen2(q.x), hi = widen2(q.y);
            *(uint4 *)(J.y16 + (size_t)(2 * cy + dy) * J.w + 2 * cx0) = make_uint4(lo.x, lo.y, hi.x, hi.y);
        }
        const size_t co = (size_t)(cy + y0 / 2) * f.cpitch;
        const unsigned u = __ldg((const unsigned *)((const unsigned char *)f.u + co) + (cx0 + x0 / 2) / 4);
        const unsigned v = __ldg((const unsigned *)((const unsigned char *)f.v + co) + (cx0 + x0 / 2) / 4);
        *(uint2 *)(J.u16 + (size_t)cy * cw + cx0) = widen2(u);
        *(uint2 *)(J.v16 + (size_t)cy * cw + cx0) = widen2(v);
        return;
    }
    for (int cx = cx0; cx < min(cx0 + 4, cw); cx++) {
#pragma unroll
        for (int dy = 0; dy < 2; dy++) {
            const int y = 2 * cy + dy;
            const unsigned a = sample_at(f.y, f.ypitch, 2 * cx + x0, y + y0, f);
            const unsigned c = sample_at(f.y, f.ypitch, 2 * cx + 1 + x0, y + y0, f);
            *(uint32_t *)(J.y16 + (size_t)y * J.w + 2 * cx) = (a << up) | ((c << up) << 16);
        }
        const int sx = (2 * cx + x0) / 2, sy = (2 * cy + y0) / 2;
        const unsigned u = f.semi ? sample_at(f.u, f.cpitch, 2 * sx, sy, f) : sample_at(f.u, f.cpitch, sx, sy, f);
        const unsigned v = f.semi ? sample_at(f.u, f.cpitch, 2 * sx + 1, sy, f) : sample_at(f.v, f.cpitch, sx, sy, f);
        J.u16[(size_t)cy * cw + cx] = (uint16_t)(u << up);
        J.v16[(size_t)cy * cw + cx] = (uint16_t)(v << up);
    }
}

constexpr int kM = 4;  // margin of a staged region: the 9 x 9 box reaches 4 pixels

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float exact_ratio(long long num, double den) { return __double2float_rn(__ddiv_rn((double)num, den)); }

__device__ __forceinline__ float oriented_of(long long jxx, long long jyy, long long jxy)
{
    const double d = (double)(jxx - jyy), x = (double)jxy;
    const double s = __dadd_rn(__dmul_rn(d, d), __dmul_rn(4.0, __dmul_rn(x, x)));
    return __double2float_rn(__ddiv_rn(__dsqrt_rn(s), 81.0));
}

// ---------------------------------------------------------------------------------------------------------------
// Window statistics of one source frame against every encode: src/kernels.cu:346-428, exact.
//
// A block of 256 threads takes a 64 x 64 tile (4 x 4 windows) of every picture in turn. Per picture: the 72 x 72 region
// (4-pixel margin, coordinates clamped) is staged in shared memory with 8-byte loads; each thread then builds the
// horizontal 3- and 9-sums of 8 columns of a region row from two 16-byte reads; then thread (c, g) walks tile column c
// down rows 16 g .. 16 g + 15 (one window's column) with running vertical sums, so the 3 x 3 and 9 x 9 sums of a pixel
// cost a few additions. The 16 lanes of a window reduce its sums with shuffles.
// ---------------------------------------------------------------------------------------------------------------
constexpr int kWT = 64;             // tile side
constexpr int kWR = kWT + 2 * kM;   // region side, 72
constexpr int kWS = 72;             // row stride of the region planes (144 bytes, a multiple of 16)

struct WinSmem {
    uint16_t y[kWR][kWS];   // y[r][j]: pixel (x0 - 4 + j, y0 - 4 + r), coordinates clamped
    uint16_t h3[kWR][kWS];  // h3[r][k]: 3-sum of row r centred at x0 - 1 + k, k < 66
    uint16_t h9[kWR][kWT];  // h9[r][c]: 9-sum of row r centred at x0 + c
};

// h3 and h9 of every region row: item (r, s) covers columns 8 s .. 8 s + 7 from y[r][8 s .. 8 s + 15].
__device__ __forceinline__ void window_horizontal_sums(WinSmem &sm)
{
    for (int i = threadIdx.x; i < kWR * 8; i += 256) {
        const int r = i >> 3, c0 = 8 * (i & 7);
        const uint4 a = *(const uint4 *)&sm.y[r][c0], b = *(const uint4 *)&sm.y[r][c0 + 8];
        const unsigned wv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        int v[16];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            v[2 * k] = (int)(wv[k] & 0xFFFFu);
            v[2 * k + 1] = (int)(wv[k] >> 16);
        }
        int s9 = 0;
#pragma unroll
        for (int k = 0; k < 9; k++) s9 += v[k];
        int h9[8], h3[10];
        h9[0] = s9;
#pragma unroll
        for (int k = 1; k < 8; k++) {
            s9 += v[k + 8] - v[k - 1];
            h9[k] = s9;
        }
#pragma unroll
        for (int k = 0; k < 10; k++) h3[k] = v[k + 2] + v[k + 3] + v[k + 4];
        *(uint4 *)&sm.h9[r][c0] = make_uint4(h9[0] | (h9[1] << 16), h9[2] | (h9[3] << 16), h9[4] | (h9[5] << 16), h9[6] | (h9[7] << 16));
        *(uint4 *)&sm.h3[r][c0] = make_uint4(h3[0] | (h3[1] << 16), h3[2] | (h3[3] << 16), h3[4] | (h3[5] << 16), h3[6] | (h3[7] << 16));
        if (c0 == 56) *(uint32_t *)&sm.h3[r][64] = h3[8] | (h3[9] << 16);
    }
}

template <typename T>
__device__ __forceinline__ T half_warp_sum(T v)
{
#pragma unroll
    for (int o = 8; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Dynamic shared memory: the region planes, then the source's fine and mid numerators of each thread's 16 rows, kept
// for the encodes' cross products (|fine| <= 9 x 1023 fits 16 bits) in shared memory so that three blocks fit an SM's
// registers, and two buffers of raw region values: the next picture's region is copied in (cp.async) while the
// current one is summed.
struct WinStatsSmem {
    WinSmem sm;
    int mr[kWin][256];
    int16_t fr[kWin][256];
    uint16_t raw[2][kWR][kWS];  // raw[b][r][j]: pixel (x0 - 4 + j, y0 - 4 + r) of a picture, coordinates clamped, unshifted
};

__device__ __forceinline__ void cp_async8(void *dst_smem, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst_smem)), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Queues the copy of `src`'s region at tile (x0, y0) into raw (unshifted; rows clamped): 8-byte asynchronous copies
// where the columns lie inside the picture and the rows are 8-byte aligned, else plain loads and stores now. Every
// thread commits one group of copies (possibly empty).
__device__ __forceinline__ void stage_raw_async(uint16_t (*raw)[kWS], const uint16_t *src, int w, int h, int x0, int y0)
{
    if (x0 >= kM && x0 + kWT + kM <= w && (w & 3) == 0 && ((uintptr_t)src & 7) == 0) {
        for (int i = threadIdx.x; i < kWR * 18; i += 256) {
            const int r = i / 18, q = i - r * 18;
            const int y = min(max(y0 - kM + r, 0), h - 1);
            cp_async8(&raw[r][4 * q], src + (size_t)y * w + (x0 - kM) + 4 * q);
        }
    } else {
        for (int i = threadIdx.x; i < kWR * kWR; i += 256) {
            const int r = i / kWR, j = i - r * kWR;
            const int x = min(max(x0 - kM + j, 0), w - 1), y = min(max(y0 - kM + r, 0), h - 1);
            raw[r][j] = src[(size_t)y * w + x];
        }
    }
    cp_async_commit();
}

// window_horizontal_sums over a raw buffer, the sums shifted left by `up` (the values at the pipeline's depth).
__device__ __forceinline__ void window_horizontal_sums_raw(WinSmem &sm, const uint16_t (*raw)[kWS], int up)
{
    for (int i = threadIdx.x; i < kWR * 8; i += 256) {
        const int r = i >> 3, c0 = 8 * (i & 7);
        const uint4 a = *(const uint4 *)&raw[r][c0], b = *(const uint4 *)&raw[r][c0 + 8];
        const unsigned wv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        int v[16];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            v[2 * k] = (int)(wv[k] & 0xFFFFu);
            v[2 * k + 1] = (int)(wv[k] >> 16);
        }
        int s9 = 0;
#pragma unroll
        for (int k = 0; k < 9; k++) s9 += v[k];
        int h9[8], h3[10];
        h9[0] = s9 << up;
#pragma unroll
        for (int k = 1; k < 8; k++) {
            s9 += v[k + 8] - v[k - 1];
            h9[k] = s9 << up;
        }
#pragma unroll
        for (int k = 0; k < 10; k++) h3[k] = (v[k + 2] + v[k + 3] + v[k + 4]) << up;
        *(uint4 *)&sm.h9[r][c0] = make_uint4(h9[0] | (h9[1] << 16), h9[2] | (h9[3] << 16), h9[4] | (h9[5] << 16), h9[6] | (h9[7] << 16));
        *(uint4 *)&sm.h3[r][c0] = make_uint4(h3[0] | (h3[1] << 16), h3[2] | (h3[3] << 16), h3[4] | (h3[5] << 16), h3[6] | (h3[7] << 16));
        if (c0 == 56) *(uint32_t *)&sm.h3[r][64] = h3[8] | (h3[9] << 16);
    }
}

__global__ void __launch_bounds__(256, 3) window_stats_kernel(const __grid_constant__ WindowBatch B)
{
    extern __shared__ __align__(16) unsigned char win_dyn[];
    WinStatsSmem &ws = *(WinStatsSmem *)win_dyn;
    WinSmem &sm = ws.sm;
    auto &fr_s = ws.fr;
    auto &mr_s = ws.mr;
    const int jb = find_job(B.njobs, (int)blockIdx.x, [&](int k) { return B.job[k].first_block; });
    const WindowJob &J = B.job[jb];
    const int bid = blockIdx.x - J.first_block;
    const int w = J.w, h = J.h, ww = w / kWin, wh = h / kWin;
    const int tiles_x = (ww + 3) / 4;
    const int x0 = (bid % tiles_x) * kWT, y0 = (bid / tiles_x) * kWT;
    const int tid = threadIdx.x, lane = tid & 31;
    const int c = tid & (kWT - 1), r0 = (tid >> 6) * kWin;  // tile column, first tile row
    const int wx = (x0 + c) / kWin, wy = (y0 + r0) / kWin;
    const bool inside = wx < ww && wy < wh;
    const int x = x0 + c;
    const bool gx_on = x > 0 && x < w - 1;
    unsigned long long src_f = 0, src_m = 0, src_xx = 0, src_yy = 0;
    long long src_xy = 0;
    const int up = J.up;
    stage_raw_async(ws.raw[0], J.yr, w, h, x0, y0);
    for (int p = 0; p <= J.nenc; p++) {
        const uint16_t(*raw)[kWS] = ws.raw[p & 1];
        __syncthreads();  // the walk of picture p - 1 is done with the buffer picture p + 1 goes to
        if (p < J.nenc) {
            stage_raw_async(ws.raw[(p + 1) & 1], J.yd[p], w, h, x0, y0);
            cp_async_wait<1>();  // picture p's copies are in; p + 1's may still be in flight
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        window_horizontal_sums_raw(sm, raw, up);
        __syncthreads();
        // tile row t is region row t + 4; h3 column c + 1 is centred at x, c and c + 2 at x -+ 1
        auto h3c = [&](int t) { return (int)sm.h3[t + kM][c + 1]; };
        auto h3l = [&](int t) { return (int)sm.h3[t + kM][c]; };
        auto h3r = [&](int t) { return (int)sm.h3[t + kM][c + 2]; };
        auto h9c = [&](int t) { return (int)sm.h9[t + kM][c]; };
        int s3_prev = h3c(r0 - 2) + h3c(r0 - 1) + h3c(r0);      // S3 at row r0 - 1
        int s3 = s3_prev - h3c(r0 - 2) + h3c(r0 + 1);            // S3 at row r0
        int s3l = h3l(r0 - 1) + h3l(r0) + h3l(r0 + 1), s3r = h3r(r0 - 1) + h3r(r0) + h3r(r0 + 1);
        int s9 = 0;
#pragma unroll
        for (int k = -4; k <= 4; k++) s9 += h9c(r0 + k);
        unsigned fine_sq = 0, jxx = 0, jyy = 0;
        int jxy = 0, fine_x = 0;
        unsigned long long mid_sq = 0;
        long long mid_x = 0;
#pragma unroll
        for (int i = 0; i < kWin; i++) {
            const int t = r0 + i, y = y0 + t;
            const int s3_next = s3 - h3c(t - 1) + h3c(t + 2);
            const int f = 9 * ((int)raw[t + kM][c + kM] << up) - s3, m = 9 * s3 - s9;
            const int gx = gx_on ? s3r - s3l : 0;
            const int gy = (y > 0 && y < h - 1) ? s3_next - s3_prev : 0;
            if (p == 0) {
                fr_s[i][tid] = (int16_t)f;
                mr_s[i][tid] = m;
            } else {
                fine_x += f * (int)fr_s[i][tid];
                mid_x += (long long)m * mr_s[i][tid];
            }
            fine_sq += (unsigned)(f * f);
            mid_sq += (unsigned long long)((long long)m * m);
            jxx += (unsigned)(gx * gx);
            jyy += (unsigned)(gy * gy);
            jxy += gx * gy;
            if (i + 1 < kWin) {
                s3_prev = s3;
                s3 = s3_next;
                s3l += h3l(t + 2) - h3l(t - 1);
                s3r += h3r(t + 2) - h3r(t - 1);
                s9 += h9c(t + 5) - h9c(t - 4);
            }
        }
        const unsigned long long sf = half_warp_sum((unsigned long long)fine_sq), sm2 = half_warp_sum(mid_sq),
                                 sxx = half_warp_sum((unsigned long long)jxx), syy = half_warp_sum((unsigned long long)jyy);
        const long long sxy = half_warp_sum((long long)jxy);
        if (p == 0) {
            src_f = sf; src_m = sm2; src_xx = sxx; src_yy = syy; src_xy = sxy;
            continue;
        }
        const long long cf = half_warp_sum((long long)fine_x), cm = half_warp_sum(mid_x);
        if (inside && (lane & 15) == 0) {
            float *o = J.stats[p - 1] + ((size_t)wy * ww + wx) * 8;
            o[0] = exact_ratio((long long)src_f, 81.0);
            o[1] = exact_ratio((long long)src_m, 6561.0);
            o[2] = exact_ratio((long long)sf, 81.0);
            o[3] = exact_ratio((long long)sm2, 6561.0);
            o[4] = exact_ratio(cf, 81.0);
            o[5] = exact_ratio(cm, 6561.0);
            o[6] = oriented_of((long long)src_xx, (long long)src_yy, src_xy);
            o[7] = oriented_of((long long)sxx, (long long)syy, sxy);
        }
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Lasting texture: src/kernels.cu:435-451, exact, from running luma sums (see PersistJob).
//
// A block of 256 threads takes a 64 x 64 tile (4 x 4 windows): it advances the running sums E and O over the tile and
// its 4-pixel margin (coordinates clamped, so the margins repeat the edges) and writes them for the tile's own pixels;
// then, as in window_stats, the horizontal 3- and 9-sums of E, of O and of each picture are built in shared memory and
// thread (c, g) walks tile column c down window row g with running vertical sums of the mid-detail numerators.
// ---------------------------------------------------------------------------------------------------------------
// mid-detail numerators 9 S3 - S9 of the 16 rows from tile row r0 at tile column c, from the horizontal sums
__device__ __forceinline__ void window_mids(const WinSmem &sm, int c, int r0, int (&m)[kWin])
{
    auto h3c = [&](int t) { return (int)sm.h3[t + kM][c + 1]; };
    auto h9c = [&](int t) { return (int)sm.h9[t + kM][c]; };
    int s3 = h3c(r0 - 1) + h3c(r0) + h3c(r0 + 1);
    int s9 = 0;
#pragma unroll
    for (int k = -4; k <= 4; k++) s9 += h9c(r0 + k);
#pragma unroll
    for (int i = 0; i < kWin; i++) {
        const int t = r0 + i;
        m[i] = 9 * s3 - s9;
        if (i + 1 < kWin) {
            s3 += h3c(t + 2) - h3c(t - 1);
            s9 += h9c(t + 5) - h9c(t - 4);
        }
    }
}

// Dynamic shared memory of persist_kernel: the region planes, the odd running sums of the region, and two buffers of
// raw picture regions (the pictures' regions are copied in asynchronously, the first one while the sums advance).
struct PersistSmem {
    WinSmem sm;
    uint16_t o_reg[kWR][kWS];
    uint16_t raw[2][kWR][kWS];
};

__global__ void __launch_bounds__(256, 3) persist_kernel(const __grid_constant__ PersistBatch B)
{
    extern __shared__ __align__(16) unsigned char persist_dyn[];
    PersistSmem &ps = *(PersistSmem *)persist_dyn;
    WinSmem &sm = ps.sm;
    auto &o_reg = ps.o_reg;
    const int jb = find_job(B.njobs, (int)blockIdx.x, [&](int k) { return B.job[k].first_block; });
    const PersistJob &J = B.job[jb];
    const int bid = blockIdx.x - J.first_block;
    const int w = J.w, h = J.h, ww = w / kWin, wh = h / kWin;
    const int tiles_x = (w + kWT - 1) / kWT;
    const int x0 = (bid % tiles_x) * kWT, y0 = (bid / tiles_x) * kWT;
    const int tid = threadIdx.x, lane = tid & 31;
    if (J.stats) stage_raw_async(ps.raw[0], J.y_c, w, h, x0, y0);  // the centre frame's region, while the sums advance
    // advance the running sums over the region: E(c) = O(c-1) - y(c) + y(c+6), O(c) = E(c-1) - y(c-7) + y(c-1)
    const uint16_t *pl[4] = {J.y_m13, J.y_m7, J.y_c, J.y_f};
    uintptr_t align = (uintptr_t)J.e_old | (uintptr_t)J.o_old | (uintptr_t)J.e_new | (uintptr_t)J.o_new;
    for (int k = 0; k < 4; k++) align |= (uintptr_t)pl[k];
    if (x0 >= kM && x0 + kWT + kM <= w && (w & 3) == 0 && (align & 7) == 0) {
        // interior columns: 18 groups of 4 pixels per region row, packed 16-bit arithmetic (no element leaves 0..65535)
        for (int i = tid; i < kWR * 18; i += 256) {
            const int r = i / 18, q = i - r * 18, yu = y0 - kM + r, y = min(max(yu, 0), h - 1);
            const size_t k = (size_t)y * w + (x0 - kM) + 4 * q;
            uint2 v[4];
#pragma unroll
            for (int n = 0; n < 4; n++) {
                v[n] = pl[n] ? __ldg((const uint2 *)(pl[n] + k)) : make_uint2(0, 0);
                v[n].x <<= J.up;
                v[n].y <<= J.up;
            }
            const uint2 oo = __ldg((const uint2 *)(J.o_old + k)), eo = __ldg((const uint2 *)(J.e_old + k));
            // no element leaves 0 .. 65535 (the leaving frame is part of the old sum), so 32-bit arithmetic on the
            // pairs carries and borrows nothing between the halves
            const uint2 e = make_uint2(oo.x - v[2].x + v[3].x, oo.y - v[2].y + v[3].y);
            const uint2 o = make_uint2(eo.x - v[0].x + v[1].x, eo.y - v[0].y + v[1].y);
            *(uint2 *)&sm.y[r][4 * q] = e;
            *(uint2 *)&o_reg[r][4 * q] = o;
            if (r >= kM && r < kM + kWT && yu < h && q >= 1 && q <= 16) {
                *(uint2 *)(J.e_new + k) = e;
                *(uint2 *)(J.o_new + k) = o;
            }
        }
    } else {
        for (int i = tid; i < kWR * kWR; i += 256) {
            const int r = i / kWR, cc = i - r * kWR;
            const int xi = x0 - kM + cc, yi = y0 - kM + r;
            const int x = min(max(xi, 0), w - 1), y = min(max(yi, 0), h - 1);
            const size_t k = (size_t)y * w + x;
            int yv[4];
#pragma unroll
            for (int n = 0; n < 4; n++) yv[n] = pl[n] ? (int)(pl[n][k] << J.up) : 0;
            const int e = (int)J.o_old[k] - yv[2] + yv[3];
            const int o = (int)J.e_old[k] - yv[0] + yv[1];
            sm.y[r][cc] = (uint16_t)e;
            o_reg[r][cc] = (uint16_t)o;
            if (xi >= x0 && xi < x0 + kWT && yi >= y0 && yi < y0 + kWT && xi < w && yi < h) {
                J.e_new[k] = (uint16_t)e;
                J.o_new[k] = (uint16_t)o;
            }
        }
    }
    if (!J.stats) return;
    const int c = tid & (kWT - 1), r0 = (tid >> 6) * kWin;
    const int wx = (x0 + c) / kWin, wy = (y0 + r0) / kWin;
    const bool inside = wx < ww && wy < wh;
    int a[kWin], bb[kWin], t[kWin];
    __syncthreads();
    window_horizontal_sums(sm);
    __syncthreads();
    window_mids(sm, c, r0, a);  // A x 486 = mid x 81 of E
    __syncthreads();
    for (int i = tid; i < kWR * kWS / 8; i += 256) ((uint4 *)&sm.y[0][0])[i] = ((const uint4 *)&o_reg[0][0])[i];
    __syncthreads();
    window_horizontal_sums(sm);
    __syncthreads();
    window_mids(sm, c, r0, bb);  // B x 486
    long long sab = 0, saa = 0, sbb = 0;
#pragma unroll
    for (int i = 0; i < kWin; i++) {
        t[i] = a[i] + bb[i];  // T x 972
        sab += (long long)a[i] * bb[i];
        saa += (long long)a[i] * a[i];
        sbb += (long long)bb[i] * bb[i];
    }
    sab = half_warp_sum(sab);
    saa = half_warp_sum(saa);
    sbb = half_warp_sum(sbb);
    long long own = 0;
    for (int p = 0; p <= J.nenc; p++) {
        __syncthreads();  // picture p - 1's sums are read, and its buffer is the one picture p + 1 goes to
        if (p < J.nenc) {
            stage_raw_async(ps.raw[(p + 1) & 1], J.yd[p], w, h, x0, y0);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        window_horizontal_sums_raw(sm, ps.raw[p & 1], J.up);
        __syncthreads();
        int m[kWin];
        window_mids(sm, c, r0, m);
        long long sp = 0;
#pragma unroll
        for (int i = 0; i < kWin; i++) sp += (long long)m[i] * t[i];
        sp = half_warp_sum(sp);
        if (p == 0) {
            own = sp;
            continue;
        }
        if (inside && (lane & 15) == 0) {
            float *o = J.out[p - 1] + ((size_t)wy * ww + wx) * 5;
            o[0] = exact_ratio(own, 78732.0);
            o[1] = exact_ratio(sp, 78732.0);
            o[2] = exact_ratio(sab, 236196.0);
            o[3] = exact_ratio(saa, 236196.0);
            o[4] = exact_ratio(sbb, 236196.0);
        }
    }
}

// ---------------------------------------------------------------------------------------------------------------
// PSNR squared errors (src/kernels.cu:454-464) and color sums (470-484), exact integers; the color strength of each
// sample sqrt(du^2 + dv^2) is rounded to units of 2^-30 so its sum is exact too. blockIdx.y picks the picture:
// 0 .. nenc-1 the encodes (squared errors against the source, and their colors), nenc the source's colors.
// ---------------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) pair_sums_kernel(const __grid_constant__ PairSumsBatch B)
{
    int jb = 0;
    while (jb + 1 < B.njobs && (int)blockIdx.y >= B.job[jb + 1].first_pic) jb++;
    const PairSumsJob &J = B.job[jb];
    const int p = blockIdx.y - J.first_pic;
    const bool src_only = p == J.nenc;
    const size_t n = (size_t)J.w * J.h, cn = n / 4;
    const size_t stride = (size_t)gridDim.x * 256, i0 = (size_t)blockIdx.x * 256 + threadIdx.x;
    unsigned long long sy = 0, su = 0, sv = 0, cu = 0, cv = 0, cs = 0;
    // 8 samples per 16-byte load (the planes are allocated aligned); the remainder one at a time
    auto sq = [](unsigned a, unsigned b) -> unsigned {  // squared differences of two pairs of 16-bit samples
        const int d0 = (int)(a & 0xFFFFu) - (int)(b & 0xFFFFu), d1 = (int)(a >> 16) - (int)(b >> 16);
        return (unsigned)(d0 * d0 + d1 * d1);
    };
    if (!src_only) {
        const uint16_t *a = J.ry, *b = J.dy[p];
        const size_t nv = (((uintptr_t)a | (uintptr_t)b) & 15) ? 0 : n / 8;
#pragma unroll 4
        for (size_t i = i0; i < nv; i += stride) {
            const uint4 x = __ldg((const uint4 *)a + i), y = __ldg((const uint4 *)b + i);
            sy += sq(x.x, y.x) + sq(x.y, y.y) + sq(x.z, y.z) + sq(x.w, y.w);
        }
        for (size_t i = nv * 8 + i0; i < n; i += stride) {
            const long long d = (long long)a[i] - (long long)b[i];
            sy += (unsigned long long)(d * d);
        }
    }
    const uint16_t *u = src_only ? J.ru : J.du[p], *v = src_only ? J.rv : J.dv[p];
    auto color = [&](unsigned uu, unsigned vv) {
        uu <<= J.up;
        vv <<= J.up;
        const int eu = (int)uu - 512, ev = (int)vv - 512;
        cu += uu;
        cv += vv;
        cs += (unsigned long long)__double2ll_rn(__dmul_rn(__dsqrt_rn((double)(eu * eu + ev * ev)), 1073741824.0));
    };
    const size_t cnv = (((uintptr_t)u | (uintptr_t)v | (uintptr_t)J.ru | (uintptr_t)J.rv) & 15) ? 0 : cn / 8;
#pragma unroll 2
    for (size_t i = i0; i < cnv; i += stride) {
        const uint4 uq = __ldg((const uint4 *)u + i), vq = __ldg((const uint4 *)v + i);
        if (!src_only) {
            const uint4 ru = __ldg((const uint4 *)J.ru + i), rv = __ldg((const uint4 *)J.rv + i);
            su += sq(ru.x, uq.x) + sq(ru.y, uq.y) + sq(ru.z, uq.z) + sq(ru.w, uq.w);
            sv += sq(rv.x, vq.x) + sq(rv.y, vq.y) + sq(rv.z, vq.z) + sq(rv.w, vq.w);
        }
        const unsigned us[4] = {uq.x, uq.y, uq.z, uq.w}, vs[4] = {vq.x, vq.y, vq.z, vq.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            color(us[k] & 0xFFFFu, vs[k] & 0xFFFFu);
            color(us[k] >> 16, vs[k] >> 16);
        }
    }
    for (size_t i = cnv * 8 + i0; i < cn; i += stride) {
        if (!src_only) {
            const long long du = (long long)J.ru[i] - (long long)u[i], dv = (long long)J.rv[i] - (long long)v[i];
            su += (unsigned long long)(du * du);
            sv += (unsigned long long)(dv * dv);
        }
        color(u[i], v[i]);
    }
    sy = warp_sum(sy); su = warp_sum(su); sv = warp_sum(sv);
    cu = warp_sum(cu); cv = warp_sum(cv); cs = warp_sum(cs);
    if ((threadIdx.x & 31) == 0) {
        if (!src_only) {
            atomicAdd(&J.sse[p * 3 + 0], sy);
            atomicAdd(&J.sse[p * 3 + 1], su);
            atomicAdd(&J.sse[p * 3 + 2], sv);
        }
        atomicAdd(&J.color[p * 3 + 0], cu);
        atomicAdd(&J.color[p * 3 + 1], cv);
        atomicAdd(&J.color[p * 3 + 2], cs);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Per-frame reduction, src/main.cpp:606-641 with quantile() of 280-289 and Histogram::add's binning of
// src/stats.hpp:14-19, in three launches: (1) the structure threshold, an exact order statistic of the source's
// oriented figures by a 3-round radix select, and the frame's structure mask; (2) every window of every encode: its
// bins and the block's sums, added in a fixed order; (3) per encode the blocks' sums, in a fixed order -- so the
// figures are the same on every run.
// ---------------------------------------------------------------------------------------------------------------
constexpr int kCT = 1024;  // threshold block
constexpr int kCW = 256;   // windows per block
constexpr int kThreshStage = 40960;  // oriented figures a threshold block stages in shared memory (160 KB)
__host__ __device__ inline int collect_blocks_dev(int windows) { return (windows + kCW - 1) / kCW; }

__device__ __forceinline__ uint16_t hist_bin(double pct)
{
    const double c = pct < -500.0 ? -500.0 : pct > 500.0 ? 500.0 : pct;
    return (uint16_t)llround(__ddiv_rn(__dadd_rn(c, 500.0), 0.05));
}

// The rank-th smallest (0-based) of the non-negative floats v[i * stride] (their bit patterns order as the values), by
// three radix rounds of 11, 11 and 10 bits; each warp adds the lanes that share a digit with one atomic.
__device__ unsigned select_kth(const float *v, int n, int stride, unsigned rank, unsigned *hist)
{
    __shared__ unsigned s_prefix, s_mask, s_rem;
    __shared__ unsigned warp_tot[kCT / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) { s_prefix = 0; s_mask = 0; s_rem = rank; }
    for (int round = 0; round < 3; round++) {
        const int shift = round == 0 ? 21 : round == 1 ? 10 : 0, nb = round == 2 ? 1024 : 2048;
        for (int i = tid; i < 2048; i += kCT) hist[i] = 0;
        __syncthreads();
        const unsigned prefix = s_prefix, mask = s_mask;
        for (int i0 = tid - lane; i0 < n; i0 += kCT) {  // the same trip count for every lane of a warp
            const int i = i0 + lane;
            const unsigned bits = i < n ? __float_as_uint(v[(size_t)i * stride]) : 0u;
            const bool in = i < n && (bits & mask) == prefix;
            if (!__any_sync(0xffffffffu, in)) continue;  // after the first round most warps hold no candidate
            const unsigned d = in ? (bits >> shift) & (unsigned)(nb - 1) : 0xFFFFFFFFu;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (in && lane == __ffs(peers) - 1) atomicAdd(&hist[d], (unsigned)__popc(peers));
        }
        __syncthreads();
        // the digit holding the rem-th smallest: thread t sums digits [t per, t per + per), a block scan places it
        const int per = nb / kCT;
        unsigned local = 0;
        for (int k = 0; k < per; k++) local += hist[tid * per + k];
        unsigned incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v2 = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v2;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        unsigned before = 0;
        for (int k = 0; k < warp; k++) before += warp_tot[k];
        incl += before;
        const unsigned rem = s_rem, excl = incl - local;
        __syncthreads();
        if (excl <= rem && rem < incl) {
            unsigned below = excl;
            int d = tid * per;
            while (below + hist[d] <= rem) below += hist[d++];
            s_rem = rem - below;
            s_prefix = prefix | ((unsigned)d << shift);
            s_mask = mask | ((unsigned)(nb - 1) << shift);
        }
        __syncthreads();
    }
    return s_prefix;
}

// The (rank + 1)-th smallest of the same floats, given bits a of the rank-th: a again when more than rank + 1 values
// are at most a, otherwise the least value above a (one pass instead of three radix rounds).
__device__ unsigned select_next(const float *v, int n, int stride, unsigned rank, unsigned a)
{
    __shared__ unsigned s_le, s_min;
    if (threadIdx.x == 0) { s_le = 0; s_min = 0xFFFFFFFFu; }
    __syncthreads();
    unsigned le = 0, mn = 0xFFFFFFFFu;
    for (int i = threadIdx.x; i < n; i += kCT) {
        const unsigned bits = __float_as_uint(v[(size_t)i * stride]);
        if (bits <= a) le++;
        else mn = min(mn, bits);
    }
    le = __reduce_add_sync(0xffffffffu, le);
    mn = __reduce_min_sync(0xffffffffu, mn);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_le, le);
        atomicMin(&s_min, mn);
    }
    __syncthreads();
    return s_le >= rank + 2 ? a : s_min;
}

// One block per source. With `staged` (every job has at most kThreshStage windows) the oriented figures, which sit
// 8 floats apart in the figure array, are first gathered into dynamic shared memory, so the radix rounds and the
// mask read them there.
__global__ void __launch_bounds__(kCT) collect_threshold_kernel(const __grid_constant__ CollectBatch B, int staged)
{
    __shared__ unsigned hist[2048];
    extern __shared__ float stage[];
    const CollectJob &J = B.job[blockIdx.x];
    const float *st = J.stats[0];  // the source's oriented figures are the same in every encode's array
    const int n = J.windows;
    const float *v = st + 6;
    int stride = 8;
    if (staged) {
#pragma unroll 8
        for (int i = threadIdx.x; i < n; i += kCT) stage[i] = __ldg(st + (size_t)i * 8 + 6);
        __syncthreads();
        v = stage;
        stride = 1;
    }
    // numpy's linear quantile at 0.8 of exact order statistics, in the reference's float / double arithmetic
    const double pos = 0.8 * (double)(n - 1);
    const unsigned lo = (unsigned)pos;
    const unsigned a_bits = select_kth(v, n, stride, lo, hist);
    const float a = __uint_as_float(a_bits);
    float q = a;
    if (lo + 1 < (unsigned)n) {
        const float b = __uint_as_float(select_next(v, n, stride, lo, a_bits));
        const float diff = __fsub_rn(b, a);
        q = __double2float_rn(__dadd_rn((double)a, __dmul_rn((double)diff, __dsub_rn(pos, (double)lo))));
    }
    if (threadIdx.x == 0) *J.threshold = q;
    for (int i = threadIdx.x; i < n; i += kCT) {
        const float o = v[(size_t)i * stride];
        J.mask[i] = o >= q && o > 0.0f;
    }
}

__global__ void __launch_bounds__(kCW) collect_windows_kernel(const __grid_constant__ CollectBatch B)
{
    __shared__ double part[kCW / 32][kCollectSums];
    int jb = 0;
    while (jb + 1 < B.njobs && (int)blockIdx.y >= B.job[jb + 1].first_enc) jb++;
    const CollectJob &J = B.job[jb];
    const int nb = collect_blocks_dev(J.windows);
    if ((int)blockIdx.x >= nb) return;  // the grid covers the job with the most windows
    const int e = blockIdx.y - J.first_enc, n = J.windows, i = blockIdx.x * kCW + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // sums: all_r[3] all_d[3] st_r[3] st_d[3] sh_all_x[2] sh_st_x[2] own mine n_structure n_lasting
    double v[kCollectSums];
#pragma unroll
    for (int k = 0; k < kCollectSums; k++) v[k] = 0.0;
    uint16_t bin[6];  // amount 0-2, matching 0-1 (valid on structure windows), lasting (valid where v[19] is 1)
    bool structure = false, lasting = false;
    if (i < n) {
        const float q = *J.threshold;
        const float *s = J.stats[e] + (size_t)i * 8;
        const bool m = s[6] >= q && s[6] > 0.0f;
        structure = m;
        const double er[3] = {(double)s[0], (double)s[1], (double)s[6]}, ed[3] = {(double)s[2], (double)s[3], (double)s[7]};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            v[k] = er[k];
            v[3 + k] = ed[k];
            if (m) {
                v[6 + k] = er[k];
                v[9 + k] = ed[k];
                bin[k] = hist_bin(__dmul_rn(100.0, __dsqrt_rn(__ddiv_rn(ed[k], fmax(er[k], 1e-9)))));
            }
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const double x = (double)s[4 + k];
            v[12 + k] = x;
            if (m) {
                v[14 + k] = x;
                bin[3 + k] = hist_bin(__ddiv_rn(__dmul_rn(100.0, x), fmax(er[k], 1e-9)));
            }
        }
        v[18] = m ? 1.0 : 0.0;
        if (J.persist[e]) {
            const float *ps = J.persist[e] + (size_t)i * 5;
            const double agree = __ddiv_rn((double)ps[2], __dsqrt_rn(fmax(__dmul_rn((double)ps[3], (double)ps[4]), 1e-9)));
            if (J.centre_mask[i] && agree > 0.5 && ps[0] > 0.0f) {
                v[16] = (double)ps[0];
                v[17] = (double)ps[1];
                v[19] = 1.0;
                lasting = true;
                bin[5] = hist_bin(__ddiv_rn(__dmul_rn(100.0, (double)ps[1]), (double)ps[0]));
            }
        }
    }
    // the bins that count, compacted (a histogram does not depend on their order): the five structure arrays share
    // one position per window, the lasting array has its own; a warp reserves its places with one atomic each
    {
        uint16_t *bins = J.bins[e];
        const unsigned below = (1u << lane) - 1u;
        const unsigned sm = __ballot_sync(0xffffffffu, structure), lm = __ballot_sync(0xffffffffu, lasting);
        unsigned sb = 0, lb = 0;
        if (sm && lane == 0) sb = atomicAdd(&J.bin_n[e][0], (unsigned)__popc(sm));
        if (lm && lane == 0) lb = atomicAdd(&J.bin_n[e][1], (unsigned)__popc(lm));
        sb = __shfl_sync(0xffffffffu, sb, 0);
        lb = __shfl_sync(0xffffffffu, lb, 0);
        if (structure) {
            const unsigned at = sb + __popc(sm & below);
#pragma unroll
            for (int k = 0; k < 5; k++) bins[(size_t)k * n + at] = bin[k];
        }
        if (lasting) bins[(size_t)5 * n + lb + __popc(lm & below)] = bin[5];
    }
#pragma unroll
    for (int k = 0; k < kCollectSums; k++) {
        const double x = warp_sum(v[k]);
        if (lane == 0) part[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < kCollectSums) {
        double s = 0.0;
        for (int k = 0; k < kCW / 32; k++) s += part[k][threadIdx.x];
        J.partials[((size_t)e * nb + blockIdx.x) * kCollectSums + threadIdx.x] = s;
    }
}

// Warp k of an encode's block makes sum k: lane l adds the partials of blocks l, l + 32, ... in order, then a fixed
// shuffle tree adds the 32 lane sums (the same order on every run).
__global__ void __launch_bounds__(32 * kCollectSums) collect_final_kernel(const __grid_constant__ CollectBatch B)
{
    int jb = 0;
    while (jb + 1 < B.njobs && (int)blockIdx.x >= B.job[jb + 1].first_enc) jb++;
    const CollectJob &J = B.job[jb];
    const int e = blockIdx.x - J.first_enc, k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nblocks = collect_blocks_dev(J.windows);
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += J.partials[((size_t)e * nblocks + b) * kCollectSums + k];
    s = warp_sum(s);
    if (lane != 0) return;
    FrameFigures *f = J.fig[e];
    if (k < 3) f->all_r[k] = s;
    else if (k < 6) f->all_d[k - 3] = s;
    else if (k < 9) f->st_r[k - 6] = s;
    else if (k < 12) f->st_d[k - 9] = s;
    else if (k < 14) f->sh_all_x[k - 12] = s;
    else if (k < 16) f->sh_st_x[k - 14] = s;
    else if (k == 16) f->own = s;
    else if (k == 17) f->mine = s;
    else if (k == 18) f->n_structure = (unsigned)s;
    else f->n_lasting = (unsigned)s;
    if (k == 0) f->threshold = *J.threshold;
}

}  // namespace

cudaError_t launch_unpack(const UnpackBatch &b, cudaStream_t s)
{
    if (b.total_blocks <= 0) return cudaSuccess;
    LaunchTimer t("frame_unpack", s);
    unpack_kernel<<<b.total_blocks, 256, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_window_stats(WindowBatch &b, cudaStream_t s)
{
    int blocks = 0;
    for (int j = 0; j < b.njobs; j++) {
        WindowJob &J = b.job[j];
        J.first_block = blocks;
        const int ww = J.w / kWin, wh = J.h / kWin;
        if (ww > 0 && wh > 0 && J.nenc > 0) blocks += ((ww + 3) / 4) * ((wh + 3) / 4);
    }
    if (blocks == 0) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(window_stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sizeof(WinStatsSmem));
    if (e != cudaSuccess) return e;
    LaunchTimer t("window_stats", s);
    window_stats_kernel<<<blocks, 256, sizeof(WinStatsSmem), s>>>(b);
    return after_launch();
}

cudaError_t launch_persist(PersistBatch &b, cudaStream_t s)
{
    int blocks = 0;
    for (int j = 0; j < b.njobs; j++) {
        PersistJob &J = b.job[j];
        J.first_block = blocks;
        blocks += ((J.w + kWT - 1) / kWT) * ((J.h + kWT - 1) / kWT);
    }
    if (blocks == 0) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(PersistSmem));
    if (e != cudaSuccess) return e;
    LaunchTimer t("persist_stats", s);
    persist_kernel<<<blocks, 256, sizeof(PersistSmem), s>>>(b);
    return after_launch();
}

cudaError_t launch_pair_sums(PairSumsBatch &b, cudaStream_t s)
{
    int pics = 0;
    for (int j = 0; j < b.njobs; j++) {
        b.job[j].first_pic = pics;
        pics += b.job[j].nenc + 1;
    }
    if (pics == 0) return cudaSuccess;
    LaunchTimer t("pair_sums", s);
    pair_sums_kernel<<<dim3(pics <= 4 ? 148 : 64, pics), 256, 0, s>>>(b);
    return after_launch();
}

int collect_blocks(int windows) { return collect_blocks_dev(windows); }

// Grid rows of each job's encodes, and the most collect blocks of a job; an error for a job without encodes or windows.
static cudaError_t collect_shape(CollectBatch &b, int &encs, int &nb, int &max_windows)
{
    encs = nb = max_windows = 0;
    for (int j = 0; j < b.njobs; j++) {
        if (b.job[j].nenc <= 0 || b.job[j].windows <= 0) return cudaErrorInvalidValue;
        b.job[j].first_enc = encs;
        encs += b.job[j].nenc;
        nb = nb > collect_blocks(b.job[j].windows) ? nb : collect_blocks(b.job[j].windows);
        max_windows = max_windows > b.job[j].windows ? max_windows : b.job[j].windows;
    }
    return cudaSuccess;
}

cudaError_t launch_collect_threshold(CollectBatch &b, cudaStream_t s)
{
    int encs, nb, max_windows;
    cudaError_t e = collect_shape(b, encs, nb, max_windows);
    if (e != cudaSuccess || encs == 0) return e;
    const int staged = max_windows <= kThreshStage;
    e = cudaFuncSetAttribute(collect_threshold_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kThreshStage * (int)sizeof(float));
    if (e != cudaSuccess) return e;
    LaunchTimer t("frame_collect_threshold", s);
    collect_threshold_kernel<<<b.njobs, kCT, staged ? (size_t)max_windows * sizeof(float) : 0, s>>>(b, staged);
    return after_launch();
}

cudaError_t launch_collect_sums(CollectBatch &b, cudaStream_t s)
{
    int encs, nb, max_windows;
    cudaError_t e = collect_shape(b, encs, nb, max_windows);
    if (e != cudaSuccess || encs == 0) return e;
    {
        LaunchTimer t("frame_collect_windows", s);
        collect_windows_kernel<<<dim3(nb, encs), kCW, 0, s>>>(b);
    }
    e = after_launch();
    if (e != cudaSuccess) return e;
    LaunchTimer t("frame_collect_final", s);
    collect_final_kernel<<<encs, 32 * kCollectSums, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_collect(CollectBatch &b, cudaStream_t s)
{
    const cudaError_t e = launch_collect_threshold(b, s);
    return e != cudaSuccess ? e : launch_collect_sums(b, s);
}

// ---------------------------------------------------------------------------------------------------------------
// The VMAF picture feed: src/kernels.cu:537-545 (to_picture), one launch for every plane of a step. A thread moves 8
// samples of a row: one 16-byte load of the 16-bit values, and one 8-byte (8-bit picture) or 16-byte store where the
// destination row allows, else sample by sample. An 8-bit picture keeps the low byte of each value, as the reference.
// ---------------------------------------------------------------------------------------------------------------
namespace {
constexpr int kPicThreads = 256;

__global__ void __launch_bounds__(kPicThreads) to_pictures_kernel(const __grid_constant__ PictureBatch b)
{
    const int j = find_job(b.njobs, (int)blockIdx.x, [&](int k) { return b.job[k].first_block; });
    const PictureJob &J = b.job[j];
    const int groups = (J.w + 7) / 8;  // 8-sample groups per row
    const long long i = (long long)(blockIdx.x - J.first_block) * kPicThreads + threadIdx.x;
    if (i >= (long long)groups * J.h) return;
    const int y = (int)(i / groups), x = (int)(i - (long long)y * groups) * 8;
    const uint16_t *src = J.src + (size_t)y * J.w + x;
    char *row = (char *)J.dst + (size_t)y * J.pitch;
    const bool src_vec = (J.w & 7) == 0 && (((uintptr_t)J.src) & 15) == 0;
    if (src_vec && x + 8 <= J.w) {
        const uint4 q = __ldg((const uint4 *)src);
        if (J.bytes == 1) {
            uint8_t *d = (uint8_t *)row + x;
            const uint2 v = make_uint2(__byte_perm(q.x, q.y, 0x6420), __byte_perm(q.z, q.w, 0x6420));
            if ((((uintptr_t)d) & 7) == 0) {
                *(uint2 *)d = v;
            } else {
                for (int k = 0; k < 4; k++) d[k] = (uint8_t)(v.x >> (8 * k));
                for (int k = 0; k < 4; k++) d[4 + k] = (uint8_t)(v.y >> (8 * k));
            }
        } else {
            uint16_t *d = (uint16_t *)row + x;
            if ((((uintptr_t)d) & 15) == 0) {
                *(uint4 *)d = q;
            } else {
                const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
                for (int k = 0; k < 8; k++) d[k] = (uint16_t)(w4[k >> 1] >> (16 * (k & 1)));
            }
        }
        return;
    }
    for (int k = 0; k < 8 && x + k < J.w; k++) {
        const uint16_t v = src[k];
        if (J.bytes == 1) ((uint8_t *)row)[x + k] = (uint8_t)v;
        else ((uint16_t *)row)[x + k] = v;
    }
}

}  // namespace

cudaError_t launch_to_pictures(PictureBatch &b, cudaStream_t s)
{
    int blocks = 0;
    for (int j = 0; j < b.njobs; j++) {
        PictureJob &J = b.job[j];
        J.first_block = blocks;
        blocks += (int)(((long long)((J.w + 7) / 8) * J.h + kPicThreads - 1) / kPicThreads);
    }
    if (blocks <= 0) return cudaSuccess;
    LaunchTimer t("to_pictures", s);
    to_pictures_kernel<<<blocks, kPicThreads, 0, s>>>(b);
    return after_launch();
}

const void *kernel_entry_unpack() { return (const void *)unpack_kernel; }
const void *kernel_entry_window_stats() { return (const void *)window_stats_kernel; }
const void *kernel_entry_persist() { return (const void *)persist_kernel; }
const void *kernel_entry_pair_sums() { return (const void *)pair_sums_kernel; }
const void *kernel_entry_collect() { return (const void *)collect_windows_kernel; }

}  // namespace es
