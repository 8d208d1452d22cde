// Temporal alignment kernels for sm_100a: the thumbnails a source and its encodes are matched by, and the per-lag
// difference totals of the offset search.
//
// The reference (src/kernels.cu:502-520, src/main.cpp:301-353) launches tiny_luma once per decoded frame, copies
// each 64 x 36 thumbnail to the host with a stream synchronisation, and searches the lags on the CPU. Here one launch
// makes the thumbnails of a whole batch of frames (one block per cell and frame), each cell's sum is an exact integer
// divided once, and the lags are searched on the device, one thread per lag, adding the differences in the same order
// and arithmetic as the reference's loop so that the chosen lag is the same.
#include "es_kernels.h"

namespace es {
namespace {

__device__ __forceinline__ unsigned luma_at(const FrameViewDev &f, int x, int y)
{
    const unsigned char *row = (const unsigned char *)f.y + (size_t)y * f.ypitch;
    const unsigned v = f.bytes == 1 ? row[x] : ((const uint16_t *)row)[x];
    return v >> f.shift;
}

// Block (tx, ty, frame): the mean of cell (tx, ty) of that frame, for any crop and alignment. Threads walk the cell as
// 8 rows of 32 columns (one warp per row, consecutive columns per lane), summing 10-bit samples exactly.
__global__ void __launch_bounds__(256) thumb_kernel(const __grid_constant__ ThumbBatch b)
{
    const FrameViewDev &f = b.f[blockIdx.z];
    const int tx = blockIdx.x, ty = blockIdx.y;
    const int xa = b.x0 + tx * b.w / kThumbW, xb = b.x0 + (tx + 1) * b.w / kThumbW;
    const int ya = b.y0 + ty * b.h / kThumbH, yb = b.y0 + (ty + 1) * b.h / kThumbH;
    const int lane = threadIdx.x & 31, row = threadIdx.x >> 5, up = 10 - f.depth;
    unsigned s = 0;  // at most a cell's share of a thread times 1023: far below 2^32 for any picture size in use
    for (int y = ya + row; y < yb; y += 8)
        for (int x = xa + lane; x < xb; x += 32) s += luma_at(f, x, y) << up;
    unsigned long long t = s;
#pragma unroll
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __shared__ unsigned long long part[8];
    if (lane == 0) part[row] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long total = 0;
        for (int k = 0; k < 8; k++) total += part[k];
        const int n = (xb - xa) * (yb - ya);
        // a cell with no pixel gives 0 / 0 = NaN, as in the reference
        b.out[((size_t)blockIdx.z * kThumbH + ty) * kThumbW + tx] = __fdiv_rn((float)total, (float)n);
    }
}

// The same thumbnails when the crop allows 16-byte (8-byte for 8-bit samples) loads of 8 columns: x0 and w multiples of
// 8, w >= 512 (every cell at least 8 columns wide, so 8 columns span at most two cells), aligned planes and pitches.
// Block (ty, frame) makes the 64 cells of thumbnail row ty from its band of rows: thread g takes the columns
// x0 + 8 g .. + 7 of every row of the band, adding them into the two cells they can fall in, and the block's cell sums
// meet in shared memory.
__global__ void __launch_bounds__(256) thumb_rows_kernel(const __grid_constant__ ThumbBatch b)
{
    const FrameViewDev &f = b.f[blockIdx.y];
    const int ty = blockIdx.x;
    const int ya = b.y0 + ty * b.h / kThumbH, yb = b.y0 + (ty + 1) * b.h / kThumbH;
    __shared__ unsigned long long cell[kThumbW];
    if (threadIdx.x < kThumbW) cell[threadIdx.x] = 0;
    __syncthreads();
    const int up = 10 - f.depth, groups = b.w / 8;
    for (int g = threadIdx.x; g < groups; g += 256) {
        const int c = 8 * g;                         // the group's first column, from x0
        int ta = 64 * c / b.w;                       // its cell: 64 c / w or the next one
        if (ta < kThumbW - 1 && (ta + 1) * b.w / kThumbW <= c) ta++;
        const int bound = (ta + 1) * b.w / kThumbW;  // first column of cell ta + 1
        unsigned sa = 0, sb = 0;
#pragma unroll 4
        for (int y = ya; y < yb; y++) {
            const unsigned char *row = (const unsigned char *)f.y + (size_t)y * f.ypitch;
            unsigned v[8];
            if (f.bytes == 2) {
                const uint4 q = __ldg((const uint4 *)((const uint16_t *)row + b.x0 + c));
                const unsigned w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    v[2 * k] = w4[k] & 0xFFFFu;
                    v[2 * k + 1] = w4[k] >> 16;
                }
            } else {
                const uint2 q = __ldg((const uint2 *)(row + b.x0 + c));
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    v[k] = (q.x >> (8 * k)) & 0xFFu;
                    v[4 + k] = (q.y >> (8 * k)) & 0xFFu;
                }
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const unsigned s = (v[k] >> f.shift) << up;
                if (c + k < bound) sa += s;
                else sb += s;
            }
        }
        atomicAdd(&cell[ta], (unsigned long long)sa);
        if (sb) atomicAdd(&cell[ta + 1], (unsigned long long)sb);  // columns past `bound` exist only when ta < 63
    }
    __syncthreads();
    if (threadIdx.x < kThumbW) {
        const int t = threadIdx.x, n = ((t + 1) * b.w / kThumbW - t * b.w / kThumbW) * (yb - ya);
        b.out[((size_t)blockIdx.y * kThumbH + ty) * kThumbW + t] = __fdiv_rn((float)cell[t], (float)n);
    }
}

// Thread l: the total of lag l, sum over probe frames i and pixels p (in that order) of |ref[l + i][p] - probe[i][p]|,
// the difference in float and the sum in double (src/main.cpp:342-346). Frames are stored one after another, so the
// pairs a lag reads are two contiguous runs of n_probe x 2304 floats. Each lag is one chain of dependent additions;
// one warp per block spreads the lags over the SMs, and with 16-byte aligned arrays (`vec`) each lane reads its values
// 8 at a time with two 16-byte loads per array, kDepth groups of 8 ahead of the additions, so the chain waits on the
// additions rather than on the loads; the order of the additions is unchanged.
constexpr int kDepth = 4;

__global__ void __launch_bounds__(32) offset_totals_kernel(const float *ref, const float *probe, int n_probe, int lags, double *totals,
                                                           int vec)
{
    const int l = blockIdx.x * 32 + threadIdx.x;
    if (l >= lags) return;
    const float *r = ref + (size_t)l * kThumbPixels;
    const long long count = (long long)n_probe * kThumbPixels;  // a multiple of 8
    double total = 0.0;
    auto add = [&](float a, float p) { total = __dadd_rn(total, (double)fabsf(__fsub_rn(a, p))); };
    if (vec) {
        const float4 *r4 = (const float4 *)r, *p4 = (const float4 *)probe;
        const long long nq = count / 4;  // float4s per array, a multiple of 2
        float4 ra[kDepth][2], pa[kDepth][2];
#pragma unroll
        for (int d = 0; d < kDepth; d++) {
            const long long q = 2 * d;
            if (q < nq) {
                ra[d][0] = __ldg(r4 + q);
                ra[d][1] = __ldg(r4 + q + 1);
                pa[d][0] = __ldg(p4 + q);
                pa[d][1] = __ldg(p4 + q + 1);
            }
        }
        for (long long k = 0; k < nq; k += 2 * kDepth) {
#pragma unroll
            for (int d = 0; d < kDepth; d++) {
                if (k + 2 * d >= nq) break;
                const float4 a0 = ra[d][0], a1 = ra[d][1], p0 = pa[d][0], p1 = pa[d][1];
                const long long q = k + 2 * d + 2 * kDepth;  // the group this slot holds next
                if (q < nq) {
                    ra[d][0] = __ldg(r4 + q);
                    ra[d][1] = __ldg(r4 + q + 1);
                    pa[d][0] = __ldg(p4 + q);
                    pa[d][1] = __ldg(p4 + q + 1);
                }
                add(a0.x, p0.x);
                add(a0.y, p0.y);
                add(a0.z, p0.z);
                add(a0.w, p0.w);
                add(a1.x, p1.x);
                add(a1.y, p1.y);
                add(a1.z, p1.z);
                add(a1.w, p1.w);
            }
        }
    } else {
#pragma unroll 8
        for (long long k = 0; k < count; k++) add(__ldg(r + k), __ldg(probe + k));
    }
    totals[l] = total;
}

}  // namespace

cudaError_t launch_thumbnails(const ThumbBatch &b, cudaStream_t s)
{
    if (b.n <= 0) return cudaSuccess;
    bool rows = b.w >= 512 && b.w % 8 == 0 && b.x0 % 8 == 0;
    for (int i = 0; i < b.n && rows; i++) {
        const unsigned a = b.f[i].bytes == 2 ? 16u : 8u;
        rows = ((uintptr_t)b.f[i].y % a) == 0 && b.f[i].ypitch % a == 0;
    }
    LaunchTimer t("align_thumbnails", s);
    if (rows) thumb_rows_kernel<<<dim3(kThumbH, b.n), 256, 0, s>>>(b);
    else thumb_kernel<<<dim3(kThumbW, kThumbH, b.n), 256, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_offset_totals(const float *ref, const float *probe, int n_probe, int lags, double *totals, cudaStream_t s)
{
    if (lags <= 0) return cudaSuccess;
    const int vec = (((uintptr_t)ref | (uintptr_t)probe) & 15) == 0;
    LaunchTimer t("align_offset_totals", s);
    offset_totals_kernel<<<(lags + 31) / 32, 32, 0, s>>>(ref, probe, n_probe, lags, totals, vec);
    return after_launch();
}

}  // namespace es
