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

// The total of lag l: the sum over probe frames i and pixels p (in that order) of |ref[l + i][p] - probe[i][p]|, the
// difference in float and the sum in double (src/main.cpp:342-346). Frames are stored one after another, so a lag
// reads two contiguous runs of n_probe x 2304 floats. One warp per lag, chunks of kChunk values, lane j holding values
// j*kLaneVals .. j*kLaneVals + kLaneVals - 1 of a chunk.
//
// The running total s is a double >= 0 and every value x is a float >= 0. While s stays in one binade [2^e, 2^(e+1)),
// s = m * u with u = 2^(e-52) and m an integer in [2^52, 2^53), and the rounded sum RN(s + x) is (m + n + r) * u where
// n = floor(x / u) and r is 1 when the remainder of x / u is above one half, 0 below, and on an exact half the value
// that makes m + n + r even (ties to even). x / u is exact (x has a 24-bit mantissa, u is a power of two), so n and the
// remainder's class come from integer shifts of x's mantissa. The only state one step passes to the next beyond the
// increment is the parity of m, so a run of values is a map from the parity coming in to (increment, parity going
// out): a pair of increments and a pair of parities. These maps compose in order, which makes the chunk an ordered
// warp reduction instead of a chain of kChunk dependent additions. If the chunk's end stays below 2^53 (m + the
// increment), every intermediate sum stayed in the binade (each exact sum is within one half of the next rounded
// one), so the result is exactly the in-order chain's. A chunk that crosses a binade, starts from s = 0, or holds a
// value the shifts cannot represent (an increment of 2^53 or more, an infinity or NaN) is added in order, one value at
// a time, from shared memory. Adding zeros leaves s as it is, so a chunk of zeros and the padding of the last chunk
// are skipped. The result equals the in-order double sum bit for bit.
constexpr int kLaneVals = 16, kChunk = 32 * kLaneVals, kLagWarps = 4;

struct ParityMap {
    unsigned long long inc0, inc1;  // increments of m for parity 0 / 1 coming in
    unsigned bits;                  // bit 0: parity out for 0 in, bit 1: for 1 in, bit 2: the chunk must be added in order
};

__device__ __forceinline__ ParityMap compose(const ParityMap &a, const ParityMap &b)
{
    const unsigned a0 = a.bits & 1u, a1 = (a.bits >> 1) & 1u, b0 = b.bits & 1u, b1 = (b.bits >> 1) & 1u;
    ParityMap r;
    r.inc0 = a.inc0 + (a0 ? b.inc1 : b.inc0);
    r.inc1 = a.inc1 + (a1 ? b.inc1 : b.inc0);
    r.bits = (a0 ? b1 : b0) | ((a1 ? b1 : b0) << 1) | ((a.bits | b.bits) & 4u);
    return r;
}

template <bool kVec>
__global__ void __launch_bounds__(32 * kLagWarps) offset_totals_kernel(const float *ref, const float *probe, int n_probe, int lags,
                                                                      double *totals)
{
    __shared__ __align__(16) double serial[kLagWarps][kChunk];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, l = blockIdx.x * kLagWarps + w;
    if (l >= lags) return;  // whole warps: one lag per warp
    const float *r = ref + (size_t)l * kThumbPixels;
    const long long count = (long long)n_probe * kThumbPixels;
    const long long chunks = (count + kChunk - 1) / kChunk;
    constexpr int Q = kLaneVals / 4;
    float4 ra[Q], pa[Q];
    auto load = [&](long long c) {  // the next chunk's values, zeros past the end
        const long long v0 = c * kChunk + lane * kLaneVals;
#pragma unroll
        for (int t = 0; t < Q; t++) {
            const long long v = v0 + 4 * t;
            if (kVec) {
                if (v < count) {
                    ra[t] = __ldg((const float4 *)(r + v));
                    pa[t] = __ldg((const float4 *)(probe + v));
                } else {
                    ra[t] = pa[t] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            } else {
                float a[4], b[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    a[k] = v + k < count ? __ldg(r + v + k) : 0.f;
                    b[k] = v + k < count ? __ldg(probe + v + k) : 0.f;
                }
                ra[t] = make_float4(a[0], a[1], a[2], a[3]);
                pa[t] = make_float4(b[0], b[1], b[2], b[3]);
            }
        }
    };
    double s = 0.0;
    if (chunks > 0) load(0);
    for (long long c = 0; c < chunks; c++) {
        float x[kLaneVals];
#pragma unroll
        for (int t = 0; t < Q; t++) {
            x[4 * t + 0] = fabsf(__fsub_rn(ra[t].x, pa[t].x));
            x[4 * t + 1] = fabsf(__fsub_rn(ra[t].y, pa[t].y));
            x[4 * t + 2] = fabsf(__fsub_rn(ra[t].z, pa[t].z));
            x[4 * t + 3] = fabsf(__fsub_rn(ra[t].w, pa[t].w));
        }
        if (c + 1 < chunks) load(c + 1);
        const unsigned long long sbits = (unsigned long long)__double_as_longlong(s);
        const int E = (int)(sbits >> 52);  // s >= 0: the biased exponent
        const int ue = E - 1075;           // u = 2^ue
        ParityMap m;
        m.inc0 = m.inc1 = 0;
        m.bits = 2u | ((E == 0 || E == 0x7ff) ? 4u : 0u);
        bool nonzero = false;
#pragma unroll
        for (int j = 0; j < kLaneVals; j++) {
            const unsigned xb = __float_as_uint(x[j]);
            nonzero |= xb != 0;
            const int ex = (int)(xb >> 23);  // x >= 0
            const unsigned M = ex ? (xb & 0x7fffffu) | 0x800000u : xb;  // x = M * 2^(ex - 150), subnormals 2^-149
            const int sh = (ex ? ex - 150 : -149) - ue;                 // x / u = M * 2^sh
            const int left = max(sh, 0), right = min(max(-sh, 0), 25);  // M < 2^24: 25 right shifts leave 0 and a low remainder
            if (ex == 255 || left > 29) m.bits |= 4u;
            const unsigned long long n = ((unsigned long long)M << min(left, 29)) >> right;
            const unsigned twice_rem = (M & ((1u << right) - 1u)) << 1, one = 1u << right;
            const unsigned above = twice_rem > one, tie = twice_rem == one, nb = (unsigned)n & 1u;
            const unsigned p0 = m.bits & 1u, p1 = (m.bits >> 1) & 1u;
            const unsigned r0 = above | (tie & (p0 ^ nb)), r1 = above | (tie & (p1 ^ nb));
            m.inc0 += n + r0;
            m.inc1 += n + r1;
            m.bits = (m.bits & 4u) | ((p0 ^ nb ^ r0) & 1u) | (((p1 ^ nb ^ r1) & 1u) << 1);
        }
        if (!__any_sync(0xffffffffu, nonzero)) continue;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {  // ordered: lane j's run, then lane j + off's
            ParityMap o;
            o.inc0 = __shfl_down_sync(0xffffffffu, m.inc0, off);
            o.inc1 = __shfl_down_sync(0xffffffffu, m.inc1, off);
            o.bits = __shfl_down_sync(0xffffffffu, m.bits, off);
            if (lane + off < 32) m = compose(m, o);
        }
        const unsigned long long inc0 = __shfl_sync(0xffffffffu, m.inc0, 0), inc1 = __shfl_sync(0xffffffffu, m.inc1, 0);
        bool in_order = (__shfl_sync(0xffffffffu, m.bits, 0) & 4u) != 0;
        if (!in_order) {
            const unsigned long long mant = (sbits & 0xfffffffffffffull) | (1ull << 52);
            const unsigned long long end = mant + ((mant & 1ull) ? inc1 : inc0);
            if (end < (1ull << 53))
                s = __longlong_as_double((long long)(((unsigned long long)E << 52) | (end & 0xfffffffffffffull)));
            else
                in_order = true;
        }
        if (in_order) {
#pragma unroll
            for (int j = 0; j < kLaneVals; j++) serial[w][lane * kLaneVals + j] = (double)x[j];
            __syncwarp();
            if (lane == 0)
                for (int i = 0; i < kChunk; i++) s = __dadd_rn(s, serial[w][i]);
            s = __shfl_sync(0xffffffffu, s, 0);
            __syncwarp();
        }
    }
    if (lane == 0) totals[l] = s;
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
    const bool vec = (((uintptr_t)ref | (uintptr_t)probe) & 15) == 0;  // rows of 2304 floats keep the alignment
    LaunchTimer t("align_offset_totals", s);
    const int blocks = (lags + kLagWarps - 1) / kLagWarps;
    if (vec) offset_totals_kernel<true><<<blocks, 32 * kLagWarps, 0, s>>>(ref, probe, n_probe, lags, totals);
    else offset_totals_kernel<false><<<blocks, 32 * kLagWarps, 0, s>>>(ref, probe, n_probe, lags, totals);
    return after_launch();
}

}  // namespace es
