// CAMBI (Contrast Aware Multiscale Banding Index) kernels for sm_100a.
//
// Per picture the reference (src/kernels.cu:14-278, src/cambi.cpp:88-184) copies or converts the plane, builds the
// zero-derivative mask, runs decimation and a mode filter per scale, counts windowed histograms into a full float
// c-value buffer that it clears every frame, and pools the top 60% with host-driven radix rounds. Here:
//
//  * prep0_kernel fuses the 8-to-10-bit conversion (or copy), the 7x7 flat-pixel count and the 3x3 mode filter of
//    scale 0 in one pass over a shared-memory tile, and packs each pixel as value | mask << 15, so every later step
//    reads one 16-bit word per pixel;
//  * decimate_mode_kernel builds scales 1-4 the same way from the previous scale's words;
//  * cvalues_kernel gives each 64 x 32 tile a 256-thread block: the tile and its window margins are staged once in
//    shared memory as band codes, the values that can matter are ranked (a handful on banded content), column counts
//    slide down the rows, and per row a warp-parallel prefix sum over the columns turns them into window counts that
//    each pixel reads in O(1). The positive c-values are summed exactly (they are multiples of 2^-24) and appended to
//    a per-scale list, so no c-value buffer is cleared or written;
//  * select_round_kernel / select_pick_kernel / sum_above_kernel find the exact k-th largest value on the device when
//    more than k values are positive (no host round trips), and score_kernel pools and weights the scales.
#include "es_kernels.h"

namespace es {
namespace {

__device__ __forceinline__ uint16_t mode3(uint16_t a, uint16_t b, uint16_t c)
{
    if (a == b || a == c) return a;
    if (b == c) return b;
    return min(a, min(b, c));
}

// ---------------------------------------------------------------------------------------------------------------
// Scale 0: src/kernels.cu:524-535 (from8), 14-40 (mask), 488-500 (mode).
// ---------------------------------------------------------------------------------------------------------------
constexpr int kP0W = 64, kP0H = 16;             // output tile
constexpr int kP0RW = kP0W + 8, kP0RH = kP0H + 8;  // input region x0-3 .. x0+kP0W+5

__global__ void __launch_bounds__(256) prep0_kernel(const __grid_constant__ Prep0Batch b)
{
    __shared__ uint16_t raw[kP0RH][kP0RW];
    __shared__ uint16_t pre[kP0RH - 1][kP0RW];
    __shared__ uint8_t flat[kP0RH - 2][kP0RW];
    __shared__ uint8_t hs[kP0RH - 2][kP0W];
    int j = 0;
    while (j + 1 < b.njobs && (int)blockIdx.x >= b.job[j + 1].first_tile) j++;
    const Prep0Job &J = b.job[j];
    const int t = blockIdx.x - J.first_tile, w = J.w, h = J.h, tid = threadIdx.x;
    const int x0 = (t % J.tiles_x) * kP0W, y0 = (t / J.tiles_x) * kP0H;
    for (int i = tid; i < kP0RH * kP0RW; i += 256) {
        const int r = i / kP0RW, c = i - r * kP0RW, x = x0 - 3 + c, y = y0 - 3 + r;
        raw[r][c] = (x >= 0 && x < w && y >= 0 && y < h) ? J.img[(size_t)y * J.pitch + x] : (uint16_t)0;
    }
    __syncthreads();
    // preprocessed values of x0-3 .. x0+kP0W+3, y0-3 .. y0+kP0H+3
    for (int i = tid; i < (kP0RH - 1) * (kP0RW - 1); i += 256) {
        const int r = i / (kP0RW - 1), c = i - r * (kP0RW - 1), x = x0 - 3 + c, y = y0 - 3 + r;
        unsigned v = 0;
        if (x >= 0 && x < w && y >= 0 && y < h) {
            if (J.depth == 8) {
                // 10 bits, then the mean of the 2x2 block to the lower right; pairs on the last row and column
                const unsigned a = (unsigned)raw[r][c] << 2;
                if (x < w - 1 && y < h - 1)
                    v = (a + ((unsigned)raw[r][c + 1] << 2) + ((unsigned)raw[r + 1][c] << 2) + ((unsigned)raw[r + 1][c + 1] << 2)) >> 2;
                else if (y < h - 1) v = (a + ((unsigned)raw[r + 1][c] << 2)) >> 1;
                else if (x < w - 1) v = (a + ((unsigned)raw[r][c + 1] << 2)) >> 1;
                else v = a;
            } else {
                v = raw[r][c];
            }
        }
        pre[r][c] = (uint16_t)v;
    }
    __syncthreads();
    // flat: equal to the right and lower neighbours (the last column / row count as equal); nothing outside
    for (int i = tid; i < (kP0RH - 2) * (kP0RW - 2); i += 256) {
        const int r = i / (kP0RW - 2), c = i - r * (kP0RW - 2), x = x0 - 3 + c, y = y0 - 3 + r;
        bool f = false;
        if (x >= 0 && x < w && y >= 0 && y < h) {
            const uint16_t v = pre[r][c];
            f = (x == w - 1 || v == pre[r][c + 1]) && (y == h - 1 || v == pre[r + 1][c]);
        }
        flat[r][c] = f;
    }
    __syncthreads();
    for (int i = tid; i < (kP0RH - 2) * kP0W; i += 256) {
        const int r = i / kP0W, c = i - r * kP0W;
        int s = 0;
#pragma unroll
        for (int k = 0; k < 7; k++) s += flat[r][c + k];
        hs[r][c] = (uint8_t)s;
    }
    __syncthreads();
    for (int i = tid; i < kP0H * kP0W; i += 256) {
        const int r = i / kP0W, c = i - r * kP0W, x = x0 + c, y = y0 + r;
        if (x >= w || y >= h) continue;
        int cnt = 0;
#pragma unroll
        for (int k = 0; k < 7; k++) cnt += hs[r + k][c];
        const int pr = r + 3, pc = c + 3;
        uint16_t v;
        if (y == 0 || y == h - 1) {
            v = pre[pr][pc];
        } else {
            uint16_t m[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const int rr = pr - 1 + k;
                m[k] = (x == 0 || x == w - 1) ? pre[rr][pc] : mode3(pre[rr][pc - 1], pre[rr][pc], pre[rr][pc + 1]);
            }
            v = mode3(m[0], m[1], m[2]);
        }
        J.word[(size_t)y * w + x] = (uint16_t)(v | (cnt > J.mask_index ? kMaskBit : 0));
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Scales 1-4: src/kernels.cu:43-53 (decimate) and 488-500 (mode) on the decimated picture, mask decimated alongside.
// ---------------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) decimate_mode_kernel(const __grid_constant__ DecBatch b)
{
    int j = 0;
    while (j + 1 < b.njobs && (int)blockIdx.x >= b.job[j + 1].first_block) j++;
    const DecJob &J = b.job[j];
    const int i = (blockIdx.x - J.first_block) * 256 + threadIdx.x;
    if (i >= J.w * J.h) return;
    const int x = i % J.w, y = i / J.w, w = J.w, h = J.h;
    auto val = [&](int xx, int yy) -> uint16_t { return J.src[(size_t)(2 * yy) * J.sw + 2 * xx] & 0x7FFF; };
    const uint16_t m = J.src[(size_t)(2 * y) * J.sw + 2 * x] & kMaskBit;
    uint16_t v;
    if (y == 0 || y == h - 1) {
        v = val(x, y);
    } else {
        uint16_t mm[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int rr = y - 1 + k;
            mm[k] = (x == 0 || x == w - 1) ? val(x, rr) : mode3(val(x - 1, rr), val(x, rr), val(x + 1, rr));
        }
        v = mode3(mm[0], mm[1], mm[2]);
    }
    J.dst[i] = (uint16_t)(v | m);
}

// ---------------------------------------------------------------------------------------------------------------
// C-values: src/kernels.cu:113-278 (cambi.c's c_value_pixel over the (2 pad + 1)^2 window of every masked pixel in
// the band, histogram windows clipped at the picture's edges).
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool needs_cvalue(int code, const Band &bd)
{
    const int value = code + bd.band_base + kDiffs;
    bool any = false;
#pragma unroll
    for (int d = 0; d < kDiffs; d++) any |= value <= bd.tvi[d] && value + d + 1 > bd.vlt;
    return any;
}

__host__ __device__ constexpr int cv_cs(int pad) { return (kCvTX + 2 * pad + 127) & ~127; }  // column stride
__host__ __device__ constexpr int cv_hs(int pad) { return cv_cs(pad) + 8; }                   // prefix row stride
__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

struct CvLayout {
    size_t codes, rank, colcnt, prefix, list, total;
};
__host__ __device__ inline CvLayout cv_layout(int pad)
{
    CvLayout l;
    const int rw = kCvTX + 2 * pad, rh = kCvTY + 2 * pad;
    l.codes = 0;
    l.rank = align16(l.codes + (size_t)rw * rh * 2);
    l.colcnt = align16(l.rank + (size_t)kMaxBand * 2);
    l.prefix = align16(l.colcnt + (size_t)kCvBins * cv_cs(pad));
    l.list = align16(l.prefix + (size_t)2 * kCvBins * cv_hs(pad) * 2);
    l.total = align16(l.list + (size_t)kCvTX * kCvTY * 4);
    return l;
}

__global__ void __launch_bounds__(kCvThreads) cvalues_kernel(const __grid_constant__ CvBatch b)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t occ[32], srv[32], rel[32];
    __shared__ uint16_t relpre[33];
    __shared__ uint32_t rowflags;
    __shared__ int any_srv;
    __shared__ unsigned list_n;
    __shared__ unsigned long long list_base;
    __shared__ unsigned long long red_sum[kCvThreads / 32];
    __shared__ unsigned red_cnt[kCvThreads / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int j = 0;
    while (j + 1 < b.njobs && (int)blockIdx.x >= b.job[j + 1].first_tile) j++;
    const CvJob &J = b.job[j];
    const Band &bd = b.band;
    const int tile = blockIdx.x - J.first_tile;
    const int x0 = (tile % J.tiles_x) * kCvTX, y0 = (tile / J.tiles_x) * kCvTY;
    const int w = J.w, h = J.h, P = J.pad;
    const int rows = min(kCvTY, h - y0), cols = min(kCvTX, w - x0);
    const int RW = kCvTX + 2 * P, RH = rows + 2 * P, CS = cv_cs(P), HS = cv_hs(P);
    const CvLayout L = cv_layout(P);
    uint16_t *codes = (uint16_t *)(smem + L.codes);
    uint16_t *rank = (uint16_t *)(smem + L.rank);
    uint8_t *colcnt = smem + L.colcnt;
    uint16_t *prefix = (uint16_t *)(smem + L.prefix);
    float *blist = (float *)(smem + L.list);

    if (tid < 32) occ[tid] = srv[tid] = 0;
    if (tid == 0) list_n = 0;
    __syncthreads();

    // stage the tile and its window margins as band codes: the value less band_base for a masked pixel in the band,
    // kNone otherwise (outside the picture too); note which codes occur and which the tile's pixels need c-values of
    const int N = RH * RW;
    for (int base = 0; base < N; base += kCvThreads) {
        const int i = base + tid;
        uint16_t code = kNone;
        bool served = false;
        if (i < N) {
            const int r = i / RW, c = i - r * RW, x = x0 - P + c, y = y0 - P + r;
            if (x >= 0 && x < w && y >= 0 && y < h) {
                const uint16_t wd = J.word[(size_t)y * w + x];
                const unsigned u = (unsigned)(wd & 0x7FFF) - (unsigned)bd.band_base;
                if ((wd & kMaskBit) && u < (unsigned)bd.band_size) code = (uint16_t)u;
            }
            codes[i] = code;
            served = code != kNone && r >= P && r < P + rows && c >= P && c < P + cols && needs_cvalue(code, bd);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, (unsigned)code);
        if (code != kNone && lane == __ffs(peers) - 1) atomicOr(&occ[code >> 5], 1u << (code & 31));
        const unsigned speers = __match_any_sync(0xffffffffu, served ? (unsigned)code : 0xFFFFFFFFu);
        if (served && lane == __ffs(speers) - 1) atomicOr(&srv[code >> 5], 1u << (code & 31));
    }
    __syncthreads();

    // the relevant codes: those that occur within kDiffs of a code that needs c-values, numbered in order
    if (warp == 0) {
        const uint32_t s = srv[lane], sp = lane > 0 ? srv[lane - 1] : 0u, sn = lane < 31 ? srv[lane + 1] : 0u;
        uint32_t dil = s;
#pragma unroll
        for (int k = 1; k <= kDiffs; k++) dil |= (s << k) | (sp >> (32 - k)) | (s >> k) | (sn << (32 - k));
        const uint32_t r = occ[lane] & dil;
        rel[lane] = r;
        const unsigned cnt = __popc(r);
        unsigned incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        relpre[lane] = (uint16_t)(incl - cnt);
        if (lane == 31) relpre[32] = (uint16_t)incl;
        const bool anys = __any_sync(0xffffffffu, s != 0u);
        if (lane == 0) any_srv = anys;
    }
    __syncthreads();
    if (!any_srv) return;
    const int R = relpre[32];
    for (int c = tid; c < bd.band_size; c += kCvThreads) {
        const uint32_t word = rel[c >> 5], bit = 1u << (c & 31);
        rank[c] = (word & bit) ? (uint16_t)(relpre[c >> 5] + __popc(word & (bit - 1u))) : kNone;
    }
    __syncthreads();

    unsigned long long my_sum = 0;
    unsigned my_cnt = 0;
    const int cv_warp0 = kCvThreads / 32 - kCvTX / 32;  // the warps that compute c-values
    const int ct = tid - cv_warp0 * 32;                // their pixel column in the tile

    // passes over the numbers b0 .. b0 + kCvBins - 1; a pass serves the pixels whose neighbours within kDiffs values
    // all fall in it (numbers of values within kDiffs of each other are within kDiffs of each other)
    for (int b0 = 0;;) {
        const int B = min(kCvBins, R - b0);
        const int lo = b0 ? b0 + kDiffs : 0, hi = b0 + kCvBins >= R ? R : b0 + kCvBins - kDiffs;
        if (tid == 0) rowflags = 0;
        for (int i = tid * 16; i < kCvBins * CS; i += kCvThreads * 16) *(uint4 *)(colcnt + i) = make_uint4(0, 0, 0, 0);
        __syncthreads();
        for (int i = tid; i < rows * kCvTX; i += kCvThreads) {
            const int r = i / kCvTX, c = i - r * kCvTX;
            if (c >= cols) continue;
            const uint16_t code = codes[(r + P) * RW + c + P];
            if (code == kNone) continue;
            const int rk = rank[code];
            if (rk != kNone && rk >= lo && rk < hi && needs_cvalue(code, bd)) atomicOr(&rowflags, 1u << r);
        }
        // column counts over the window rows of tile row 0 (region rows 0 .. 2P)
        if (tid < RW) {
            uint8_t *col = colcnt + tid;
            const int last = min(2 * P, RH - 1);
            for (int r = 0; r <= last; r++) {
                const uint16_t code = codes[r * RW + tid];
                if (code != kNone) {
                    const int k = (int)rank[code] - b0;
                    if ((unsigned)k < (unsigned)B) col[k * CS]++;
                }
            }
        }
        __syncthreads();
        const uint32_t flags = rowflags;
        for (int r = 0; r < rows; r++) {
            if (r > 0 && tid < RW) {
                uint8_t *col = colcnt + tid;
                const uint16_t cl = codes[(r - 1) * RW + tid];
                if (cl != kNone) {
                    const int k = (int)rank[cl] - b0;
                    if ((unsigned)k < (unsigned)B) col[k * CS]--;
                }
                if (r + 2 * P < RH) {
                    const uint16_t ce = codes[(r + 2 * P) * RW + tid];
                    if (ce != kNone) {
                        const int k = (int)rank[ce] - b0;
                        if ((unsigned)k < (unsigned)B) col[k * CS]++;
                    }
                }
            }
            if (!((flags >> r) & 1u)) continue;
            __syncthreads();
            // inclusive prefix sums of each number's column counts: window counts are differences of two
            uint16_t *hb = prefix + (size_t)(r & 1) * kCvBins * HS;
            for (int k = warp; k < B; k += kCvThreads / 32) {
                const uint8_t *col = colcnt + k * CS;
                uint16_t *hrow = hb + k * HS;
                unsigned carry = 0;
                for (int base = 0; base < CS; base += 128) {
                    const uint32_t four = *(const uint32_t *)(col + base + 4 * lane);
                    const unsigned s1 = four & 255u, s2 = s1 + ((four >> 8) & 255u), s3 = s2 + ((four >> 16) & 255u),
                                   s4 = s3 + (four >> 24);
                    unsigned incl = s4;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += v;
                    }
                    const unsigned ex = incl - s4 + carry;
                    uint2 out;
                    out.x = (ex + s1) | ((ex + s2) << 16);
                    out.y = (ex + s3) | ((ex + s4) << 16);
                    *(uint2 *)(hrow + base + 4 * lane) = out;
                    carry += __shfl_sync(0xffffffffu, incl, 31);
                }
            }
            __syncthreads();
            if (warp >= cv_warp0) {
                float c = 0.0f;
                bool served = false;
                if (ct < cols) {
                    const uint16_t code = codes[(r + P) * RW + ct + P];
                    if (code != kNone) {
                        const int rk = rank[code];
                        if (rk >= lo && rk < hi && needs_cvalue(code, bd)) {
                            served = true;
                            auto count = [&](int q) -> unsigned {
                                if (q < 0 || q >= bd.band_size) return 0u;
                                const int k = rank[q];
                                if (k == kNone) return 0u;
                                const uint16_t *row = hb + (k - b0) * HS;
                                return (unsigned)row[ct + 2 * P] - (ct > 0 ? (unsigned)row[ct - 1] : 0u);
                            };
                            const int value = code + bd.band_base + kDiffs;
                            const unsigned p0 = count(code);
#pragma unroll
                            for (int d = 0; d < kDiffs; d++) {
                                if (value <= bd.tvi[d] && value + d + 1 > bd.vlt) {
                                    const unsigned p1 = count(code + d + 1), p2 = count(code - d - 1);
                                    const unsigned pm = p1 > p2 ? p1 : p2;
                                    const float val = __fmul_rn(__uint2float_rn((unsigned)bd.weight[d] * p0 * pm), __ldg(b.lut + p0 + pm));
                                    if (val > c) c = val;
                                }
                            }
                        }
                    }
                }
                const bool pos = c > 0.0f;
                const unsigned m = __ballot_sync(0xffffffffu, pos);
                if (m) {
                    unsigned at = 0;
                    if (lane == __ffs(m) - 1) at = atomicAdd(&list_n, (unsigned)__popc(m));
                    at = __shfl_sync(0xffffffffu, at, __ffs(m) - 1);
                    if (pos) blist[at + __popc(m & ((1u << lane) - 1u))] = c;
                }
                if (served && J.plane) J.plane[(size_t)(y0 + r) * w + x0 + ct] = c;
                if (pos) {
                    my_sum += __float2ull_rn(__fmul_rn(c, 16777216.0f));
                    my_cnt++;
                }
            }
        }
        if (hi == R) break;
        b0 = hi - kDiffs;
        __syncthreads();
    }

    // block totals, and this block's positive c-values appended to the scale's list
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        my_sum += __shfl_down_sync(0xffffffffu, my_sum, o);
        my_cnt += __shfl_down_sync(0xffffffffu, my_cnt, o);
    }
    if (lane == 0) {
        red_sum[warp] = my_sum;
        red_cnt[warp] = my_cnt;
    }
    __syncthreads();
    CvSlot &S = b.slots[J.slot];
    if (tid == 0) {
        unsigned long long s = 0;
        unsigned c = 0;
        for (int k = 0; k < kCvThreads / 32; k++) {
            s += red_sum[k];
            c += red_cnt[k];
        }
        if (c) {
            atomicAdd(&S.sum_fx, s);
            atomicAdd(&S.count, (unsigned long long)c);
            list_base = atomicAdd(&S.list_n, (unsigned long long)list_n);
        }
    }
    __syncthreads();
    const unsigned ln = list_n;
    for (unsigned i = tid; i < ln; i += kCvThreads) S.list[list_base + i] = blist[i];
}

// ---------------------------------------------------------------------------------------------------------------
// Pooling: src/cambi.cpp:137-184 with the radix rounds on the device.
// ---------------------------------------------------------------------------------------------------------------
struct SlotInit {
    unsigned long long n, k;
};

__global__ void slots_reset_kernel(CvSlot *slots, int nslots, const unsigned long long *n, const unsigned long long *k)
{
    const int s = blockIdx.x;
    if (s >= nslots) return;
    CvSlot &S = slots[s];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) S.hist[i] = 0;
    if (threadIdx.x == 0) {
        S.sum_fx = S.count = S.list_n = 0;
        S.n = n[s];
        S.k = k[s];
        S.remaining = k[s];
        S.above_fx = S.above_n = 0;
        S.prefix = S.mask = 0;
    }
}

__global__ void __launch_bounds__(256) select_hist_kernel(CvSlot *slots, int shift, int width)
{
    CvSlot &S = slots[blockIdx.y];
    if (S.count <= S.k) return;
    __shared__ unsigned hist[2048];
    const int nb = 1 << width;
    for (int i = threadIdx.x; i < nb; i += 256) hist[i] = 0;
    __syncthreads();
    const unsigned *v = (const unsigned *)S.list;
    const unsigned long long n = S.list_n;
    const unsigned mask = S.mask, prefix = S.prefix;
    for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < n; i += (unsigned long long)gridDim.x * 256ull) {
        const unsigned bits = v[i];
        if ((bits & mask) == prefix) atomicAdd(&hist[(bits >> shift) & (unsigned)(nb - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += 256)
        if (hist[i]) atomicAdd(&S.hist[i], hist[i]);
}

__global__ void __launch_bounds__(256) select_pick_kernel(CvSlot *slots, int shift, int width)
{
    CvSlot &S = slots[blockIdx.x];
    if (S.count <= S.k) return;
    __shared__ unsigned long long part[256];
    const int nb = 1 << width, per = nb / 256, t = threadIdx.x;
    // thread t holds the digits nb - (t + 1) per .. nb - t per - 1, counted from the top
    const int top = nb - t * per - 1;
    unsigned long long mine = 0;
    for (int d = 0; d < per; d++) mine += S.hist[top - d];
    part[t] = mine;
    __syncthreads();
    // exclusive sum of the counts above this thread's digits (256 entries, a simple serial-per-thread scan)
    unsigned long long above = 0;
    for (int k = 0; k < t; k++) above += part[k];
    const unsigned long long remaining = S.remaining;
    __syncthreads();
    if (above < remaining && above + mine >= remaining) {
        int digit = top;
        for (int d = 0; d < per; d++, digit--) {
            const unsigned c = S.hist[digit];
            if (above + c >= remaining || digit == 0) break;
            above += c;
        }
        S.remaining = remaining - above;
        S.prefix |= (unsigned)digit << shift;
        S.mask |= (unsigned)(nb - 1) << shift;
    }
    __syncthreads();
    for (int i = t; i < nb; i += 256) S.hist[i] = 0;
}

__global__ void __launch_bounds__(256) sum_above_kernel(CvSlot *slots)
{
    CvSlot &S = slots[blockIdx.y];
    if (S.count <= S.k) return;
    const float threshold = __uint_as_float(S.prefix);
    const unsigned long long n = S.list_n;
    unsigned long long s = 0, c = 0;
    for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < n; i += (unsigned long long)gridDim.x * 256ull) {
        const float v = S.list[i];
        if (v > threshold) {
            s += __float2ull_rn(__fmul_rn(v, 16777216.0f));
            c++;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0 && c) {
        atomicAdd(&S.above_fx, s);
        atomicAdd(&S.above_n, c);
    }
}

__global__ void score_kernel(const __grid_constant__ ScoreBatch b)
{
    const int j = threadIdx.x;
    if (j >= b.njobs) return;
    const ScoreJob &J = b.job[j];
    const double kScaleWeight[kScales] = {16.0, 8.0, 4.0, 2.0, 1.0};
    double total = 0.0;
    for (int s = 0; s < kScales; s++) {
        const CvSlot &S = b.slots[J.first_slot + s];
        const double k = __ull2double_rn(S.k);
        double pooled;
        if (S.count <= S.k) {
            pooled = __ddiv_rn(__dmul_rn(__ull2double_rn(S.sum_fx), 1.0 / 16777216.0), k);
        } else {
            const double above = __dmul_rn(__ull2double_rn(S.above_fx), 1.0 / 16777216.0);
            const double rest = __dmul_rn(__ull2double_rn(S.k - S.above_n), (double)__uint_as_float(S.prefix));
            pooled = __ddiv_rn(__dadd_rn(above, rest), k);
        }
        total = __dadd_rn(total, __dmul_rn(pooled, kScaleWeight[s]));
        J.score[1 + s] = pooled;
    }
    const int odd = 2 * (J.window >> 1) + 1;
    const double score = __ddiv_rn(total, (double)(odd * odd));
    J.score[0] = score < 1000.0 ? score : 1000.0;
}

}  // namespace

cudaError_t launch_prep0(const Prep0Batch &b, cudaStream_t s)
{
    if (b.total_tiles <= 0) return cudaSuccess;
    prep0_kernel<<<b.total_tiles, 256, 0, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_decimate_mode(const DecBatch &b, cudaStream_t s)
{
    if (b.total_blocks <= 0) return cudaSuccess;
    decimate_mode_kernel<<<b.total_blocks, 256, 0, s>>>(b);
    return cudaGetLastError();
}

size_t cvalues_smem_bytes(int max_pad) { return cv_layout(max_pad).total; }

cudaError_t launch_cvalues(const CvBatch &b, cudaStream_t s)
{
    if (b.total_tiles <= 0) return cudaSuccess;
    const size_t smem = cvalues_smem_bytes(b.max_pad);
    cudaError_t e = cudaFuncSetAttribute(cvalues_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cvalues_kernel<<<b.total_tiles, kCvThreads, smem, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_slots_reset(CvSlot *slots, int nslots, const unsigned long long *n, const unsigned long long *k,
                               cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    slots_reset_kernel<<<nslots, 256, 0, s>>>(slots, nslots, n, k);
    return cudaGetLastError();
}

cudaError_t launch_select_round(CvSlot *slots, int nslots, int shift, int width, cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    select_hist_kernel<<<dim3(64, nslots), 256, 0, s>>>(slots, shift, width);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    select_pick_kernel<<<nslots, 256, 0, s>>>(slots, shift, width);
    return cudaGetLastError();
}

cudaError_t launch_sum_above(CvSlot *slots, int nslots, cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    sum_above_kernel<<<dim3(64, nslots), 256, 0, s>>>(slots);
    return cudaGetLastError();
}

cudaError_t launch_score(const ScoreBatch &b, cudaStream_t s)
{
    if (b.njobs <= 0) return cudaSuccess;
    score_kernel<<<1, 32, 0, s>>>(b);
    return cudaGetLastError();
}

const void *kernel_entry_prep0() { return (const void *)prep0_kernel; }
const void *kernel_entry_decimate_mode() { return (const void *)decimate_mode_kernel; }
const void *kernel_entry_cvalues() { return (const void *)cvalues_kernel; }

}  // namespace es
