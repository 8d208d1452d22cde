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
//  * the c-values themselves are in cvalues_kernels.cu;
//  * select_round_kernel / select_pick_kernel / sum_above_kernel find the exact k-th largest value on the device when
//    more than k values are positive (no host round trips), and score_kernel pools and weights the scales.
#include "cambi_codes.h"
#include "es_kernels.h"

namespace es {
namespace {

// The mode of three values (the smallest when all differ), as selects rather than branches: neighbouring pixels of a
// warp take different cases.
__device__ __forceinline__ uint16_t mode3(uint16_t a, uint16_t b, uint16_t c)
{
    const unsigned mn = min((unsigned)a, min((unsigned)b, (unsigned)c));
    const unsigned bc = b == c ? (unsigned)b : mn;
    return (uint16_t)((a == b || a == c) ? (unsigned)a : bc);
}

// ---------------------------------------------------------------------------------------------------------------
// Scale 0: src/kernels.cu:524-535 (from8), 14-40 (mask), 488-500 (mode), in one pass over a 64 x 64 tile.
// The plane is staged with its margins (8-byte loads for tiles inside the picture); an 8-bit plane is turned into
// 10-bit anti-dithered values, a 10-bit one is used as staged. A warp per row packs the flat pixels into bit words by
// ballot; each thread then walks 16 rows of one column, counting the 7 flat bits around each pixel with a funnel shift
// and a popcount, summing 7 rows as it goes, and applying the separable mode filter from running row modes.
// Staged region: columns x0-4 .. x0+71 (index x - (x0-4)), rows y0-3 .. y0+68 (index y - (y0-3)).
// ---------------------------------------------------------------------------------------------------------------
constexpr int kP0T = 64;                    // output tile side
constexpr int kP0C = kP0T + 12, kP0R = kP0T + 8;  // staged columns (76) and rows (72)
constexpr int kP0F = kP0T + 6;              // flat pixels per side: x0-3 .. x0+66, y0-3 .. y0+66

__global__ void __launch_bounds__(256, 5) prep0_kernel(const __grid_constant__ Prep0Batch b)
{
    __shared__ __align__(16) uint16_t raw[kP0R][kP0C];
    __shared__ __align__(16) uint16_t pre8[kP0R - 1][kP0C];
    __shared__ uint32_t flatbits[kP0F][3];
    __shared__ uint32_t needbits[32];
    const int j = find_job(b.njobs, (int)blockIdx.x, [&](int k) { return b.job[k].first_tile; });
    const Prep0Job &J = b.job[j];
    const int t = blockIdx.x - J.first_tile, w = J.w, h = J.h, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int x0 = (t % J.tiles_x) * kP0T, y0 = (t / J.tiles_x) * kP0T;
    const int xs = x0 - 4, ys = y0 - 3;
    if (J.feat && b.need_span < 0) {  // the codes that need c-values when they are no single range: bit c of word
                                      // c / 32 (warp w makes words w, w + 8, ...)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int code = (warp + 8 * k) * 32 + lane;
            const unsigned m = __ballot_sync(0xffffffffu, code < b.band.band_size && needs_cvalue(code, b.band));
            if (lane == 0) needbits[warp + 8 * k] = m;
        }
    }
    const bool inside = xs >= 0 && xs + kP0C <= w && ys >= 0 && ys + kP0R <= h && (J.pitch & 3) == 0 && (((uintptr_t)J.img) & 7) == 0;
    if (inside) {
        for (int i = tid; i < kP0R * (kP0C / 4); i += 256) {
            const int r = i / (kP0C / 4), q = i - r * (kP0C / 4);
            *(uint2 *)&raw[r][4 * q] = __ldg((const uint2 *)(J.img + (size_t)(ys + r) * J.pitch + xs) + q);
        }
    } else {
        for (int i = tid; i < kP0R * kP0C; i += 256) {
            const int r = i / kP0C, c = i - r * kP0C, x = xs + c, y = ys + r;
            raw[r][c] = (x >= 0 && x < w && y >= 0 && y < h) ? J.img[(size_t)y * J.pitch + x] : (uint16_t)0;
        }
    }
    __syncthreads();
    // preprocessed values of x0-4 .. x0+71, y0-3 .. y0+67: an 8-bit plane at 10 bits, the mean of the 2 x 2 block to
    // the lower right (pairs on the last row and column); a 10-bit plane as staged (0 outside the picture)
    if (J.depth == 8) {
        for (int i = tid; i < (kP0R - 1) * (kP0C - 1); i += 256) {
            const int r = i / (kP0C - 1), c = i - r * (kP0C - 1), x = xs + c, y = ys + r;
            unsigned v = 0;
            if (x >= 0 && x < w && y >= 0 && y < h) {
                const unsigned a = (unsigned)raw[r][c] << 2;
                if (x < w - 1 && y < h - 1)
                    v = (a + ((unsigned)raw[r][c + 1] << 2) + ((unsigned)raw[r + 1][c] << 2) + ((unsigned)raw[r + 1][c + 1] << 2)) >> 2;
                else if (y < h - 1) v = (a + ((unsigned)raw[r + 1][c] << 2)) >> 1;
                else if (x < w - 1) v = (a + ((unsigned)raw[r][c + 1] << 2)) >> 1;
                else v = a;
            }
            pre8[r][c] = (uint16_t)v;
        }
        __syncthreads();
        // back into the staged plane, so every later read names one shared array (32-bit shared addressing)
        for (int i = tid; i < (kP0R - 1) * (kP0C - 1); i += 256) {
            const int r = i / (kP0C - 1), c = i - r * (kP0C - 1);
            raw[r][c] = pre8[r][c];
        }
        __syncthreads();
    }
    auto &pre = raw;
    // flat: equal to the right and lower neighbours (the last column / row count as equal); nothing outside
    const bool interior = x0 >= 3 && x0 + kP0T + 3 < w && y0 >= 3 && y0 + kP0T + 3 < h;
    for (int q = warp; q < kP0F; q += 8) {
        const int y = ys + q;
        uint32_t words[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int c = lane + 32 * k, x = x0 - 3 + c;  // staged column c + 1
            bool f = false;
            if (c < kP0F) {
                const uint16_t v = pre[q][c + 1];
                if (interior) f = v == pre[q][c + 2] && v == pre[q + 1][c + 1];
                else if (x >= 0 && x < w && y >= 0 && y < h)
                    f = (x == w - 1 || v == pre[q][c + 2]) && (y == h - 1 || v == pre[q + 1][c + 1]);
            }
            words[k] = __ballot_sync(0xffffffffu, f);
        }
        if (lane < 3) flatbits[q][lane] = lane == 0 ? words[0] : lane == 1 ? words[1] : words[2];
    }
    __syncthreads();
    const int c = tid & (kP0T - 1), g = tid >> 6, x = x0 + c;
    const bool feat = J.feat != nullptr;  // the same for the whole block
    if (x >= w && !feat) return;
    // flat count of the 7 columns around x in flat row 16 g + q (bit c of a row is column x - 3), and the horizontal
    // mode of picture row y0 + 16 g - 1 + k (staged row 16 g + 2 + k), each made once as the window moves down and
    // kept only while the window holds it, so few registers stay live and 5 blocks share an SM
    const int kw = c >> 5, sh = c & 31;
    auto h7 = [&](int q) { return __popc(__funnelshift_r(flatbits[16 * g + q][kw], flatbits[16 * g + q][kw + 1], sh) & 0x7Fu); };
    const bool edge_x = x == 0 || x == w - 1;
    auto hmode = [&](int k) -> uint16_t {
        const uint16_t *row = pre[16 * g + 2 + k];
        return edge_x ? row[c + 4] : mode3(row[c + 3], row[c + 4], row[c + 5]);
    };
    int cnt = 0, hv[22];  // hv[q] = h7(q), each kept for the 7 rows of the window it enters
#pragma unroll
    for (int q = 0; q < 6; q++) {
        hv[q] = h7(q);
        cnt += hv[q];
    }
    uint16_t m0 = hmode(0), m1 = hmode(1);
    // features of the 4 x 4 blocks (the proposal's block_features): value sum, masked and counted pixels of this
    // column's 4 rows, then summed over the block's 4 columns (lanes c .. c + 3 of one warp)
    unsigned fpack = 0;  // value sum (bits 0-15, at most 16 x 1023), masked pixels (16-20), counted pixels (24-28)
    bool need = false;
    const bool need_range = b.need_span >= 0;
    const unsigned need_lo = (unsigned)b.need_lo, need_span = (unsigned)b.need_span;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        hv[i + 6] = h7(i + 6);
        cnt += hv[i + 6];
        const uint16_t m2 = hmode(i + 2);
        const int y = y0 + 16 * g + i;
        if (y < h && x < w) {
            const uint16_t v = (y == 0 || y == h - 1) ? pre[16 * g + 3 + i][c + 4] : mode3(m0, m1, m2);
            const uint16_t word = (uint16_t)(v | (cnt > J.mask_index ? kMaskBit : 0));
            J.word[(size_t)y * w + x] = word;
            if (feat) {
                fpack += (unsigned)v | ((unsigned)(word >> 15) << 16) | (1u << 24);
                if (need_range) {
                    need |= (word >> 15) && (unsigned)v - need_lo <= need_span;
                } else {
                    const uint16_t code = code_of(word, b.band);
                    need |= code != kNone && ((needbits[code >> 5] >> (code & 31)) & 1u);
                }
            }
        }
        cnt -= hv[i];
        m0 = m1;
        m1 = m2;
        if (feat && (i & 3) == 3) {
            fpack += __shfl_xor_sync(0xffffffffu, fpack, 1);
            fpack += __shfl_xor_sync(0xffffffffu, fpack, 2);
            const int fw = (w + 3) / 4, fh = (h + 3) / 4, u = x >> 2, v4 = (y0 + 16 * g + i - 3) >> 2;
            if ((c & 3) == 0 && u < fw && v4 < fh) {
                const unsigned fsum = fpack & 0xFFFFu, fmask = (fpack >> 16) & 0xFFu, fn = fpack >> 24;
                // (sum / n - 512) / 256 rounded once to float; for a whole block (n = 16) every step is exact in
                // float, so the double path is needed only at the picture's edges
                const float f0 = fn == 16 ? __fmul_rn(__fsub_rn(__fmul_rn((float)fsum, 0.0625f), 512.0f), 0.00390625f)
                                          : fn ? (float)(((double)fsum / (double)fn - 512.0) / 256.0) : 0.0f;
                J.feat[(size_t)v4 * fw + u] = make_float2(f0, __fmul_rn((float)fmask, 0.0625f));
            }
            fpack = 0;
        }
    }
    if (feat) {
        need = __syncthreads_or(need);
        if (tid == 0) J.need[t] = need ? 1u : 0u;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Scales 1-4: src/kernels.cu:43-53 (decimate) and 488-500 (mode) on the decimated picture, mask decimated alongside.
// A block of 256 threads makes a 64 x 16 tile: the decimated words of the tile and a 1-pixel margin (the even rows
// and columns of the previous scale, 4-byte loads keeping the even half) are staged in shared memory; thread (c, g)
// then makes column c of rows 4 g .. 4 g + 3 from 6 horizontal modes.
// ---------------------------------------------------------------------------------------------------------------
constexpr int kDTW = 64, kDTH = 16;

__global__ void __launch_bounds__(256) decimate_mode_kernel(const __grid_constant__ DecBatch b)
{
    __shared__ uint16_t d[kDTH + 2][kDTW + 2];
    const int j = find_job(b.njobs, (int)blockIdx.x, [&](int k) { return b.job[k].first_block; });
    const DecJob &J = b.job[j];
    const int w = J.w, h = J.h, tiles_x = (w + kDTW - 1) / kDTW, t = blockIdx.x - J.first_block;
    const int x0 = (t % tiles_x) * kDTW, y0 = (t / tiles_x) * kDTH;
    for (int i = threadIdx.x; i < (kDTH + 2) * (kDTW + 2); i += 256) {
        const int r = i / (kDTW + 2), c = i - r * (kDTW + 2), X = x0 - 1 + c, Y = y0 - 1 + r;
        uint16_t v = 0;
        if (X >= 0 && X < w && Y >= 0 && Y < h) {  // word (2 X, 2 Y) of the previous scale
            const uint16_t *p = J.src + (size_t)(2 * Y) * J.sw + 2 * X;
            // the low half of a 4-byte load, unless the word ends an odd-width row (the high half would be past it)
            v = 2 * X + 1 < J.sw ? (uint16_t)(__ldg((const unsigned *)p) & 0xFFFFu) : *p;
        }
        d[r][c] = v;
    }
    __syncthreads();
    const int c = threadIdx.x & (kDTW - 1), r0 = (threadIdx.x >> 6) * 4, x = x0 + c;
    if (x >= w) return;
    auto val = [&](int r, int cc) -> uint16_t { return d[r][cc] & 0x7FFF; };
    const bool edge_x = x == 0 || x == w - 1;
    uint16_t hm[6];  // horizontal modes of tile rows r0 - 1 .. r0 + 4 (staged rows r0 .. r0 + 5)
#pragma unroll
    for (int k = 0; k < 6; k++)
        hm[k] = edge_x ? val(r0 + k, c + 1) : mode3(val(r0 + k, c), val(r0 + k, c + 1), val(r0 + k, c + 2));
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int y = y0 + r0 + i;
        if (y >= h) break;
        const uint16_t word = d[r0 + i + 1][c + 1];
        const uint16_t v = (y == 0 || y == h - 1) ? (uint16_t)(word & 0x7FFF) : mode3(hm[i], hm[i + 1], hm[i + 2]);
        J.dst[(size_t)y * w + x] = (uint16_t)(v | (word & kMaskBit));
    }
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

// One radix round over every slot whose positive count exceeds k; block b takes the b-th share of each such slot's list.
// One block of kSelThreads per SM: each block merges one shared histogram per slot into the slot's, so fewer, larger
// blocks mean fewer global atomics for the same reads.
constexpr int kSelThreads = 1024, kSelBlocks = 148;

__global__ void __launch_bounds__(kSelThreads) select_hist_kernel(CvSlot *slots, int nslots, int shift, int width)
{
    __shared__ unsigned hist[2048];
    const int nb = 1 << width;
    for (int sl = 0; sl < nslots; sl++) {
        CvSlot &S = slots[sl];
        if (S.count <= S.k) continue;  // the same for the whole block
        for (int i = threadIdx.x; i < nb; i += kSelThreads) hist[i] = 0;
        __syncthreads();
        const unsigned *v = (const unsigned *)S.list;
        const unsigned long long n = S.list_n, n4 = n / 4, stride = (unsigned long long)gridDim.x * kSelThreads;
        const unsigned mask = S.mask, prefix = S.prefix;
        // neighbouring c-values of the list are often equal (they come from the same tile), so each thread adds runs
        // of equal digits at once; 4 values per 16-byte load
        unsigned last = 0, run = 0;
        auto add = [&](unsigned bits) {
            if ((bits & mask) != prefix) return;
            const unsigned d = (bits >> shift) & (unsigned)(nb - 1);
            if (run && d == last) {
                run++;
                return;
            }
            if (run) atomicAdd(&hist[last], run);
            last = d;
            run = 1;
        };
        // four 16-byte loads in flight per thread, then the rest one by one
        unsigned long long i = (unsigned long long)blockIdx.x * kSelThreads + threadIdx.x;
        for (; i + 3 * stride < n4; i += 4 * stride) {
            uint4 q[4];
#pragma unroll
            for (int u = 0; u < 4; u++) q[u] = __ldg((const uint4 *)v + i + u * stride);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                add(q[u].x);
                add(q[u].y);
                add(q[u].z);
                add(q[u].w);
            }
        }
        for (; i < n4; i += stride) {
            const uint4 q = __ldg((const uint4 *)v + i);
            add(q.x);
            add(q.y);
            add(q.z);
            add(q.w);
        }
        for (unsigned long long i = n4 * 4 + (unsigned long long)blockIdx.x * kSelThreads + threadIdx.x; i < n; i += stride) add(v[i]);
        if (run) atomicAdd(&hist[last], run);
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += kSelThreads)
            if (hist[i]) atomicAdd(&S.hist[i], hist[i]);
        __syncthreads();
    }
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

__global__ void __launch_bounds__(kSelThreads) sum_above_kernel(CvSlot *slots, int nslots)
{
    for (int sl = 0; sl < nslots; sl++) {
        CvSlot &S = slots[sl];
        if (S.count <= S.k) continue;
        const float threshold = __uint_as_float(S.prefix);
        const unsigned long long n = S.list_n, n4 = n / 4, stride = (unsigned long long)gridDim.x * kSelThreads;
        unsigned long long s = 0, c = 0;
        auto add = [&](float v) {
            if (v > threshold) {
                s += __float2ull_rn(__fmul_rn(v, 16777216.0f));
                c++;
            }
        };
        // four 16-byte loads in flight per thread, then the rest one by one
        unsigned long long i = (unsigned long long)blockIdx.x * kSelThreads + threadIdx.x;
        for (; i + 3 * stride < n4; i += 4 * stride) {
            float4 q[4];
#pragma unroll
            for (int u = 0; u < 4; u++) q[u] = __ldg((const float4 *)S.list + i + u * stride);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                add(q[u].x);
                add(q[u].y);
                add(q[u].z);
                add(q[u].w);
            }
        }
        for (; i < n4; i += stride) {
            const float4 q = __ldg((const float4 *)S.list + i);
            add(q.x);
            add(q.y);
            add(q.z);
            add(q.w);
        }
        for (unsigned long long i = n4 * 4 + (unsigned long long)blockIdx.x * kSelThreads + threadIdx.x; i < n; i += stride) add(S.list[i]);
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

cudaError_t launch_prep0(Prep0Batch &b, cudaStream_t s)
{
    int tiles = 0;
    for (int j = 0; j < b.njobs; j++) {
        Prep0Job &J = b.job[j];
        J.tiles_x = (J.w + kP0T - 1) / kP0T;
        J.first_tile = tiles;
        tiles += J.tiles_x * ((J.h + kP0T - 1) / kP0T);
    }
    b.total_tiles = tiles;
    if (b.total_tiles <= 0) return cudaSuccess;
    // the values whose codes need c-values, as one range when they are one (they are for CAMBI's thresholds)
    int lo = -1, hi = -2;
    bool one_range = true;
    for (int code = 0; code < b.band.band_size; code++) {
        if (!cvalue_dists(code, b.band)) continue;
        if (lo < 0) lo = code;
        else if (code != hi + 1) one_range = false;
        hi = code;
    }
    b.need_lo = lo < 0 ? 0 : lo + b.band.band_base;
    b.need_span = !one_range ? -1 : lo < 0 ? -1 : hi - lo;
    LaunchTimer t("cambi_prep0", s);
    prep0_kernel<<<b.total_tiles, 256, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_decimate_mode(DecBatch &b, cudaStream_t s)
{
    int blocks = 0;
    for (int j = 0; j < b.njobs; j++) {
        b.job[j].first_block = blocks;
        blocks += ((b.job[j].w + kDTW - 1) / kDTW) * ((b.job[j].h + kDTH - 1) / kDTH);
    }
    b.total_blocks = blocks;
    if (b.total_blocks <= 0) return cudaSuccess;
    LaunchTimer t("cambi_decimate_mode", s);
    decimate_mode_kernel<<<b.total_blocks, 256, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_slots_reset(CvSlot *slots, int nslots, const unsigned long long *n, const unsigned long long *k,
                               cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    LaunchTimer t("cambi_reset", s);
    slots_reset_kernel<<<nslots, 256, 0, s>>>(slots, nslots, n, k);
    return after_launch();
}

cudaError_t launch_select_round(CvSlot *slots, int nslots, int shift, int width, cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    {
        LaunchTimer t("cambi_select_hist", s);
        select_hist_kernel<<<kSelBlocks, kSelThreads, 0, s>>>(slots, nslots, shift, width);
    }
    cudaError_t e = after_launch();
    if (e != cudaSuccess) return e;
    LaunchTimer t("cambi_select_pick", s);
    select_pick_kernel<<<nslots, 256, 0, s>>>(slots, shift, width);
    return after_launch();
}

cudaError_t launch_sum_above(CvSlot *slots, int nslots, cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    LaunchTimer t("cambi_sum_above", s);
    sum_above_kernel<<<kSelBlocks, kSelThreads, 0, s>>>(slots, nslots);
    return after_launch();
}

cudaError_t launch_score(const ScoreBatch &b, cudaStream_t s)
{
    if (b.njobs <= 0) return cudaSuccess;
    LaunchTimer t("cambi_score", s);
    score_kernel<<<1, kScoreMaxJobs, 0, s>>>(b);
    return after_launch();
}

const void *kernel_entry_prep0() { return (const void *)prep0_kernel; }
const void *kernel_entry_decimate_mode() { return (const void *)decimate_mode_kernel; }

}  // namespace es
