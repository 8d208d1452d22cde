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
//  * select_hist_kernel / select_pick_kernel find the exact k-th largest value, and the sum above it, on the device
//    when more than k values are positive (no host round trips; the first radix digit is counted by the c-value
//    kernel), and score_kernel pools and weights the scales.
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
// Scales 0 and 1: src/kernels.cu:524-535 (from8), 14-40 (mask), 488-500 (mode), 43-53 (decimation), in one pass over a
// 64 x 64 tile of scale 0 and the 32 x 32 tile of scale 1 beneath it.
//
// The plane is staged with its margins (16-byte loads for tiles inside the picture; an 8-bit plane becomes 10-bit
// anti-dithered values in a second buffer). A warp per staged row packs the flat pixels into bit words by ballot. Each
// warp then walks 8 rows of the tile, a lane taking two neighbouring columns as the two halves of 32-bit words: the 7
// flat bits around each column come from one funnel shift and two popcounts and are summed over 7 rows as they go (both
// counts in one register), and the 3 x 3 mode filter reads both columns' neighbours with 32-bit loads. The scale-0 words at even
// positions, with a ring of them one step outside the tile (made on their own), then give the tile's scale-1 words
// (decimation and mode filter of the decimated values) without another read of scale 0.
// Staged region: columns x0-8 .. x0+71 (index x - (x0-8)), rows y0-5 .. y0+69 (index y - (y0-5)).
// ---------------------------------------------------------------------------------------------------------------
constexpr int kP0T = 64;                 // scale-0 tile side
constexpr int kP0C = 80, kP0R = 75;      // staged columns and rows
constexpr int kP0X = 8, kP0Y = 5;        // staged index of x0, y0
constexpr int kP0FR = 73, kP0FX = 5;     // flat rows y0-5 .. y0+67; bit i of a row is column x0-5+i
constexpr int kP0D = 34;                 // scale-0 words (x0-2+2X, y0-2+2Y), X, Y in 0 .. 33

// The mode of three values per 16-bit half (the smallest when all three differ), from SIMD minima and maxima only:
// with two or three equal values the repeated one is the median, and it equals the largest unless the pair is the
// two smallest, when it equals the smallest; with three different values the mode is the smallest. So the mode is
// the median where the median equals the largest, else the smallest. The halves' differences are never negative, so
// 32-bit subtraction keeps them apart, and "median below the largest" is a per-half nonzero test. (16-bit SIMD
// compares, and two scalar modes, measured slower.)
__device__ __forceinline__ uint32_t vmin_u16x2(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vmax_u16x2(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t mode3x2(uint32_t a, uint32_t b, uint32_t c)
{
    const uint32_t lo = vmin_u16x2(a, b), hi = vmax_u16x2(a, b);
    const uint32_t mn = vmin_u16x2(lo, c), mx = vmax_u16x2(hi, c), md = vmax_u16x2(lo, vmin_u16x2(hi, c));
    const uint32_t d = mx - md;  // per half, never negative: no borrow between the halves
    const uint32_t t = (((d & 0x7FFF7FFFu) + 0x7FFF7FFFu) | d) & 0x80008000u;  // bit 15 of a half: median below max
    const uint32_t nz = t | (t - (t >> 15));
    return mn + ((md - mn) & ~nz);
}

__global__ void __launch_bounds__(256, 5) prep0_kernel(const __grid_constant__ Prep0Batch b)
{
    __shared__ __align__(16) uint16_t buf[2][kP0R][kP0C];  // [0]: the staged plane; [1]: 8-bit planes at 10 bits
    __shared__ uint32_t flatbits[kP0FR][4];                // 3 words of bits and a zero word
    __shared__ uint16_t dw[kP0D][kP0D];                    // scale-0 words at even positions, for scale 1
    __shared__ uint32_t needbits[32];
    const int j = find_job(b.njobs, (int)blockIdx.x, [&](int k) { return b.job[k].first_tile; });
    const Prep0Job &J = b.job[j];
    const int t = blockIdx.x - J.first_tile, w = J.w, h = J.h, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int x0 = (t % J.tiles_x) * kP0T, y0 = (t / J.tiles_x) * kP0T;
    const int xs = x0 - kP0X, ys = y0 - kP0Y;
    if (J.feat && b.need_span < 0) {  // the codes that need c-values when they are no single range: bit c of word
                                      // c / 32 (warp w makes words w, w + 8, ...)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int code = (warp + 8 * k) * 32 + lane;
            const unsigned m = __ballot_sync(0xffffffffu, code < b.band.band_size && needs_cvalue(code, b.band));
            if (lane == 0) needbits[warp + 8 * k] = m;
        }
    }
    if (tid < kP0FR) flatbits[tid][3] = 0;
    const bool inside = xs >= 0 && xs + kP0C <= w && ys >= 0 && ys + kP0R <= h && (J.pitch & 7) == 0 && (((uintptr_t)J.img) & 15) == 0;
    if (inside) {
        for (int i = tid; i < kP0R * (kP0C / 8); i += 256) {
            const int r = i / (kP0C / 8), q = i - r * (kP0C / 8);
            *(uint4 *)&buf[0][r][8 * q] = __ldg((const uint4 *)(J.img + (size_t)(ys + r) * J.pitch + xs) + q);
        }
    } else {
        for (int i = tid; i < kP0R * kP0C; i += 256) {
            const int r = i / kP0C, c = i - r * kP0C, x = xs + c, y = ys + r;
            buf[0][r][c] = (x >= 0 && x < w && y >= 0 && y < h) ? J.img[(size_t)y * J.pitch + x] : (uint16_t)0;
        }
    }
    __syncthreads();
    // preprocessed values of x0-5 .. x0+68, y0-5 .. y0+68: an 8-bit plane at 10 bits, the mean of the 2 x 2 block to
    // the lower right (pairs on the last row and column); a 10-bit plane as staged (0 outside the picture)
    const int sel = J.depth == 8 ? 1 : 0;
    if (sel) {
        for (int i = tid; i < 74 * 74; i += 256) {
            const int r = i / 74, c = 3 + (i - r * 74), x = xs + c, y = ys + r;
            unsigned v = 0;
            if (x >= 0 && x < w && y >= 0 && y < h) {
                const unsigned a = (unsigned)buf[0][r][c] << 2;
                if (x < w - 1 && y < h - 1)
                    v = (a + ((unsigned)buf[0][r][c + 1] << 2) + ((unsigned)buf[0][r + 1][c] << 2) + ((unsigned)buf[0][r + 1][c + 1] << 2)) >> 2;
                else if (y < h - 1) v = (a + ((unsigned)buf[0][r + 1][c] << 2)) >> 1;
                else if (x < w - 1) v = (a + ((unsigned)buf[0][r][c + 1] << 2)) >> 1;
                else v = a;
            }
            buf[1][r][c] = (uint16_t)v;
        }
        __syncthreads();
    }
    // flat: equal to the right and lower neighbours (the last column / row count as equal); nothing outside. A warp
    // takes whole flat rows, 3 ballots of 32 columns each (73 columns used).
    {
        const bool interior = x0 >= 5 && x0 + kP0T + 4 < w && y0 >= 5 && y0 + kP0T + 4 < h;
        for (int q = warp; q < kP0FR; q += 8) {
            const uint16_t *row = buf[sel][q], *nxt = buf[sel][q + 1];
            const int y = ys + q;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const int i = 32 * k + lane, c = i + (kP0X - kP0FX), x = x0 - kP0FX + i;
                bool f = false;
                if (k < 2 || i < kP0FR) {
                    const uint16_t v = row[c];
                    if (interior) f = v == row[c + 1] && v == nxt[c];
                    else if (x >= 0 && x < w && y >= 0 && y < h)
                        f = (x == w - 1 || v == row[c + 1]) && (y == h - 1 || v == nxt[c]);
                }
                const uint32_t word = __ballot_sync(0xffffffffu, f);
                if (lane == k) flatbits[q][k] = word;
            }
        }
    }
    __syncthreads();

    // the walk: warp g makes rows y0 + 8 g .. + 7, lane l columns x0 + 2 l and + 1
    const int x = x0 + 2 * lane, g = warp;
    const int kw = (2 * lane + 2) >> 5, sh = (2 * lane + 2) & 31;  // flat bit of column x - 3
    auto h7 = [&](int q) -> uint32_t {  // flat counts of the 7 columns around x and x + 1 in flat row q, as halves
        const uint32_t bits = __funnelshift_r(flatbits[q][kw], flatbits[q][kw + 1], sh);
        return (uint32_t)__popc(bits & 0x7Fu) | ((uint32_t)__popc((bits >> 1) & 0x7Fu) << 16);
    };
    // columns x and x + 1 at a picture edge keep their own value in the horizontal mode
    const uint32_t edge = ((x == 0 || x == w - 1) ? 0x0000FFFFu : 0u) | ((x + 1 == w - 1) ? 0xFFFF0000u : 0u);
    const int c = x - xs;  // staged column of x (even)
    auto pair = [&](int r, int cc) -> uint32_t { return *(const uint32_t *)&buf[sel][r][cc]; };
    auto hmode = [&](int y) -> uint32_t {  // horizontal modes of x and x + 1 in picture row y
        const int r = y - ys;
        const uint32_t l2 = pair(r, c - 2), m2 = pair(r, c), r2 = pair(r, c + 2);
        const uint32_t left = __byte_perm(l2, m2, 0x5432), right = __byte_perm(m2, r2, 0x5432);
        return (m2 & edge) | (mode3x2(left, m2, right) & ~edge);
    };
    const bool feat = J.feat != nullptr;  // the same for the whole block
    // mask bit 15 of each half where the count exceeds mask_index: counts <= 49 and 0x7FFF - mask_index added per
    // half reach bit 15 exactly then, without a carry into the other half
    const uint32_t idx2 = (0x7FFFu - (uint32_t)J.mask_index) * 0x10001u;
    const bool vec_store = (w & 1) == 0 && (((uintptr_t)J.word) & 3) == 0;
    const bool need_range = b.need_span >= 0;
    const int yb = y0 + 8 * g;
    uint32_t hv[14];  // h7 of flat rows yb-3 .. yb+10 (flat row index y - (y0-5))
    uint32_t cnt = 0;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        hv[q] = h7(yb - 3 - ys + q);
        cnt += hv[q];
    }
    uint32_t m0 = hmode(yb - 1), m1 = hmode(yb);
    // features of this lane's two columns over the current 4 rows, as 16-bit pairs (a pair holds 2 rows of sums of
    // values below 2^15, then it is folded into fsum; counts up to 4)
    uint32_t fsum = 0, fsum2 = 0, fmask2 = 0, fn2 = 0;
    // the smallest (value - need_lo) of the lane's masked pixels per half, wrapping for values below need_lo: a pixel
    // needs a c-value when it is at most need_span (unmasked pixels count as 0x8000, above any span)
    const uint32_t lo2 = (uint32_t)(b.need_lo & 0x7FFF) * 0x10001u;
    uint32_t dmin = 0xFFFFFFFFu;
    bool need = false;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int y = yb + i;
        hv[i + 6] = h7(y + 3 - ys);
        cnt += hv[i + 6];
        const uint32_t m2 = hmode(y + 1);
        uint32_t v2 = mode3x2(m0, m1, m2);
        if (y == 0 || y == h - 1) v2 = pair(y - ys, c);  // (the same for the whole warp)
        const uint32_t mk = (cnt + idx2) & 0x80008000u;
        const uint32_t word2 = v2 | mk;
        if (y < h) {
            if (vec_store && x + 1 < w) {
                *(uint32_t *)(J.word + (size_t)y * w + x) = word2;
            } else {
                if (x < w) J.word[(size_t)y * w + x] = (uint16_t)word2;
                if (x + 1 < w) J.word[(size_t)y * w + x + 1] = (uint16_t)(word2 >> 16);
            }
            if ((i & 1) == 0 && x < w) dw[4 * g + i / 2 + 1][lane + 1] = (uint16_t)word2;
            if (feat) {
                const uint32_t ok = (x + 1 < w) ? 0xFFFFFFFFu : (x < w ? 0x0000FFFFu : 0u);
                const uint32_t mm = (mk >> 15) & ok & 0x10001u;
                fsum2 += v2 & ok;
                if (i & 1) {
                    fsum += (fsum2 & 0xFFFFu) + (fsum2 >> 16);
                    fsum2 = 0;
                }
                fmask2 += mm;
                fn2 += ok & 0x10001u;
                uint32_t hit = 0;
                if (need_range) {
                    // per half (value | 0x8000) - need_lo never borrows; flipping bit 15 leaves value - need_lo
                    // modulo 2^16, which is at most need_span exactly when the value is in the range
                    const uint32_t d = ((((v2 | 0x80008000u) - lo2) & (mm * 0xFFFFu)) ^ 0x80008000u);
                    dmin = vmin_u16x2(dmin, d);
                } else {
                    for (int k = 0; k < 2; k++) {
                        const uint16_t code = code_of((uint16_t)(word2 >> (16 * k)), b.band);
                        if (((ok >> (16 * k)) & 1u) && code != kNone && ((needbits[code >> 5] >> (code & 31)) & 1u)) hit = 1;
                    }
                }
                need |= hit != 0;
            }
        }
        cnt -= hv[i];
        m0 = m1;
        m1 = m2;
        if (feat && (i & 3) == 3) {
            // the 4 x 4 block of columns x - 2 l % 4 .. + 3: this lane's pair and its neighbour's
            fsum += (fsum2 & 0xFFFFu) + (fsum2 >> 16);  // a last row past the picture leaves a pair unfolded
            uint32_t fmask = (fmask2 & 0xFFFFu) + (fmask2 >> 16), fn = (fn2 & 0xFFFFu) + (fn2 >> 16);
            fsum += __shfl_xor_sync(0xffffffffu, fsum, 1);
            fmask += __shfl_xor_sync(0xffffffffu, fmask, 1);
            fn += __shfl_xor_sync(0xffffffffu, fn, 1);
            const int fw = (w + 3) / 4, fh = (h + 3) / 4, u = x >> 2, v4 = (y - 3) >> 2;
            if ((lane & 1) == 0 && u < fw && v4 < fh) {
                // (sum / n - 512) / 256 rounded once to float; for a whole block (n = 16) every step is exact in
                // float, so the double path is needed only at the picture's edges
                const float f0 = fn == 16 ? __fmul_rn(__fsub_rn(__fmul_rn((float)fsum, 0.0625f), 512.0f), 0.00390625f)
                                          : fn ? (float)(((double)fsum / (double)fn - 512.0) / 256.0) : 0.0f;
                J.feat[(size_t)v4 * fw + u] = make_float2(f0, __fmul_rn((float)fmask, 0.0625f));
            }
            fsum = fsum2 = fmask2 = fn2 = 0;
        }
    }
    if (feat) {
        if (need_range) need = (dmin & 0xFFFFu) <= (unsigned)b.need_span || (dmin >> 16) <= (unsigned)b.need_span;
        need = __syncthreads_or(need);
        if (tid == 0) J.need[t] = need ? 1u : 0u;
    }
    if (!J.word1) return;  // the same for the whole block

    // the ring of scale-0 words one step outside the tile that scale 1 reads: rows y0-2 and y0+64 (X = 0 .. 33), then
    // columns x0-2 and x0+64 (Y = 1 .. 32)
    if (tid < 2 * kP0D + 2 * (kP0D - 2)) {
        int X, Y;
        if (tid < 2 * kP0D) {
            X = tid % kP0D;
            Y = tid < kP0D ? 0 : kP0D - 1;
        } else {
            Y = 1 + (tid - 2 * kP0D) % (kP0D - 2);
            X = tid - 2 * kP0D < kP0D - 2 ? 0 : kP0D - 1;
        }
        const int px = x0 - 2 + 2 * X, py = y0 - 2 + 2 * Y;
        if (px >= 0 && px < w && py >= 0 && py < h) {
            const int bi = px - (x0 - kP0FX) - 3, bw = bi >> 5, bs = bi & 31;
            int n = 0;
#pragma unroll
            for (int dy = -3; dy <= 3; dy++)
                n += __popc(__funnelshift_r(flatbits[py + dy - ys][bw], flatbits[py + dy - ys][bw + 1], bs) & 0x7Fu);
            const int pc = px - xs;
            auto hm1 = [&](int yy) -> uint16_t {
                const uint16_t *row = buf[sel][yy - ys];
                return (px == 0 || px == w - 1) ? row[pc] : (uint16_t)(mode3x2(row[pc - 1], row[pc], row[pc + 1]) & 0xFFFFu);
            };
            const uint16_t v = (py == 0 || py == h - 1) ? buf[sel][py - ys][pc]
                                                        : (uint16_t)(mode3x2(hm1(py - 1), hm1(py), hm1(py + 1)) & 0xFFFFu);
            dw[Y][X] = (uint16_t)(v | (n > J.mask_index ? kMaskBit : 0));
        }
    }
    __syncthreads();
    // scale 1: the decimated words dw, mode-filtered (rows and columns at the picture's edges keep their value); thread
    // (cx, q) makes column cx of rows 4 q .. 4 q + 3 of the 32 x 32 tile
    {
        const int w1 = J.w1, h1 = J.h1, X0 = x0 >> 1, Y0 = y0 >> 1;
        const int cx = tid & 31, q = tid >> 5, X1 = X0 + cx;
        if (X1 < w1) {
            const int X = cx + 1;
            const bool edge1 = X1 == 0 || X1 == w1 - 1;
            auto val = [&](int Y, int XX) -> uint32_t { return dw[Y][XX] & 0x7FFFu; };
            uint32_t hm[6];  // rows Y0 + 4 q - 1 .. + 4 (dw rows 4 q .. 4 q + 5)
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const int Y = 4 * q + k, Yp = Y0 + Y - 1;
                hm[k] = (Yp < 0 || Yp >= h1) ? 0u : edge1 ? val(Y, X) : (mode3x2(val(Y, X - 1), val(Y, X), val(Y, X + 1)) & 0xFFFFu);
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int Y1 = Y0 + 4 * q + i;
                if (Y1 >= h1) break;
                const uint16_t word = dw[4 * q + i + 1][X];
                const uint32_t v = (Y1 == 0 || Y1 == h1 - 1) ? (uint32_t)(word & 0x7FFFu) : (mode3x2(hm[i], hm[i + 1], hm[i + 2]) & 0xFFFFu);
                J.word1[(size_t)Y1 * w1 + X1] = (uint16_t)(v | (word & kMaskBit));
            }
        }
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
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) S.dsum[i] = 0;
    if (threadIdx.x == 0) {
        S.sum_fx = S.count = S.list_n = 0;
        S.n = n[s];
        S.k = k[s];
        S.remaining = k[s];
        S.above_fx = S.above_n = 0;
        S.prefix = S.mask = 0;
    }
}

// A positive c-value in units of 2^-24 (exact: c-values are multiples of 2^-24).
__device__ __forceinline__ unsigned long long fx_of(unsigned bits) { return __float2ull_rn(__fmul_rn(__uint_as_float(bits), 16777216.0f)); }

// One radix round over every slot whose positive count exceeds k (the first round's counts come from the c-value
// kernel); block b takes the b-th share of each such slot's list. One block of kSelThreads per SM: each block merges
// one shared histogram per slot into the slot's, so fewer, larger blocks mean fewer global atomics for the same reads.
// The last round (last = 1) also sums, per digit, the values that match the prefix (they are equal when their digits
// are), and the values whose prefix is greater than the selected one (all of them lie above the k-th value).
constexpr int kSelThreads = 1024, kSelBlocks = 148;

__global__ void __launch_bounds__(kSelThreads) select_hist_kernel(CvSlot *slots, int nslots, int shift, int width, int last)
{
    __shared__ unsigned hist[2048];
    __shared__ unsigned long long dsum[1024];
    const int nb = 1 << width;
    for (int sl = 0; sl < nslots; sl++) {
        CvSlot &S = slots[sl];
        if (S.count <= S.k) continue;  // the same for the whole block
        for (int i = threadIdx.x; i < nb; i += kSelThreads) {
            hist[i] = 0;
            if (last) dsum[i] = 0;
        }
        __syncthreads();
        const unsigned *v = (const unsigned *)S.list;
        const unsigned long long n = S.list_n, n4 = n / 4, stride = (unsigned long long)gridDim.x * kSelThreads;
        const unsigned mask = S.mask, prefix = S.prefix;
        unsigned long long above_fx = 0, above_n = 0;
        // neighbouring c-values of the list are often equal (they come from the same tile), so each thread adds runs
        // of equal digits at once; 4 values per 16-byte load
        unsigned lastd = 0, run = 0;
        auto flush_run = [&]() {
            atomicAdd(&hist[lastd], run);
            if (last) atomicAdd(&dsum[lastd], (unsigned long long)run * fx_of(prefix | lastd));
        };
        auto add = [&](unsigned bits) {
            if ((bits & mask) != prefix) {
                if (last && (bits & mask) > prefix) {
                    above_fx += fx_of(bits);
                    above_n++;
                }
                return;
            }
            const unsigned d = (bits >> shift) & (unsigned)(nb - 1);
            if (run && d == lastd) {
                run++;
                return;
            }
            if (run) flush_run();
            lastd = d;
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
        if (run) flush_run();
        if (last) {
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                above_fx += __shfl_down_sync(0xffffffffu, above_fx, o);
                above_n += __shfl_down_sync(0xffffffffu, above_n, o);
            }
            if ((threadIdx.x & 31) == 0 && above_n) {
                atomicAdd(&S.above_fx, above_fx);
                atomicAdd(&S.above_n, above_n);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += kSelThreads) {
            if (hist[i]) atomicAdd(&S.hist[i], hist[i]);
            if (last && dsum[i]) atomicAdd(&S.dsum[i], dsum[i]);
        }
        __syncthreads();
    }
}

// Picks the digit of the k-th largest value from a round's counts; the last round then adds the values of the greater
// digits to the sum and count above it.
__global__ void __launch_bounds__(256) select_pick_kernel(CvSlot *slots, int shift, int width, int last)
{
    CvSlot &S = slots[blockIdx.x];
    if (S.count <= S.k) return;
    __shared__ unsigned long long part[256];
    __shared__ int picked;
    const int nb = 1 << width, per = nb / 256, t = threadIdx.x;
    if (t == 0) picked = 0;
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
        picked = digit;
    }
    __syncthreads();
    if (last) {
        // the values of the digits above the picked one: their sums and counts, added to those of greater prefixes
        const int D = picked;
        unsigned long long fx = 0, cnt = 0;
        for (int d = D + 1 + t; d < nb; d += 256) {
            fx += S.dsum[d];
            cnt += S.hist[d];
        }
        part[t] = fx;
        __syncthreads();
        for (int o = 128; o; o >>= 1) {
            if (t < o) part[t] += part[t + o];
            __syncthreads();
        }
        const unsigned long long fx_all = part[0];
        __syncthreads();
        part[t] = cnt;
        __syncthreads();
        for (int o = 128; o; o >>= 1) {
            if (t < o) part[t] += part[t + o];
            __syncthreads();
        }
        if (t == 0) {
            S.above_fx += fx_all;
            S.above_n += part[0];
        }
        __syncthreads();
        for (int i = t; i < nb; i += 256) S.dsum[i] = 0;
    }
    for (int i = t; i < nb; i += 256) S.hist[i] = 0;
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

cudaError_t launch_topk(CvSlot *slots, int nslots, cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    static const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
    for (int round = 0; round < 3; round++) {
        const int last = round == 2;
        if (round > 0) {  // the first round's counts were made by the c-value kernel
            LaunchTimer t("cambi_select_hist", s);
            select_hist_kernel<<<kSelBlocks, kSelThreads, 0, s>>>(slots, nslots, shifts[round], widths[round], last);
        }
        cudaError_t e = round > 0 ? after_launch() : cudaSuccess;
        if (e != cudaSuccess) return e;
        {
            LaunchTimer t("cambi_select_pick", s);
            select_pick_kernel<<<nslots, 256, 0, s>>>(slots, shifts[round], widths[round], last);
        }
        e = after_launch();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
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
