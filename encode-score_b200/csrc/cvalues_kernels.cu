// CAMBI c-values for sm_100a: src/kernels.cu:113-278 (cambi.c's c_value_pixel over the (2 pad + 1)^2 window of every
// masked pixel in the band, histogram windows clipped at the picture's edges), bit-exact, with a different algorithm.
//
// One 256-thread block per 64 x 64 tile of any scale of any picture (a table of jobs):
//  1. a pre-check of the tile's own pixels (16-byte loads) lets tiles with nothing to compute -- most tiles of most
//     pictures -- leave after reading them;
//  2. the tile and its window margins are staged in shared memory as band codes (value - band_base of a masked pixel
//     in the band, kNone otherwise) with 16-byte loads from an 8-pixel-aligned start; the codes that can matter --
//     occurring within kDiffs of a code whose c-value is needed -- are ranked in order, and each needed code gets its
//     8 neighbours' rank offsets and the mask of ranks it reads;
//  3. per pass over 32 ranks: column counts (u8) of the ranks slide down the rows; per row, the rank pairs some pixel
//     reads are prefix-summed over the columns (two ranks per 32-bit lane) and turned into window counts of the 64
//     tile columns; every 4 rows all 8 warps compute the 256 c-values from those counts.
// Positive c-values are summed exactly (they are multiples of 2^-24) and counted, and each block appends them to its
// scale's list (for the top-k selection) through a bounded shared-memory buffer; nothing per pixel is written unless
// the caller asks for the c-value planes.
#include "es_kernels.h"

namespace es {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kCvChunk = kCvThreads / kCvTX;  // rows whose c-values are computed together
constexpr int kListCap = 1024;                // positive c-values buffered per block before a flush

__host__ __device__ constexpr int cv_rw(int pad) { return kCvTX + 2 * pad; }
// the staged region starts at the multiple of 8 at or left of x0 - pad; its row stride is a whole number of vectors
__host__ __device__ constexpr int cv_stride(int pad) { return (cv_rw(pad) + 7 + 7) & ~7; }
__host__ __device__ constexpr int cv_cs(int pad) { return (cv_rw(pad) + 127) & ~127; }  // column stride (scan width)
__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

struct CvLayout {
    size_t codes, rank, nbr, relneed, colcnt, prefix, wcount, list, total;
};
__host__ __device__ inline CvLayout cv_layout(int pad)
{
    CvLayout l;
    l.codes = 0;
    l.rank = align16((size_t)cv_stride(pad) * (kCvTY + 2 * pad) * 2);
    l.nbr = align16(l.rank + (size_t)kMaxBand * 2);
    l.relneed = align16(l.nbr + (size_t)kMaxBand * 4);
    l.colcnt = align16(l.relneed + (size_t)kMaxBand * 2);
    l.prefix = align16(l.colcnt + (size_t)kCvBins * cv_cs(pad));
    l.wcount = align16(l.prefix + (size_t)(kCvThreads / 32) * cv_cs(pad) * 4);
    l.list = align16(l.wcount + (size_t)kCvChunk * (kCvBins / 2) * kCvTX * 4);
    l.total = align16(l.list + (size_t)kListCap * 4);
    return l;
}

// the distances d + 1 at which a code's c-value looks (src/kernels.cu:195-197): bit d
__host__ __device__ inline unsigned cvalue_dists(int code, const Band &bd)
{
    const int value = code + bd.band_base + kDiffs;
    unsigned m = 0;
    for (int d = 0; d < kDiffs; d++) m |= (unsigned)(value <= bd.tvi[d] && value + d + 1 > bd.vlt) << d;
    return m;
}
__device__ __forceinline__ bool needs_cvalue(int code, const Band &bd) { return cvalue_dists(code, bd) != 0; }

__device__ __forceinline__ uint16_t code_of(unsigned word, const Band &bd)
{
    const unsigned u = (word & 0x7FFFu) - (unsigned)bd.band_base;
    return ((word & kMaskBit) && u < (unsigned)bd.band_size) ? (uint16_t)u : kNone;
}

__global__ void __launch_bounds__(kCvThreads) cvalues_kernel(const __grid_constant__ CvBatch b)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t occ[32], srv[32], rel[32], needbits[32];
    __shared__ uint16_t relpre[33];
    __shared__ uint32_t rowneed[kCvTY];
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
    const bool vec = (w & 7) == 0 && (((uintptr_t)J.word) & 15) == 0;  // rows of 16-byte vectors
    // the codes whose c-value is needed (some d has value <= tvi[d] and value + d + 1 > vlt): warp w, words w + 8 k
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int code = (warp + 8 * k) * 32 + lane;
        const unsigned m = __ballot_sync(kFull, code < bd.band_size && needs_cvalue(code, bd));
        if (lane == 0) needbits[warp + 8 * k] = m;
    }
    __syncthreads();
    auto needed = [&](unsigned code) { return (needbits[code >> 5] >> (code & 31)) & 1u; };

    // 1. does any pixel of the tile need a c-value?
    bool any = false;
    if (vec && cols == kCvTX) {
        for (int i = tid; i < kCvTY * (kCvTX / 8); i += kCvThreads) {
            const int r = i >> 3, v = i & 7;
            if (r >= rows) continue;
            const uint4 q = __ldg((const uint4 *)(J.word + (size_t)(y0 + r) * w + x0) + v);
            auto test = [&](unsigned word) {
                const uint16_t c0 = code_of(word & 0xFFFFu, bd), c1 = code_of(word >> 16, bd);
                any |= (c0 != kNone && needed(c0)) || (c1 != kNone && needed(c1));
            };
            test(q.x);
            test(q.y);
            test(q.z);
            test(q.w);
        }
    } else {
        for (int i = tid; i < kCvTX * kCvTY; i += kCvThreads) {
            const int r = i >> 6, c = i & (kCvTX - 1);
            if (r < rows && c < cols) {
                const uint16_t code = code_of(J.word[(size_t)(y0 + r) * w + x0 + c], bd);
                any |= code != kNone && needed(code);
            }
        }
    }
    if (!__syncthreads_or(any)) return;

    const int RW = cv_rw(P), RH = rows + 2 * P, CS = cv_cs(P), S = cv_stride(P);
    const int xs = ((x0 - P) >> 3) << 3, ox = (x0 - P) - xs;  // region start (aligned) and the offset of x0 - P in it
    const CvLayout L = cv_layout(P);
    uint16_t *codes = (uint16_t *)(smem + L.codes);           // [RH][S]: element e of row r is pixel (xs + e, y0 - P + r)
    uint16_t *rank = (uint16_t *)(smem + L.rank);
    uint32_t *nbr = (uint32_t *)(smem + L.nbr);
    uint16_t *relneed = (uint16_t *)(smem + L.relneed);
    uint8_t *colcnt = smem + L.colcnt;
    uint32_t *prefix = (uint32_t *)(smem + L.prefix);        // per-warp prefix rows
    uint32_t *wcount = (uint32_t *)(smem + L.wcount);        // [chunk row][rank pair][column] packed window counts
    float *blist = (float *)(smem + L.list);
    if (tid < 32) occ[tid] = srv[tid] = 0;
    if (tid == 0) list_n = 0;
    __syncthreads();

    // 2. stage the region, 8 elements per thread and step
    {
        const int nv = S >> 3, total = RH * nv;
        for (int i = tid; i < total; i += kCvThreads) {
            const int r = i / nv, v = i - r * nv, y = y0 - P + r, xv = xs + 8 * v;
            uint16_t cs[8];
            if (vec && y >= 0 && y < h && xv >= 0 && xv + 8 <= w) {
                const uint4 q = __ldg((const uint4 *)(J.word + (size_t)y * w + xv));
                cs[0] = code_of(q.x & 0xFFFFu, bd);
                cs[1] = code_of(q.x >> 16, bd);
                cs[2] = code_of(q.y & 0xFFFFu, bd);
                cs[3] = code_of(q.y >> 16, bd);
                cs[4] = code_of(q.z & 0xFFFFu, bd);
                cs[5] = code_of(q.z >> 16, bd);
                cs[6] = code_of(q.w & 0xFFFFu, bd);
                cs[7] = code_of(q.w >> 16, bd);
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int x = xv + k;
                    cs[k] = (y >= 0 && y < h && x >= 0 && x < w) ? code_of(J.word[(size_t)y * w + x], bd) : kNone;
                }
            }
            uint4 st;
            st.x = cs[0] | ((unsigned)cs[1] << 16);
            st.y = cs[2] | ((unsigned)cs[3] << 16);
            st.z = cs[4] | ((unsigned)cs[5] << 16);
            st.w = cs[6] | ((unsigned)cs[7] << 16);
            *(uint4 *)(codes + r * S + 8 * v) = st;
            const bool row_in_tile = r >= P && r < P + rows;
            uint16_t prev = kNone, prev_srv = kNone;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint16_t code = cs[k];
                if (code == kNone) continue;
                if (code != prev) atomicOr(&occ[code >> 5], 1u << (code & 31));
                prev = code;
                const int x = xv + k;
                if (row_in_tile && x >= x0 && x < x0 + cols && code != prev_srv && needed(code)) {
                    atomicOr(&srv[code >> 5], 1u << (code & 31));
                    prev_srv = code;
                }
            }
        }
    }
    __syncthreads();

    // the relevant codes: occurring within kDiffs of a code that needs c-values, ranked in order
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
            const unsigned v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
        }
        relpre[lane] = (uint16_t)(incl - cnt);
        if (lane == 31) relpre[32] = (uint16_t)incl;
    }
    __syncthreads();
    const int R = relpre[32];
    for (int c = tid; c < bd.band_size; c += kCvThreads) {
        const uint32_t word = rel[c >> 5], bit = 1u << (c & 31);
        rank[c] = (word & bit) ? (uint16_t)(relpre[c >> 5] + __popc(word & (bit - 1u))) : kNone;
    }
    __syncthreads();
    // for each served code: the rank offsets (+4) of its neighbours u-4 .. u-1, u+1 .. u+4 (15 = none), and the mask of
    // the ranks rank-4 .. rank+4 it reads (bit 4 is its own)
    for (int c = tid; c < bd.band_size; c += kCvThreads) {
        if (!(srv[c >> 5] & (1u << (c & 31)))) continue;
        const int rc = rank[c];
        const unsigned dists = cvalue_dists(c, bd);
        uint32_t packed = 0;
        unsigned mask = 1u << 4;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int q = c + (i < 4 ? i - 4 : i - 3);
            const int d = i < 4 ? 3 - i : i - 4;  // distance d + 1
            unsigned nib = 15u;
            if (q >= 0 && q < bd.band_size && rank[q] != kNone) {
                nib = (unsigned)((int)rank[q] - rc + 4);
                if ((dists >> d) & 1u) mask |= 1u << nib;
            }
            packed |= nib << (4 * i);
        }
        nbr[c] = packed;
        relneed[c] = (uint16_t)mask;
    }

    unsigned long long my_sum = 0;
    unsigned my_cnt = 0;
    CvSlot &SL = b.slots[J.slot];
    // moves the block's buffered c-values to the scale's list (called by all threads, list_n > 0)
    auto flush = [&]() {
        if (tid == 0) list_base = atomicAdd(&SL.list_n, (unsigned long long)list_n);
        __syncthreads();
        const unsigned ln = list_n;
        for (unsigned i = tid; i < ln; i += kCvThreads) SL.list[list_base + i] = blist[i];
        __syncthreads();
        if (tid == 0) list_n = 0;
        __syncthreads();
    };

    for (int b0 = 0;;) {
        const int B = min(kCvBins, R - b0);
        const int lo = b0 ? b0 + kDiffs : 0, hi = b0 + kCvBins >= R ? R : b0 + kCvBins - kDiffs;
        if (tid < kCvTY) rowneed[tid] = 0;
        for (int i = tid * 16; i < kCvBins * CS; i += kCvThreads * 16) *(uint4 *)(colcnt + i) = make_uint4(0, 0, 0, 0);
        __syncthreads();
        // the ranks each row's pixels read in this pass: a warp covers 32 pixels of one row
        for (int i = tid; i < kCvTY * kCvTX; i += kCvThreads) {
            const int r = i >> 6, c = i & (kCvTX - 1);
            uint32_t need = 0;
            if (r < rows && c < cols) {
                const uint16_t code = codes[(r + P) * S + c + P + ox];
                if (code != kNone && (srv[code >> 5] & (1u << (code & 31)))) {
                    const int rk = rank[code];
                    if (rk >= lo && rk < hi) {
                        const int sh = rk - b0 - 4;
                        const uint32_t m = relneed[code];
                        need = sh >= 0 ? m << sh : m >> -sh;
                    }
                }
            }
            need = __reduce_or_sync(kFull, need);
            if (lane == 0 && need) atomicOr(&rowneed[r], need);
        }
        // column counts over the window rows of tile row 0 (region rows 0 .. 2P)
        if (tid < RW) {
            uint8_t *col = colcnt + tid;
            const int last = min(2 * P, RH - 1);
            for (int r = 0; r <= last; r++) {
                const uint16_t code = codes[r * S + tid + ox];
                if (code != kNone) {
                    const int k = (int)rank[code] - b0;
                    if ((unsigned)k < (unsigned)B) col[k * CS]++;
                }
            }
        }
        __syncthreads();
        // Rows go in chunks of kCvChunk. Per row: (a) slide the column counts down to it; (b) each warp turns every 8th
        // pair of the ranks the row reads into a packed prefix sum over the columns (two ranks per 32-bit lane) and
        // then into the window counts of the tile's 64 columns. Per chunk: (c) every thread computes one pixel's
        // c-value from those counts.
        auto slide = [&](int r) {
            if (tid >= RW) return;
            uint8_t *col = colcnt + tid;
            const uint16_t cl = codes[(r - 1) * S + tid + ox];
            if (cl != kNone) {
                const int k = (int)rank[cl] - b0;
                if ((unsigned)k < (unsigned)B) col[k * CS]--;
            }
            if (r + 2 * P < RH) {
                const uint16_t ce = codes[(r + 2 * P) * S + tid + ox];
                if (ce != kNone) {
                    const int k = (int)rank[ce] - b0;
                    if ((unsigned)k < (unsigned)B) col[k * CS]++;
                }
            }
        };
        auto window_counts = [&](int r, int i) {  // row r into chunk slot i
            const uint32_t need = rowneed[r];
            uint32_t *wpre = prefix + warp * CS;
            const uint32_t pairs = (need | (need >> 1)) & 0x55555555u;  // bit 2p: pair p is read
            uint32_t pp = pairs;  // warp w takes pairs w, w + 8 (in the order of the read pairs)
            for (int t = 0; t < warp && pp; t++) pp &= pp - 1u;
            while (pp) {
                const int p = (__ffs(pp) - 1) >> 1;
                for (int t = 0; t < kCvThreads / 32 && pp; t++) pp &= pp - 1u;
                const uint8_t *ca = colcnt + (2 * p) * CS, *cb = ca + CS;
                unsigned carry = 0;
                for (int base = 0; base < CS; base += 128) {
                    const uint32_t fa = *(const uint32_t *)(ca + base + 4 * lane), fb = *(const uint32_t *)(cb + base + 4 * lane);
                    const uint32_t a0 = fa & 0x00FF00FFu, c0 = fb & 0x00FF00FFu, a1 = (fa >> 8) & 0x00FF00FFu, c1 = (fb >> 8) & 0x00FF00FFu;
                    // column 4 lane + i of rank 2p in the low 16 bits, of rank 2p + 1 in the high 16 bits
                    const unsigned s1 = __byte_perm(a0, c0, 0x5410), s2 = s1 + __byte_perm(a1, c1, 0x5410),
                                   s3 = s2 + __byte_perm(a0, c0, 0x7632), s4 = s3 + __byte_perm(a1, c1, 0x7632);
                    unsigned incl = s4;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const unsigned v = __shfl_up_sync(kFull, incl, o);
                        if (lane >= o) incl += v;
                    }
                    const unsigned ex = incl - s4 + carry;
                    *(uint4 *)(wpre + base + 4 * lane) = make_uint4(ex + s1, ex + s2, ex + s3, ex + s4);
                    carry += __shfl_sync(kFull, incl, 31);
                }
                __syncwarp();
                uint32_t *wrow = wcount + (i * (kCvBins / 2) + p) * kCvTX;
#pragma unroll
                for (int h2 = 0; h2 < 2; h2++) {
                    const int x = lane + 32 * h2;
                    wrow[x] = wpre[x + 2 * P] - (x > 0 ? wpre[x - 1] : 0u);
                }
                __syncwarp();
            }
        };
        const int ci = tid >> 6, cc = tid & (kCvTX - 1);  // this thread's pixel in a chunk
        for (int r0 = 0; r0 < rows; r0 += kCvChunk) {
            const int n_rows = min(kCvChunk, rows - r0);
            bool chunk_any = false;
            for (int i = 0; i < n_rows; i++) {
                const int r = r0 + i;
                if (r > 0) slide(r);
                if (!rowneed[r]) continue;
                chunk_any = true;
                __syncthreads();
                window_counts(r, i);
                __syncthreads();
            }
            if (!chunk_any) continue;
            // (c) the chunk's c-values, one pixel per thread
            float c = 0.0f;
            bool served = false;
            const int r = r0 + ci;
            if (ci < n_rows && cc < cols) {
                const uint16_t code = codes[(r + P) * S + cc + P + ox];
                if (code != kNone && (srv[code >> 5] & (1u << (code & 31)))) {
                    const int rk = rank[code];
                    if (rk >= lo && rk < hi) {
                        served = true;
                        const uint32_t nb = nbr[code];
                        const int base = rk - b0 - 4;
                        const uint32_t *wc = wcount + ci * (kCvBins / 2) * kCvTX + cc;
                        auto count = [&](int k) -> unsigned { return (wc[(k >> 1) * kCvTX] >> ((k & 1) * 16)) & 0xFFFFu; };
                        const int value = code + bd.band_base + kDiffs;
                        const unsigned p0 = count(rk - b0);
#pragma unroll
                        for (int d = 0; d < kDiffs; d++) {
                            if (value <= bd.tvi[d] && value + d + 1 > bd.vlt) {
                                const unsigned o1 = (nb >> (4 * (4 + d))) & 15u, o2 = (nb >> (4 * (3 - d))) & 15u;
                                const unsigned p1 = o1 != 15u ? count(base + (int)o1) : 0u;
                                const unsigned p2 = o2 != 15u ? count(base + (int)o2) : 0u;
                                const unsigned pm = p1 > p2 ? p1 : p2;
                                const float val = __fmul_rn(__uint2float_rn((unsigned)bd.weight[d] * p0 * pm), __ldg(b.lut + p0 + pm));
                                if (val > c) c = val;
                            }
                        }
                    }
                }
            }
            const bool pos = c > 0.0f;
            const unsigned m = __ballot_sync(kFull, pos);
            if (m) {
                unsigned at = 0;
                if (lane == __ffs(m) - 1) at = atomicAdd(&list_n, (unsigned)__popc(m));
                at = __shfl_sync(kFull, at, __ffs(m) - 1);
                if (pos) blist[at + __popc(m & ((1u << lane) - 1u))] = c;
            }
            if (served && J.plane) J.plane[(size_t)(y0 + r) * w + x0 + cc] = c;
            if (pos) {
                my_sum += __float2ull_rn(__fmul_rn(c, 16777216.0f));
                my_cnt++;
            }
            __syncthreads();
            if (list_n > kListCap - kCvThreads) flush();
        }
        if (hi == R) break;
        b0 = hi - kDiffs;
        __syncthreads();
    }

    // block totals, and the rest of this block's positive c-values appended to the scale's list
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        my_sum += __shfl_down_sync(kFull, my_sum, o);
        my_cnt += __shfl_down_sync(kFull, my_cnt, o);
    }
    if (lane == 0) {
        red_sum[warp] = my_sum;
        red_cnt[warp] = my_cnt;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long s = 0;
        unsigned c = 0;
        for (int k = 0; k < kCvThreads / 32; k++) {
            s += red_sum[k];
            c += red_cnt[k];
        }
        if (c) {
            atomicAdd(&SL.sum_fx, s);
            atomicAdd(&SL.count, (unsigned long long)c);
        }
    }
    if (list_n) flush();
}

}  // namespace

size_t cvalues_smem_bytes(int max_pad) { return cv_layout(max_pad).total; }

cudaError_t launch_cvalues(const CvBatch &b, cudaStream_t s)
{
    if (b.total_tiles <= 0) return cudaSuccess;
    const size_t smem = cvalues_smem_bytes(b.max_pad);
    cudaError_t e = cudaFuncSetAttribute(cvalues_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    LaunchTimer t("cambi_cvalues", s);
    cvalues_kernel<<<b.total_tiles, kCvThreads, smem, s>>>(b);
    return after_launch();
}

const void *kernel_entry_cvalues() { return (const void *)cvalues_kernel; }

}  // namespace es
