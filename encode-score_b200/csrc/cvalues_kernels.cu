// CAMBI c-values for sm_100a: src/kernels.cu:113-278 (cambi.c's c_value_pixel over the (2 pad + 1)^2 window of every
// masked pixel in the band, histogram windows clipped at the picture's edges), bit-exact, with a different algorithm.
//
// One 256-thread block per 64 x 64 tile of any scale of any picture (a table of jobs):
//  1. a pre-check of the tile's own pixels (16-byte loads) lets tiles with nothing to compute -- most tiles of most
//     pictures -- leave after reading them;
//  2. the band codes (value - band_base of a masked pixel in the band, kNone otherwise) of the tile and its window
//     margins are read with 16-byte loads from an 8-pixel-aligned start; the codes that can matter -- occurring within
//     kDiffs of a code whose c-value is needed -- are ranked in order, each rank gets its code, the rank offsets of
//     its 8 neighbour codes and the mask of ranks its c-value reads (tiles where no code has a neighbour code leave:
//     their c-values are all 0); the codes, kept as 16-bit values in the shared memory that later holds the rank
//     plane and the counts (when the region fits there; else read again), become a plane of 8-bit ranks in place;
//  3. per pass over 32 ranks, the ranks' column counts (8 bits per column and rank: pixels of the 2 pad + 1 window rows)
//     sit in shared memory as a 32 x region-width byte matrix and slide down the rows (the leaving and entering row's
//     rank per column); on rows whose pixels read the pass's ranks, the window counts of the 64 tile columns are one
//     exact integer matrix product on the tensor cores (mma.sync u8, counts x a band of ones 2 pad + 1 wide), each warp
//     making 16 ranks x 16 columns. Every 4 rows all 8 warps compute the 256 c-values from those counts.
// Positive c-values are summed exactly (they are multiples of 2^-24) and counted, and each block appends them to its
// scale's list (for the top-k selection) through a bounded shared-memory buffer; nothing per pixel is written unless
// the caller asks for the c-value planes.
#include <type_traits>

#include "cambi_codes.h"
#include "es_kernels.h"

namespace es {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kCvChunk = 4;                   // rows whose c-values are computed together (threads = 4 x tile width)
// One column-count buffer, slid by one row between the rows' window counts (a slide and two barriers per row): two or
// four buffers, each slid by two or four rows so that rows share barriers, measured slower (more slide work).
constexpr int kListCap = 2048;                // positive c-values buffered per block before a flush (1024: 1 % slower)
constexpr unsigned kNoRank = 0xFFu;           // rank plane: no relevant code
constexpr int kMaxPlaneRank = 254;            // ranks a plane of absolute ranks can hold

// Tiles are TX columns wide (64 or 128); a block has 4 TX threads.
__host__ __device__ constexpr int cv_rw(int tx, int pad) { return tx + 2 * pad; }
// the staged region starts at the multiple of 8 at or left of x0 - pad; its row stride is a whole number of vectors
__host__ __device__ constexpr int cv_stride(int tx, int pad) { return (cv_rw(tx, pad) + 7 + 7) & ~7; }
__host__ __device__ constexpr int cv_cs(int tx, int pad) { return (cv_rw(tx, pad) + 127) & ~127; }  // rank plane row
// k-steps of 32 region columns, and the row of the column counts (bytes; 16 more than the k-steps, so the 8 rows an
// ldmatrix phase reads fall on different banks)
__host__ __device__ constexpr int cv_nk(int tx, int pad) { return (cv_rw(tx, pad) + 31) >> 5; }
__host__ __device__ constexpr int cv_cstr(int tx, int pad) { return 32 * cv_nk(tx, pad) + 16; }
// k-steps one warp's window counts reach (output columns xb .. xb + 23 with xb % 32 <= 8, and 2 pad more), at most
constexpr int kCvMaxK = (8 + 23 + 2 * kMaxPad) / 32 + 1;
__host__ __device__ constexpr int cv_ws(int tx) { return tx + 2; }  // window-count row (u16): an odd number of words
__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// Shared memory: the rank plane, the per-code and per-rank tables and the pass buffers. (The band codes are read from
// global memory twice, once for the code tables and once for the rank plane, instead of being staged: the smaller
// footprint lets 4 blocks share an SM.)
struct CvLayout {
    size_t rplane, rank, nbr, relneed, wcount, cols, list, total;
};
__host__ __device__ inline CvLayout cv_layout(int tx, int pad)
{
    const size_t rh = (size_t)kCvTY + 2 * pad;
    CvLayout l;
    // the rank plane, window counts and column counts first: until the plane is built they hold the region's band
    // codes (16 bits each) when those fit
    l.rplane = 0;
    l.wcount = align16(l.rplane + rh * cv_cs(tx, pad));
    l.cols = align16(l.wcount + (size_t)kCvChunk * kCvBins * cv_ws(tx) * 2);
    l.rank = align16(l.cols + (size_t)kCvBins * cv_cstr(tx, pad));
    l.nbr = align16(l.rank + (size_t)kMaxBand * 2);
    l.relneed = align16(l.nbr + (size_t)kMaxBand * 4);
    l.list = align16(l.relneed + (size_t)kMaxBand * 2);
    l.total = align16(l.list + (size_t)kListCap * 4);
    return l;
}


__device__ __forceinline__ void ldmatrix_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

// d += a (16 x 32 u8, row-major) x b (32 x 8 u8, column-major), exact in 32-bit integers.
__device__ __forceinline__ void mma_u8(int (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// The band codes of the two words of x (value | mask << 15 per 16-bit half): value - band_base where masked and in the
// band, kNone (0xFFFF) otherwise, per half.
__device__ __forceinline__ uint32_t codes2(uint32_t x, uint32_t base2, uint32_t size2)
{
    const uint32_t u = __vsub2(x & 0x7FFF7FFFu, base2);  // wraps below the band
    const uint32_t in = __vcmpltu2(u, size2) & __vcmpne2(x & 0x80008000u, 0u);
    return u | ~in;
}

template <int TX>
__global__ void __launch_bounds__(4 * TX, 256 / TX) cvalues_kernel(const __grid_constant__ CvBatch b)
{
    constexpr int kCvThreads = 4 * TX, kWarps = kCvThreads / 32, kCvWS = cv_ws(TX);
    constexpr int kQuads = TX / 4;  // 4-pixel groups of a tile row
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t occ[32], srv[32], rel[32], needbits[32];
    __shared__ uint16_t relpre[33];
    __shared__ uint32_t rowneed[kCvTY];
    __shared__ unsigned list_n;
    __shared__ unsigned long long list_base;
    __shared__ unsigned long long red_sum[kWarps];
    __shared__ unsigned red_cnt[kWarps];
    __shared__ unsigned hist1[kCvDigits];  // the tile's positive c-values by their first radix digit

    __shared__ unsigned next_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const Band &bd = b.band;
    // the codes whose c-value is needed (some d has value <= tvi[d] and value + d + 1 > vlt): warp w, words w + kWarps k
    for (int word = warp; word < 32; word += kWarps) {
        const int code = word * 32 + lane;
        const unsigned m = __ballot_sync(kFull, code < bd.band_size && needs_cvalue(code, bd));
        if (lane == 0) needbits[word] = m;
    }
    __syncthreads();
    auto needed = [&](unsigned code) { return (needbits[code >> 5] >> (code & 31)) & 1u; };

  // one tile, gt its global number; all threads return together
  auto tile_body = [&](const int gt) {
    const int j = find_job(b.njobs, gt, [&](int k) { return b.job[k].first_tile; });
    const CvJob &J = b.job[j];
    if (b.run && !b.run[J.run_index]) return;
    const int tile = gt - J.first_tile;
    const int th = J.tile_rows ? J.tile_rows : kCvTY;  // shorter tiles use the same buffers, like a picture's last row
    const int x0 = (tile % J.tiles_x) * TX, y0 = (tile / J.tiles_x) * th;
    const int w = J.w, h = J.h, P = J.pad;
    const int rows = min(th, h - y0), cols = min(TX, w - x0);
    const bool vec = (w & 7) == 0 && (((uintptr_t)J.word) & 15) == 0;  // rows of 16-byte vectors

    // 1. does any pixel of the tile need a c-value?
    bool any = false;
    const uint32_t base2 = (uint32_t)bd.band_base * 0x10001u, size2 = (uint32_t)bd.band_size * 0x10001u;
    if (vec && cols == TX) {
        const bool range = b.need_span >= 0;
        const uint32_t lo2 = (uint32_t)b.need_lo * 0x10001u, span2 = (uint32_t)(range ? b.need_span : 0) * 0x10001u;
        for (int i = tid; i < kCvTY * (TX / 8); i += kCvThreads) {
            const int r = i / (TX / 8), v = i % (TX / 8);
            if (r >= rows) continue;
            const uint4 q = __ldg((const uint4 *)(J.word + (size_t)(y0 + r) * w + x0) + v);
            auto test = [&](uint32_t word) {
                if (range) {  // masked values in the one range of needed values, both halves at once
                    any |= (__vcmpleu2(__vsub2(word & 0x7FFF7FFFu, lo2), span2) & __vcmpne2(word & 0x80008000u, 0u)) != 0;
                } else {
                    const uint32_t c2 = codes2(word, base2, size2);
                    const uint16_t c0 = (uint16_t)c2, c1 = (uint16_t)(c2 >> 16);
                    any |= (c0 != kNone && needed(c0)) || (c1 != kNone && needed(c1));
                }
            };
            test(q.x);
            test(q.y);
            test(q.z);
            test(q.w);
        }
    } else {
        for (int i = tid; i < TX * kCvTY; i += kCvThreads) {
            const int r = i / TX, c = i % TX;
            if (r < rows && c < cols) {
                const uint16_t code = code_of(J.word[(size_t)(y0 + r) * w + x0 + c], bd);
                any |= code != kNone && needed(code);
            }
        }
    }
    if (!__syncthreads_or(any)) {
        if (b.tile_mass && tid == 0) b.tile_mass[gt] = 0;
        return;
    }

    const int RW = cv_rw(TX, P), RH = rows + 2 * P, CS = cv_cs(TX, P), S = cv_stride(TX, P);
    const int xs = ((x0 - P) >> 3) << 3, ox = (x0 - P) - xs;  // region start (aligned) and the offset of x0 - P in it
    const CvLayout L = cv_layout(TX, P);
    uint8_t *rplane = smem + L.rplane;                   // [RH][CS]: rank (- offset) of pixel (x0 - P + j, y0 - P + r)
    uint16_t *rank = (uint16_t *)(smem + L.rank);        // code -> rank
    uint32_t *nbr = (uint32_t *)(smem + L.nbr);          // rank -> neighbour rank offsets
    uint16_t *relneed = (uint16_t *)(smem + L.relneed);  // rank -> ranks read (bit 4: itself); 0: not served
    float *blist = (float *)(smem + L.list);
    // during the staging the rank table's bytes are two flag arrays: [0, kMaxBand) codes held by the region,
    // [kMaxBand, 2 kMaxBand) codes held by the tile's own pixels (plain byte stores: racing writers store the same 1)
    uint8_t *seen = smem + L.rank;
    for (int i = tid; i < 2 * kMaxBand / 16; i += kCvThreads) ((uint4 *)seen)[i] = make_uint4(0, 0, 0, 0);
    if (tid < kCvDigits) hist1[tid] = 0;
    if (tid == 0) list_n = 0;
    __syncthreads();

    // the band codes of region row r, pixels xs + 8 v .. + 7, packed in pairs (16-byte loads where the row allows)
    auto load8 = [&](int r, int v) -> uint4 {
        const int y = y0 - P + r, xv = xs + 8 * v;
        if (vec && y >= 0 && y < h && xv >= 0 && xv + 8 <= w) {
            const uint4 q = __ldg((const uint4 *)(J.word + (size_t)y * w + xv));
            return make_uint4(codes2(q.x, base2, size2), codes2(q.y, base2, size2), codes2(q.z, base2, size2),
                              codes2(q.w, base2, size2));
        }
        uint32_t c2[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            uint32_t pairv = 0;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int x = xv + 2 * k + e;
                const uint32_t code = (y >= 0 && y < h && x >= 0 && x < w) ? code_of(J.word[(size_t)y * w + x], bd) : kNone;
                pairv |= code << (16 * e);
            }
            c2[k] = pairv;
        }
        return make_uint4(c2[0], c2[1], c2[2], c2[3]);
    };
    // 2. the codes the region holds (occ) and the codes own pixels need (srv), 8 pixels per thread and step (all
    // threads busy: a warp per row would leave lanes idle on narrow regions), as flags turned into bit words after;
    // the codes themselves are kept in shared memory (row r, vector v at 16-bit element r S + 8 v) when they fit below
    // the rank tables, so the rank plane is built without a second read of the scale
    uint16_t *codes16 = (uint16_t *)(smem + L.rplane);
    const bool staged = (size_t)RH * S * 2 <= L.rank;
    const int nv = S >> 3;  // vectors of a region row
    const unsigned nv_magic = 0xFFFFFFFFu / (unsigned)nv + 1u;  // i / nv = umulhi(i, magic) for i < 2^16, nv < 64
    for (int i = tid; i < RH * nv; i += kCvThreads) {
        const int r = (int)__umulhi((unsigned)i, nv_magic), v = i - r * nv;
        const bool row_in_tile = r >= P && r < P + rows;
        {
            const int xv = xs + 8 * v;
            const uint4 q = load8(r, v);
            if (staged) ((uint4 *)codes16)[i] = q;
            const uint32_t wv[4] = {q.x, q.y, q.z, q.w};
            const bool whole = row_in_tile && xv >= x0 && xv + 8 <= x0 + cols;  // all 8 pixels are the tile's
            const bool part = row_in_tile && !whole && xv + 8 > x0 && xv < x0 + cols;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint16_t code = (uint16_t)(wv[k >> 1] >> (16 * (k & 1)));
                if (code == kNone) continue;
                seen[code] = 1;
                const int x = xv + k;
                if (whole || (part && x >= x0 && x < x0 + cols)) seen[kMaxBand + code] = 1;
            }
        }
    }
    __syncthreads();
    for (int word = warp; word < 32; word += kWarps) {
        const unsigned o = __ballot_sync(kFull, seen[32 * word + lane] != 0);
        const unsigned t = __ballot_sync(kFull, seen[kMaxBand + 32 * word + lane] != 0);
        if (lane == 0) {
            occ[word] = o;
            srv[word] = t & needbits[word];
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
    // per rank of a served code: the rank offsets (+4) of the neighbours u-4 .. u-1, u+1 .. u+4 its c-value
    // reads (15 = none: not in the region, or at a distance d + 1 whose diff CAMBI's thresholds switch off for this
    // code, which gives the same c-value as a neighbour with no pixels) and the mask of the ranks rank-4 .. rank+4 read
    // (bit 4 is its own)
    bool any_served = false;
    for (int c = tid; c < bd.band_size; c += kCvThreads) {
        const int rc = rank[c];
        if (rc == kNone) continue;
        if (!(srv[c >> 5] & (1u << (c & 31)))) {
            relneed[rc] = 0;
            continue;
        }
        const unsigned dists = cvalue_dists(c, bd);
        uint32_t packed = 0;
        unsigned mask = 1u << 4;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int q = c + (i < 4 ? i - 4 : i - 3);
            const int d = i < 4 ? 3 - i : i - 4;  // distance d + 1
            unsigned nib = 15u;
            if (q >= 0 && q < bd.band_size && rank[q] != kNone && ((dists >> d) & 1u)) {
                nib = (unsigned)((int)rank[q] - rc + 4);
                mask |= 1u << nib;
            }
            packed |= nib << (4 * i);
        }
        nbr[rc] = packed;
        // with no neighbour code in the region its c-value is 0 (pm = 0 for every distance): not served, so rows of
        // such pixels (whole plateaus, codes requantised in steps over 4) count nothing
        relneed[rc] = mask == (1u << 4) ? (uint16_t)0 : (uint16_t)mask;
        any_served |= mask != (1u << 4);
    }
    // every c-value of the tile is 0: nothing to count
    if (!__syncthreads_or(any_served)) {
        if (b.tile_mass && tid == 0) b.tile_mass[gt] = 0;
        return;
    }
    // the rank plane: absolute ranks once for the tile when they fit in a byte, else per pass relative to the pass
    const bool per_pass = R > kMaxPlaneRank + 1;
    auto build_plane = [&](int b0) {  // b0 < 0: absolute ranks; else ranks of the pass from b0 (others: no rank)
        for (int i = tid; i < RH * CS / 16; i += kCvThreads) ((uint4 *)rplane)[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
        __syncthreads();
        for (int i = tid; i < RH * nv; i += kCvThreads) {
            const int r = i / nv, v = i - r * nv;
            const uint4 q = load8(r, v);
            const uint32_t wv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int j = 8 * v + k - ox;  // region column
                const uint16_t code = (uint16_t)(wv[k >> 1] >> (16 * (k & 1)));
                if (j < 0 || j >= RW || code == kNone) continue;
                const int rk0 = rank[code];
                if (rk0 == kNone) continue;
                const int rk = b0 < 0 ? rk0 : rk0 - b0;
                if (b0 >= 0 && (rk < 0 || rk >= kCvBins)) continue;
                rplane[r * CS + j] = (uint8_t)rk;
            }
        }
    };
    if (!per_pass && staged) {
        // the codes, vector by vector, into 8-bit ranks in place: the rank bytes of vector i (row r, bytes r CS + 8 v
        // + k - ox) lie within the code bytes of vector i or of earlier ones (16 i + 15 at most, as CS <= 2 S), so a
        // step's writes only cover codes read before its barrier; every region column gets a rank or kNoRank
        auto rank_of = [&](uint32_t wv, int e) -> uint32_t {
            const uint16_t code = (uint16_t)(wv >> (16 * e));
            const unsigned rk = code == kNone ? kNoRank : rank[code];
            return rk == kNone ? kNoRank : rk;
        };
        const int total = RH * nv;
        for (int c0 = 0; c0 < total; c0 += kCvThreads) {
            const int i = c0 + tid;
            uint4 q = make_uint4(0, 0, 0, 0);
            if (i < total) q = ((const uint4 *)codes16)[i];
            __syncthreads();
            if (i < total) {
                const int r = (int)__umulhi((unsigned)i, nv_magic), v = i - r * nv;
                const uint32_t wv[4] = {q.x, q.y, q.z, q.w};
                if (ox == 0 && 8 * v + 8 <= RW) {
                    const uint32_t lo = rank_of(wv[0], 0) | (rank_of(wv[0], 1) << 8) | (rank_of(wv[1], 0) << 16) | (rank_of(wv[1], 1) << 24);
                    const uint32_t hi = rank_of(wv[2], 0) | (rank_of(wv[2], 1) << 8) | (rank_of(wv[3], 0) << 16) | (rank_of(wv[3], 1) << 24);
                    *(uint2 *)(rplane + r * CS + 8 * v) = make_uint2(lo, hi);
                } else {
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int j = 8 * v + k - ox;
                        if (j < 0 || j >= RW) continue;
                        rplane[r * CS + j] = (uint8_t)rank_of(wv[k >> 1], k & 1);
                    }
                }
            }
        }
    } else if (!per_pass) {
        build_plane(-1);
    }
    __syncthreads();

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

    // Window counts on the tensor cores: per row, W[rank][x] = sum over region columns j of C[rank][j] B[j][x], where C
    // holds the ranks' column counts (8 bits: at most 2 pad + 1 rows) and B[j][x] = 1 for x <= j <= x + 2 pad; exact
    // in the 32-bit accumulators. Warp w makes output columns 8 w .. 8 w + 7 (one n tile) for ranks 0-15 and 16-31 (two
    // m tiles), over the k-steps of 32 region columns its window reaches.
    uint8_t *colc = smem + L.cols;                       // [buffer][rank][CSTR]: column counts of the pass's ranks
    uint16_t *wc16 = (uint16_t *)(smem + L.wcount);      // [chunk row][rank][kCvWS]: window counts
    const int NK = cv_nk(TX, P), CSTR = cv_cstr(TX, P);
    const int g = lane >> 2, t = lane & 3;
    // warp w makes the window counts of one m tile (ranks 16 mt .. 16 mt + 15) at two n tiles 16 columns apart,
    // output columns xb .. xb + 7 and xb + 16 .. xb + 23: the column counts it loads serve 16 columns, and the second n
    // tile's band of ones is the first's one half k-step on, so both share one set of B fragments
    constexpr int kGroups = kWarps / 2;
    const int mt = warp / kGroups, grp = warp % kGroups, xb = 32 * (grp >> 1) + 8 * (grp & 1);
    const int ks_lo = xb >> 5, ks_hi = min(NK - 1, (xb + 23 + 2 * P) >> 5);
    uint32_t bfrag[2 * kCvMaxK + 1];  // bfrag[h]: rows (region columns) 32 ks_lo + 16 (h - 1) + 4 t + i, column xb + g
#pragma unroll
    for (int hh = 0; hh < 2 * kCvMaxK + 1; hh++) {
        uint32_t word = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int j = 32 * ks_lo + 16 * (hh - 1) + 4 * t + i, x = xb + g;
            word |= (uint32_t)(j >= x && j <= x + 2 * P) << (8 * i);
        }
        bfrag[hh] = word;
    }
    const uint32_t cbase = (uint32_t)__cvta_generic_to_shared(colc);
    const int lrow = ((lane >> 3) & 1) * 8 + (lane & 7), lcol = (lane >> 4) * 16;  // this lane's ldmatrix row address
    for (int b0 = 0;;) {
        const int lo = b0 ? b0 + kDiffs : 0, hi = b0 + kCvBins >= R ? R : b0 + kCvBins - kDiffs;
        const int off = per_pass ? 0 : b0;  // plane value of pass rank k: k + off
        if (per_pass) build_plane(b0);
        if (tid < kCvTY) rowneed[tid] = 0;
        for (int i = tid; i < kCvBins * CSTR / 16; i += kCvThreads) ((uint4 *)colc)[i] = make_uint4(0, 0, 0, 0);
        __syncthreads();
        // the pass ranks each row's pixels read: first the served pass ranks present in each row (TX / 4 lanes per
        // row, 4 pixels per lane from two aligned words of the rank plane), then, per row, the ranks those read
        for (int i = tid; i < kCvTY * kQuads; i += kCvThreads) {
            const int r = i / kQuads, q = i % kQuads;
            uint32_t bits = 0;
            if (r < rows) {
                const int at = (r + P) * CS + P + 4 * q;  // tile columns 4 q .. 4 q + 3
                const uint32_t *wp = (const uint32_t *)(rplane + (at & ~3));
                const uint32_t quad = __funnelshift_r(wp[0], wp[1], 8 * (at & 3));
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const unsigned v = (quad >> (8 * e)) & 0xFFu;
                    const int k = (int)v - off, rk = b0 + k;
                    if (v != kNoRank && 4 * q + e < cols && rk >= lo && rk < hi) bits |= 1u << k;
                }
            }
#pragma unroll
            for (int o = kQuads / 2; o; o >>= 1) bits |= __shfl_xor_sync(kFull, bits, o);
            if ((lane & (kQuads - 1)) == 0 && r < kCvTY) rowneed[r] = bits;
        }
        __syncthreads();
        if (tid < rows) {
            uint32_t present = rowneed[tid], need = 0;
            while (present) {
                const int k = __ffs(present) - 1;
                present &= present - 1;
                const uint32_t m = relneed[b0 + k];
                need |= k >= 4 ? m << (k - 4) : m >> (4 - k);
            }
            rowneed[tid] = need;
        }
        __syncthreads();
        const bool pass_any = __syncthreads_or(tid < kCvTY && rowneed[tid] != 0);
        // pass rank (0 .. 31) of region pixel (c, rr), or -1
        auto rank_at = [&](int rr, int c) -> int {
            const unsigned v = rplane[rr * CS + c];
            const int k = (int)v - off;
            return (v != kNoRank && k >= 0 && k < kCvBins) ? k : -1;
        };
        // the column counts of tile row 0: region rows 0 .. 2 pad, a thread per column (splitting the rows between two
        // threads and adding the halves measured no faster)
        if (pass_any) {
            for (int c = tid; c < RW; c += kCvThreads) {
                uint8_t *col = colc + c;
                for (int rr = 0; rr <= min(2 * P, RH - 1); rr++) {
                    const int k = rank_at(rr, c);
                    if (k >= 0) col[k * CSTR]++;
                }
            }
        }
        __syncthreads();
        // moves the column counts on from tile row t0 to t0 + 1, a thread per column (the leaving and the entering
        // pixel of a column on two threads measured slower: twice the rank reads)
        auto slide = [&](int t0) {
            const int enter = t0 + 2 * P + 1;
            for (int c = tid; c < RW; c += kCvThreads) {
                const int kl = rank_at(t0, c), ke = enter < RH ? rank_at(enter, c) : -1;
                if (kl != ke) {
                    if (kl >= 0) colc[kl * CSTR + c]--;
                    if (ke >= 0) colc[ke * CSTR + c]++;
                }
            }
        };
        // window counts of chunk row i, for the m tiles the row reads, over N k-steps (N the same for the warp)
        auto window_counts_n = [&](auto n_ksteps, int i, uint32_t need) {
            constexpr int N = decltype(n_ksteps)::value;
            if (((need >> (16 * mt)) & 0xFFFFu) == 0) return;  // no pixel of the row reads this m tile's ranks
            int acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
            const uint32_t at0 = cbase + (16 * mt + lrow) * CSTR + 32 * ks_lo + lcol;
#pragma unroll
            for (int kk = 0; kk < N; kk++) {
                uint32_t a0, a1, a2, a3;
                ldmatrix_x4(at0 + 32 * kk, a0, a1, a2, a3);
                mma_u8(acc[0], a0, a1, a2, a3, bfrag[2 * kk + 1], bfrag[2 * kk + 2]);
                mma_u8(acc[1], a0, a1, a2, a3, bfrag[2 * kk], bfrag[2 * kk + 1]);
            }
            // rank 16 mt + g (+ 8) at columns xb + 2 t and + 1, and 16 on (counts below 2^16: the low halves of the
            // accumulators)
            uint16_t *wrow = wc16 + (size_t)i * kCvBins * kCvWS + (16 * mt + g) * kCvWS + xb + 2 * t;
#pragma unroll
            for (int n = 0; n < 2; n++) {
                *(uint32_t *)(wrow + 16 * n) = __byte_perm((uint32_t)acc[n][0], (uint32_t)acc[n][1], 0x5410);
                *(uint32_t *)(wrow + 16 * n + 8 * kCvWS) = __byte_perm((uint32_t)acc[n][2], (uint32_t)acc[n][3], 0x5410);
            }
        };
        auto window_counts = [&](int i, uint32_t need) {
            switch (ks_hi - ks_lo) {  // the same for the whole warp
            case 0: window_counts_n(std::integral_constant<int, 1>{}, i, need); break;
            case 1: window_counts_n(std::integral_constant<int, 2>{}, i, need); break;
            case 2: window_counts_n(std::integral_constant<int, 3>{}, i, need); break;
            case 3: window_counts_n(std::integral_constant<int, 4>{}, i, need); break;
            default: window_counts_n(std::integral_constant<int, 5>{}, i, need); break;
            }
        };
        const int ci = tid / TX, cc = tid % TX;  // this thread's pixel in a chunk
        for (int r0 = 0; r0 < rows; r0 += kCvChunk) {
            const int n_rows = min(kCvChunk, rows - r0);
            bool chunk_any = false;
            for (int i = 0; i < n_rows; i++) {
                const int r = r0 + i;
                if (i > 0 && pass_any) {  // the counts on to row r
                    __syncthreads();  // every warp has read the counts of the row before
                    slide(r - 1);
                    __syncthreads();
                }
                const uint32_t need = rowneed[r];
                chunk_any |= need != 0;
                if (need) window_counts(i, need);
            }
            __syncthreads();
            // the counts move past this chunk beside its c-values (they touch nothing the c-values read)
            if (pass_any && r0 + kCvChunk < rows) slide(r0 + kCvChunk - 1);
            if (!chunk_any) {
                __syncthreads();
                continue;
            }
            // the chunk's c-values, one pixel per thread
            float c = 0.0f;
            bool served = false;
            const int r = r0 + ci;
            if (ci < n_rows && cc < cols) {
                const unsigned v = rplane[(r + P) * CS + cc + P];
                if (v != kNoRank) {
                    const int k = (int)v - off, rk = b0 + k;
                    if (rk >= lo && rk < hi && relneed[rk]) {
                        served = true;
                        const uint32_t nb = nbr[rk];
                        const int base = k - 4;
                        const uint16_t *wc = wc16 + (size_t)ci * kCvBins * kCvWS + cc;
                        auto count = [&](int kk) -> unsigned { return wc[kk * kCvWS]; };
                        const unsigned p0 = count(k);
                        // a diff with no neighbour (pm = 0) gives 0, which never raises c
#pragma unroll
                        for (int d = 0; d < kDiffs; d++) {
                            const unsigned o1 = (nb >> (4 * (4 + d))) & 15u, o2 = (nb >> (4 * (3 - d))) & 15u;
                            const unsigned p1 = o1 != 15u ? count(base + (int)o1) : 0u;
                            const unsigned p2 = o2 != 15u ? count(base + (int)o2) : 0u;
                            const unsigned pm = p1 > p2 ? p1 : p2;
                            if (pm) {
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
                // the first radix digit of the top-k selection, counted once per group of equal digits
                const unsigned dg = pos ? (__float_as_uint(c) >> 21) - kCvDigit0 : 0xFFFFFFFFu;
                const unsigned peers = __match_any_sync(kFull, dg);
                if (pos && lane == __ffs(peers) - 1) {
                    if (dg < kCvDigits) atomicAdd(&hist1[dg], (unsigned)__popc(peers));
                    else atomicAdd(&SL.hist[dg + kCvDigit0], (unsigned)__popc(peers));  // not reached: c in [0.5, 2^13)
                }
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
    if (tid < kCvDigits && hist1[tid]) atomicAdd(&SL.hist[kCvDigit0 + tid], hist1[tid]);
    if (tid == 0) {
        unsigned long long s = 0;
        unsigned c = 0;
        for (int k = 0; k < kWarps; k++) {
            s += red_sum[k];
            c += red_cnt[k];
        }
        if (c) {
            atomicAdd(&SL.sum_fx, s);
            atomicAdd(&SL.count, (unsigned long long)c);
        }
        if (b.tile_mass) b.tile_mass[gt] = s;
    }
    if (list_n) flush();
  };

    if (!b.tiles) {
        tile_body((int)blockIdx.x);
        return;
    }
    const unsigned count = *b.tile_count;
    for (;;) {
        if (tid == 0) next_tile = atomicAdd(b.tile_next, 1u);
        __syncthreads();
        const unsigned i = next_tile;
        if (i >= count) break;
        tile_body((int)b.tiles[i]);
        __syncthreads();
    }
}

}  // namespace

size_t cvalues_smem_bytes(int max_pad, int tile_cols) { return cv_layout(tile_cols == 128 ? 128 : 64, max_pad).total; }

namespace {
template <int TX>
cudaError_t launch_cvalues_tx(const CvBatch &b, cudaStream_t s)
{
    const size_t smem = cvalues_smem_bytes(b.max_pad, TX);
    cudaError_t e = cudaFuncSetAttribute(cvalues_kernel<TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    LaunchTimer t("cambi_cvalues", s);
    const int list_blocks = kCvListBlocks * 64 / TX;  // the same threads per SM for either width
    const int grid = b.tiles ? (b.total_tiles < list_blocks ? b.total_tiles : list_blocks) : b.total_tiles;
    cvalues_kernel<TX><<<grid, 4 * TX, smem, s>>>(b);
    return after_launch();
}

int tile_cols_of(const CvJob &j) { return j.tile_cols == 128 ? 128 : 64; }
}  // namespace

cudaError_t launch_cvalues(const CvBatch &batch, cudaStream_t s)
{
    if (batch.total_tiles <= 0) return cudaSuccess;
    CvBatch b = batch;
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
    bool has64 = false, has128 = false;
    for (int j = 0; j < b.njobs; j++) (tile_cols_of(b.job[j]) == 128 ? has128 : has64) = true;
    if (!(has64 && has128)) return has128 ? launch_cvalues_tx<128>(b, s) : launch_cvalues_tx<64>(b, s);
    // tiles of both widths: one launch per width, each over its own jobs (a tile list or per-tile masses name tiles
    // of one numbering, so they need one width)
    if (b.tiles || b.tile_mass) return cudaErrorInvalidValue;
    for (int width : {128, 64}) {
        CvBatch sub = b;
        sub.njobs = 0;
        int tiles = 0;
        for (int j = 0; j < b.njobs; j++) {
            if (tile_cols_of(b.job[j]) != width) continue;
            CvJob job = b.job[j];
            const int th = job.tile_rows ? job.tile_rows : kCvTY;
            job.first_tile = tiles;
            tiles += job.tiles_x * ((job.h + th - 1) / th);
            sub.job[sub.njobs++] = job;
        }
        sub.total_tiles = tiles;
        if (tiles == 0) continue;
        const cudaError_t e = width == 128 ? launch_cvalues_tx<128>(sub, s) : launch_cvalues_tx<64>(sub, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

const void *kernel_entry_cvalues() { return (const void *)cvalues_kernel<64>; }

}  // namespace es
