// Learned tile proposal for sm_100a: a small network predicts which 64 x 64 tiles of scale 0 carry CAMBI c-values, so
// the exact c-value kernel runs only on those tiles (and their covering tiles of scale 1) plus a random audit sample,
// with a fallback to every tile when the audit estimates that the skipped tiles matter. The reference has no
// counterpart: it computes c-values of every tile (src/kernels.cu:224-278).
//
//  * features: per 4 x 4 block of scale-0 words (value | mask << 15), the mean value as (mean - 512) / 256 and the
//    share of masked pixels (blocks outside the picture are 0);
//  * training kernels (FP32, SIMT): valid 3 x 3 convolutions forward and backward on crops, the tile loss and Adam;
//    weights are used rounded to bfloat16;
//  * predict_kernel: one 128-thread block per scale-0 tile runs all four layers on the tile's 24 x 24 feature window
//    in shared memory; the two 16 -> 16 layers are implicit-GEMM products on the fifth-generation tensor cores
//    (tcgen05.mma, bfloat16 operands from shared-memory descriptors, FP32 accumulators in tensor memory, read back
//    with tcgen05.ld), the first and last layers bfloat16 mma.sync products; tiles with no pixel that needs a c-value
//    get -inf;
//  * propose_kernel / audit_kernel: the per-step tile lists and the audit's estimate, all on the device.
#include <cuda_bf16.h>

#include "cambi_codes.h"
#include "es_kernels.h"

namespace es {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo, in the low half
    return *(const uint32_t *)&v;
}

// ---------------------------------------------------------------------------------------------------------------
// Features of the 4 x 4 block of scale-0 pixels from (X, Y); with a band, `need` tells whether a pixel of the block
// needs a c-value.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void block_features(const uint16_t *word, int w, int h, int X, int Y, const Band *bd,
                                               const uint32_t *needbits, float &f0, float &f1, bool &need)
{
    unsigned sum = 0, n = 0, m = 0;
    bool nd = false;
    // 8-byte loads need the row start (word + y w + X) 8-byte aligned: X and w multiples of 4, word 8-byte aligned
    const bool vec = X >= 0 && X + 4 <= w && (X & 3) == 0 && (w & 3) == 0 && (((uintptr_t)word) & 7) == 0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int y = Y + r;
        if (y < 0 || y >= h) continue;
        unsigned q[4];
        int cnt = 0;
        if (vec) {
            const uint2 v = __ldg((const uint2 *)(word + (size_t)y * w + X));
            q[0] = v.x & 0xFFFFu;
            q[1] = v.x >> 16;
            q[2] = v.y & 0xFFFFu;
            q[3] = v.y >> 16;
            cnt = 4;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int x = X + k;
                if (x >= 0 && x < w) q[cnt++] = word[(size_t)y * w + x];
            }
        }
        for (int k = 0; k < cnt; k++) {
            sum += q[k] & 0x7FFFu;
            m += (q[k] >> 15) & 1u;
            if (bd) {  // needbits: bit c set when code c needs a c-value
                const uint16_t c = code_of(q[k], *bd);
                nd |= c != kNone && ((needbits[c >> 5] >> (c & 31)) & 1u);
            }
        }
        n += cnt;
    }
    f0 = n ? (float)(((double)sum / (double)n - 512.0) / 256.0) : 0.0f;
    f1 = (float)((double)m / 16.0);
    need = nd;
}

__global__ void __launch_bounds__(256) net_features_kernel(const uint16_t *word, int w, int h, const int *xy, int n, int fw,
                                                           int fh, float *out)
{
    const size_t per = (size_t)fw * fh, total = per * n;
    for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < total; i += (size_t)gridDim.x * 256) {
        const int c = (int)(i / per), r = (int)(i - (size_t)c * per), v = r / fw, u = r - v * fw;
        float f0, f1;
        bool need;
        block_features(word, w, h, xy[2 * c] + 4 * u, xy[2 * c + 1] + 4 * v, nullptr, nullptr, f0, f1, need);
        out[(size_t)c * 2 * per + r] = f0;
        out[(size_t)c * 2 * per + per + r] = f1;
    }
}

// The feature map of every picture of a prediction (one thread per 4 x 4 block) and the need flag of each scale-0 tile.
__global__ void __launch_bounds__(256) feature_map_kernel(const __grid_constant__ PredBatch b)
{
    __shared__ uint32_t needbits[32];
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int code = (warp + 8 * k) * 32 + lane;
            const unsigned m = __ballot_sync(0xffffffffu, code < b.band.band_size && needs_cvalue(code, b.band));
            if (lane == 0) needbits[warp + 8 * k] = m;
        }
    }
    __syncthreads();
    const int j = find_job(b.njobs, (int)blockIdx.x, [&](int k) { return b.job[k].first_block; });
    const PredJob &J = b.job[j];
    const int fw = (J.w + 3) / 4, fh = (J.h + 3) / 4;
    const int i = (blockIdx.x - J.first_block) * 256 + threadIdx.x;
    if (i >= fw * fh) return;
    const int v = i / fw, u = i - v * fw;
    float f0, f1;
    bool need;
    block_features(J.word, J.w, J.h, 4 * u, 4 * v, &b.band, needbits, f0, f1, need);
    J.feat[i] = make_float2(f0, f1);
    if (need) {  // most blocks of a tile that needs c-values find the flag already set: read before the atomic
        unsigned *flag = &b.need[J.first_tile + (v >> 4) * J.tiles_x + (u >> 4)];
        if (!*(volatile unsigned *)flag) atomicOr(flag, 1u);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Training: valid 3 x 3 convolutions on NCHW float crops, weights rounded to bfloat16.
// ---------------------------------------------------------------------------------------------------------------
template <int CI, int CO>
__global__ void __launch_bounds__(256) conv_fwd_kernel(const float *in, int n, int h, int w, const float *P, int woff, int boff,
                                                       bool relu, float *out)
{
    __shared__ float W[CO * CI * 9], B[CO];
    for (int i = threadIdx.x; i < CO * CI * 9; i += 256) W[i] = bf16r(P[woff + i]);
    for (int i = threadIdx.x; i < CO; i += 256) B[i] = bf16r(P[boff + i]);
    __syncthreads();
    const int ho = h - 2, wo = w - 2;
    const size_t plane = (size_t)ho * wo, total = plane * n;
    for (size_t idx = (size_t)blockIdx.x * 256 + threadIdx.x; idx < total; idx += (size_t)gridDim.x * 256) {
        const int nn = (int)(idx / plane), r = (int)(idx - (size_t)nn * plane), y = r / wo, x = r - y * wo;
        float acc[CO];
#pragma unroll
        for (int co = 0; co < CO; co++) acc[co] = B[co];
        for (int ci = 0; ci < CI; ci++) {
            const float *src = in + ((size_t)(nn * CI + ci) * h + y) * w + x;
#pragma unroll
            for (int k = 0; k < 9; k++) {
                const float v = src[(k / 3) * w + (k % 3)];
#pragma unroll
                for (int co = 0; co < CO; co++) acc[co] = __fmaf_rn(v, W[(co * CI + ci) * 9 + k], acc[co]);
            }
        }
#pragma unroll
        for (int co = 0; co < CO; co++)
            out[((size_t)(nn * CO + co) * ho + y) * wo + x] = relu ? fmaxf(acc[co], 0.0f) : acc[co];
    }
}

// gin = (full correlation of gout with the flipped kernel) x (in > 0): the gradient of the layer's input, through the
// ReLU that produced it.
template <int CI, int CO>
__global__ void __launch_bounds__(256) conv_bwd_data_kernel(const float *gout, const float *in, int n, int h, int w,
                                                            const float *P, int woff, float *gin)
{
    __shared__ float W[CO * CI * 9];
    for (int i = threadIdx.x; i < CO * CI * 9; i += 256) W[i] = bf16r(P[woff + i]);
    __syncthreads();
    const int ho = h - 2, wo = w - 2;
    const size_t plane = (size_t)h * w, total = plane * n;
    for (size_t idx = (size_t)blockIdx.x * 256 + threadIdx.x; idx < total; idx += (size_t)gridDim.x * 256) {
        const int nn = (int)(idx / plane), r = (int)(idx - (size_t)nn * plane), y = r / w, x = r - y * w;
        float acc[CI];
#pragma unroll
        for (int ci = 0; ci < CI; ci++) acc[ci] = 0.0f;
        for (int co = 0; co < CO; co++) {
#pragma unroll
            for (int k = 0; k < 9; k++) {
                const int oy = y - k / 3, ox = x - k % 3;
                if (oy < 0 || oy >= ho || ox < 0 || ox >= wo) continue;
                const float g = gout[((size_t)(nn * CO + co) * ho + oy) * wo + ox];
#pragma unroll
                for (int ci = 0; ci < CI; ci++) acc[ci] = __fmaf_rn(g, W[(co * CI + ci) * 9 + k], acc[ci]);
            }
        }
#pragma unroll
        for (int ci = 0; ci < CI; ci++) {
            const size_t at = ((size_t)(nn * CI + ci) * h + y) * w + x;
            gin[at] = in[at] > 0.0f ? acc[ci] : 0.0f;
        }
    }
}

// One block per (co, ci): the 9 weight gradients (and the bias gradient when ci == 0), summed in a fixed order.
template <int CI, int CO>
__global__ void __launch_bounds__(256) conv_bwd_weight_kernel(const float *gout, const float *in, int n, int h, int w,
                                                              float *G, int woff, int boff)
{
    __shared__ float part[8][10];
    const int co = blockIdx.x / CI, ci = blockIdx.x % CI;
    const int ho = h - 2, wo = w - 2;
    const size_t plane = (size_t)ho * wo, total = plane * n;
    float acc[10];
#pragma unroll
    for (int k = 0; k < 10; k++) acc[k] = 0.0f;
    for (size_t idx = threadIdx.x; idx < total; idx += 256) {
        const int nn = (int)(idx / plane), r = (int)(idx - (size_t)nn * plane), y = r / wo, x = r - y * wo;
        const float g = gout[((size_t)(nn * CO + co) * ho + y) * wo + x];
        const float *src = in + ((size_t)(nn * CI + ci) * h + y) * w + x;
#pragma unroll
        for (int k = 0; k < 9; k++) acc[k] = __fmaf_rn(g, src[(k / 3) * w + (k % 3)], acc[k]);
        acc[9] += g;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 10; k++) {
        float v = acc[k];
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        if (lane == 0) part[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        float s = 0.0f;
        for (int k = 0; k < 8; k++) s += part[k][threadIdx.x];
        if (threadIdx.x < 9) G[woff + (co * CI + ci) * 9 + threadIdx.x] = s;
        else if (ci == 0) G[boff + co] = s;
    }
}

// One block per crop: the mean of each 16 x 16 block of z against its label; gz = d loss / d z with
// loss = mean over all tiles of (mean - label)^2.
__global__ void __launch_bounds__(256) net_loss_kernel(const float *z, const float *labels, int n, int ta, int tb, float *gz,
                                                       float *loss_parts)
{
    const int c = blockIdx.x, W = 16 * tb, H = 16 * ta, tiles = ta * tb;
    const float scale = 2.0f / (float)(n * tiles) / 256.0f;
    const int row = threadIdx.x & 15;
    for (int t0 = 0; t0 < tiles; t0 += 16) {  // the same trip count for every thread: the shuffles see full warps
        const int t = t0 + (threadIdx.x >> 4), by = t / tb, bx = t % tb;
        const bool on = t < tiles;
        float s = 0.0f;
        if (on) {
            const float *src = z + (size_t)c * H * W + (size_t)(16 * by + row) * W + 16 * bx;
#pragma unroll
            for (int k = 0; k < 16; k++) s += src[k];
        }
#pragma unroll
        for (int o = 8; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
        if (!on) continue;
        const float d = s / 256.0f - labels[(size_t)c * tiles + t];
        if (row == 0) loss_parts[(size_t)c * tiles + t] = d * d;
        float *dst = gz + (size_t)c * H * W + (size_t)(16 * by + row) * W + 16 * bx;
#pragma unroll
        for (int k = 0; k < 16; k++) dst[k] = d * scale;
    }
}

__global__ void net_adam_kernel(float *P, float *R, const float *G, float *M, float *V, int count, float lr, float b1, float b2,
                                float eps, int t)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.0f - b1) * g, v = b2 * V[i] + (1.0f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    const float p = P[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    P[i] = p;
    R[i] = bf16r(p);
}

// ---------------------------------------------------------------------------------------------------------------
// Inference: one block of 128 threads per scale-0 tile, all four layers in shared memory.
// ---------------------------------------------------------------------------------------------------------------
constexpr int kPT = 128;
constexpr int kPredBlocks = 148 * 5;  // persistent grid: 5 blocks of 42 KB (and 64 tensor-memory columns) per SM
// Layers 1 and 2 are products of 128 output rows on the tensor cores, over the input's raster: output row oy iw + ox
// (iw = the input's width), so a layer computes ceil(ow iw / 128) blocks of rows and reads the input up to row
// 128 blocks + 2 iw + 2; its planes have that many rows (zero past the picture, computed and dropped).
constexpr int kL1Blocks = (20 * 22 + 127) / 128, kL1Rows = 128 * kL1Blocks + 2 * 22 + 8;  // 4 blocks, 564 rows
constexpr int kL2Blocks = (18 * 20 + 127) / 128, kL2Rows = 128 * kL2Blocks + 2 * 20 + 8;  // 3 blocks, 432 rows
constexpr int kTmemCols = 16 * kL1Blocks;                                                  // 64
struct PredSmem {
    float b0[16], w3[145];                        // layer 0's biases; layer 3's weights then bias (bfloat16 values)
    float b12[2][16];
    // layer 1's input (layer 0's 22 x 22 output): two planes of kL1Rows 16-byte rows, channels 8 h .. 8 h + 7 of pixel p
    // in plane h, row p; later layer 2's 18 x 18 output in the head's layout ([pixel][16 channels], phys_half)
    __align__(128) uint32_t a1[2 * kL1Rows * 4];
    // layer 2's input (layer 1's 20 x 20 output), the same plane form; until layer 1 writes it, its first 4.6 KB hold
    // the tile's features (per pixel the (head, remainder) bfloat16 pairs of channels 0, 1), rows the planes' padding
    // does not reach
    __align__(128) uint32_t a2[2 * kL2Rows * 4];
    // the B operands of layers 1 and 2: [layer][tap][K half][output channel n][4 words of 2 input channels]
    __align__(128) uint32_t wt[2 * 9 * 128];
    uint64_t bar;   // the products' completion barrier
    uint32_t tmem;  // the block's tensor-memory columns
    float part[kPT / 32];
};

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

// Activation planes hold pixel p's 16 channels in 32 bytes, its two 16-byte halves swapped when bit 2 of p is set,
// so the 8 rows an ldmatrix phase reads (consecutive pixels) fall on different banks.
__device__ __forceinline__ int phys_half(int p, int half) { return half ^ ((p >> 2) & 1); }

// ---- fifth-generation tensor cores (tcgen05): products in tensor memory from shared-memory operands ----------------
// A shared-memory matrix descriptor without swizzle, K-major: rows of 16 bytes (8 bfloat16 of K) contiguous, groups of
// 8 rows `sbo` bytes apart, the two 8-wide halves of K `lbo` bytes apart; version 1 (sm_100) in bits 46-47.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           ((uint64_t)1 << 46);
}
// The instruction descriptor of a bfloat16 product with FP32 accumulation, both operands K-major, M = 128, N = 16.
constexpr uint32_t kUmmaIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

// D (tensor memory, 128 lanes x 16 FP32 columns) = A (128 x 16) x B (16 x 16)^T, plus D when `accumulate`.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                 ::"r"(tmem_d), "l"(a), "l"(b), "r"(kUmmaIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
// The products issued so far arrive on the barrier when they are done.
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"((uint32_t)__cvta_generic_to_shared(bar)) : "memory");
}
// Waits, a bounded number of times, for the barrier's phase `parity` to complete; false if it never did.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (int it = 0; it < (1 << 20); it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}
// This warp's 32 lanes of tensor memory (its quarter of the 128), 16 columns from `taddr`, as FP32; the values may be
// used only after a tcgen05.wait::ld.
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, float (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]), "=f"(v[8]),
                   "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy writes to shared memory made visible to the tensor cores' reads (before a barrier and the products).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One 16 -> 16 layer (bias, ReLU, bfloat16) on the tensor cores with tcgen05. The input is layer planes of `rows`
// 16-byte rows (channels 8 h .. 8 h + 7 of pixel p in plane h, row p; pixels row by row, IW wide, zero past the
// picture). Output row q = oy IW + ox of the product is output pixel (oy, ox): tap (dy, dx) multiplies the input from
// row q + dy IW + dx, so each block of 128 output rows is 9 products (one per tap, accumulated in 16 tensor-memory
// columns) whose A operand is the planes from the tap's row on; B is the tap's 16 x 16 weights. Thread 0 issues them,
// every thread then reads its own row of each block (warp w: lanes 32 w .. 32 w + 31) and hands the output pixels
// (ox < OW, oy < OW) with their 8 packed channel pairs to `store`. False if the products never completed.
template <int IW, int OW, int BLOCKS, typename Store>
__device__ __forceinline__ bool umma_layer(PredSmem &sm, const uint32_t *in, int rows, int layer, uint32_t &phase,
                                           const float *bias, Store store)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    fence_async_smem();  // this thread's writes of the input (and of the weights) reach the tensor cores' reads
    tc_fence_before();   // and its reads of tensor memory (the previous layer's) are done before the barrier
    __syncthreads();
    tc_fence_after();
    // lane 0 of warp m issues block m's nine products and commits them (the barrier expects one arrival per warp);
    // a descriptor's start field counts 16 bytes, so a tap's row offset is added to it directly
    if (lane == 0) {
        const int m = warp;
        const uint32_t in_s = (uint32_t)__cvta_generic_to_shared(in), w_s = (uint32_t)__cvta_generic_to_shared(sm.wt);
        const uint64_t a0 = umma_desc(in_s + 16u * 128u * m, 16u * rows, 128u), b0 = umma_desc(w_s + 512u * 9 * layer, 256u, 128u);
        if (m < BLOCKS) {
#pragma unroll
            for (int k = 0; k < 9; k++) umma_bf16(sm.tmem + 16u * m, a0 + (uint64_t)((k / 3) * IW + (k % 3)), b0 + (uint64_t)(32 * k), k > 0);
        }
        umma_commit(&sm.bar);  // with nothing issued it arrives at once
    }
    const bool ok = mbar_wait(&sm.bar, phase);
    phase ^= 1u;
    tc_fence_after();
    if (!ok) return false;
    auto emit = [&](int m, const float (&v)[16]) {
        const int q = 128 * m + 32 * warp + lane, oy = q / IW, ox = q - oy * IW;
        if (oy < OW && ox < OW) {
            uint32_t packed[8];
#pragma unroll
            for (int i = 0; i < 8; i++)
                packed[i] = pack_bf16(fmaxf(v[2 * i] + bias[2 * i], 0.0f), fmaxf(v[2 * i + 1] + bias[2 * i + 1], 0.0f));
            store(oy * OW + ox, packed);
        }
    };
    const uint32_t tl = sm.tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
    for (int m = 0; m < BLOCKS; m += 2) {  // two loads in flight, then one wait
        float v0[16], v1[16];
        tmem_ld16_nowait(tl + 16u * m, v0);
        if (m + 1 < BLOCKS) tmem_ld16_nowait(tl + 16u * (m + 1), v1);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        emit(m, v0);
        if (m + 1 < BLOCKS) emit(m + 1, v1);
    }
    return true;
}

// Layer 0 (2 -> 16) on the tensor cores, 22 x 22 outputs from the 24 x 24 feature window: each FP32 feature enters as
// a bfloat16 head and the bfloat16 of its remainder (k = 4 tap + 2 part + channel), so the products keep about 16 bits
// of it; one 32-bit load gives a lane both channels of a pixel's part. Warp w takes m tiles w, w + 4, ... The output
// goes to layer 1's two planes (channels 8 j .. 8 j + 7 of pixel p in plane j, row p).
__device__ __forceinline__ void mma_layer0(const uint32_t (*fin)[2], uint32_t *out, const uint32_t *frags, const float *bias)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int ow = 22, iw = kFeatTile, npx = ow * ow, tiles = (npx + 15) / 16;
    const int g = lane >> 2, t = lane & 3, part = t & 1;
    for (int mt = warp; mt < tiles; mt += kPT / 32) {
        int base[2];
#pragma unroll
        for (int hrow = 0; hrow < 2; hrow++) {
            const int p = min(16 * mt + g + 8 * hrow, npx - 1);  // rows past the last pixel read a valid one, not stored
            const int oy = p / ow;
            base[hrow] = oy * iw + (p - oy * ow);
        }
        float c[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
        for (int ks = 0; ks < 3; ks++) {
            const int ta = 4 * ks + (t >> 1), tb = ta + 2;  // the taps of k 16 ks + 2 t and 16 ks + 2 t + 8
            auto ld = [&](int hrow, int tap) -> uint32_t {
                return tap < 9 ? fin[base[hrow] + (tap / 3) * iw + tap % 3][part] : 0u;
            };
            const uint32_t a0 = ld(0, ta), a1 = ld(1, ta), a2 = ld(0, tb), a3 = ld(1, tb);
            const uint32_t *fk = frags + ks * 4 * 32 + lane;
            mma_bf16(c[0], a0, a1, a2, a3, fk[0], fk[32]);
            mma_bf16(c[1], a0, a1, a2, a3, fk[64], fk[96]);
        }
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int ch = 8 * j + 2 * t;
#pragma unroll
            for (int hrow = 0; hrow < 2; hrow++) {
                const int pr = 16 * mt + g + 8 * hrow;
                if (pr >= npx) continue;
                const float v0 = fmaxf(c[j][2 * hrow] + bias[ch], 0.0f), v1 = fmaxf(c[j][2 * hrow + 1] + bias[ch + 1], 0.0f);
                out[j * (kL1Rows * 4) + pr * 4 + t] = pack_bf16(v0, v1);  // plane j, row pr
            }
        }
    }
}

// Layer 3 (16 -> 1) on the 16 x 16 output from the 18 x 18 plane `in`: one 8-wide n tile whose column 0 holds the
// output channel. Returns this warp's sum of its output pixels (lanes with lane % 4 == 0 hold column 0 of rows g and
// g + 8), bias excluded.
__device__ __forceinline__ float mma_head(const uint32_t *in, const uint32_t *frags)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int mrow = ((lane >> 3) & 1) * 8 + (lane & 7), khalf = lane >> 4;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(in);
    uint32_t bf[9][2];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        bf[k][0] = frags[k * 2 * 32 + lane];
        bf[k][1] = frags[k * 2 * 32 + 32 + lane];
    }
    float sum = 0.0f;
    for (int mt = warp; mt < 16; mt += kPT / 32) {  // m tile mt: output row mt, 16 pixels
        float c[4] = {0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const int q = (mt + k / 3) * 18 + mrow + k % 3;
            uint32_t a0, a1, a2, a3;
            ldmatrix_x4(base + q * 32 + phys_half(q, khalf) * 16, a0, a1, a2, a3);
            mma_bf16(c, a0, a1, a2, a3, bf[k][0], bf[k][1]);
        }
        if ((lane & 3) == 0) sum += c[0] + c[2];
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
    return sum;
}

// Persistent: each block loads the parameters once, allocates its tensor-memory columns, then takes tiles from a
// counter (need[total_tiles]) until none is left. Should a product never complete (a bounded wait), the block stops
// using the tensor cores and gives every tile it takes the prediction +inf, so those tiles are computed exactly.
__global__ void __launch_bounds__(kPT, 5) predict_kernel(const __grid_constant__ PredBatch b)
{
    __shared__ PredSmem sm;
    __shared__ int next;
    uint32_t(*feat)[2] = (uint32_t(*)[2])sm.a2;
    static_assert(kFeatTile * kFeatTile * 2 <= 400 * 4, "the features stay below layer 2's padding rows");
    const int tid = threadIdx.x;
    if (tid < 16) sm.b0[tid] = b.params[net_b(0) + tid];
    for (int i = tid; i < 145; i += kPT) sm.w3[i] = b.params[net_w(3) + i];
    if (tid < 32) sm.b12[tid >> 4][tid & 15] = b.params[(tid < 16 ? net_b(1) : net_b(2)) + (tid & 15)];
    // the planes past the pictures stay zero (only dropped output rows read them)
    for (int i = tid; i < 2 * kL1Rows; i += kPT) ((uint4 *)sm.a1)[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < 2 * kL2Rows; i += kPT) ((uint4 *)sm.a2)[i] = make_uint4(0, 0, 0, 0);
    // layers 1 and 2's weights from their mma.sync fragments (word i: layer 1 + (i / 128) / 9, tap (i / 128) % 9,
    // n = 8 ((i / 64) % 2) + (i % 32) / 4, input channels c, c + 1 with c = 2 (i % 4) + 8 ((i / 32) % 2)) into the
    // tensor cores' K-major tiles: half c / 8, row n, word (c % 8) / 2
    for (int i = tid; i < kNetFrags12; i += kPT) {
        const int lane = i & 31, r = (i >> 5) & 1, j = (i >> 6) & 1, lk = i >> 7, n = 8 * j + (lane >> 2);
        sm.wt[lk * 128 + r * 64 + n * 4 + (lane & 3)] = b.frags[i];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(&sm.bar)), "r"(kPT / 32));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(&sm.tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t phase = 0;
    bool broken = false;
    for (;;) {
        __syncthreads();  // every thread is done with the previous tile (and with `next`)
        if (tid == 0) next = (int)atomicAdd(b.need + b.total_tiles, 1u);
        __syncthreads();
        const int gt = next;
        if (gt >= b.total_tiles) break;
        if (!b.need[gt] || broken) {  // nothing to predict, or no tensor cores: the same for the whole block
            if (tid == 0) b.pred[gt] = b.need[gt] ? INFINITY : -INFINITY;
            continue;
        }
        const int j = find_job(b.njobs, gt, [&](int k) { return b.job[k].first_tile; });
        const PredJob &J = b.job[j];
        const int tile = gt - J.first_tile, tx = tile % J.tiles_x, ty = tile / J.tiles_x;
        // the 24 x 24 feature window: map pixels 16 tx - 4 .. 16 tx + 19 (a tile is 16 map pixels; 0 outside the map)
        const int fw = (J.w + 3) / 4, fh = (J.h + 3) / 4;
        for (int i = tid; i < kFeatTile * kFeatTile; i += kPT) {
            const int v = i / kFeatTile, u = i - v * kFeatTile, gu = 16 * tx - 4 + u, gv = 16 * ty - 4 + v;
            float2 f = make_float2(0.0f, 0.0f);
            if (gu >= 0 && gu < fw && gv >= 0 && gv < fh) f = J.feat[(size_t)gv * fw + gu];
            const float h0 = bf16r(f.x), h1 = bf16r(f.y);
            feat[i][0] = pack_bf16(h0, h1);
            feat[i][1] = pack_bf16(f.x - h0, f.y - h1);  // the remainders are exact in FP32
        }
        __syncthreads();
        // layer 0's B fragments come from global memory (L1-resident), layers 1 and 2's from `wt`
        mma_layer0(feat, sm.a1, b.frags + kNetFrags3, sm.b0);  // layer 0: 22 x 22, into layer 1's planes
        bool ok = umma_layer<22, 20, kL1Blocks>(sm, sm.a1, kL1Rows, 0, phase, sm.b12[0], [&](int q, const uint32_t(&pk)[8]) {
            ((uint4 *)sm.a2)[q] = make_uint4(pk[0], pk[1], pk[2], pk[3]);  // layer 1: 20 x 20, into layer 2's planes
            ((uint4 *)sm.a2)[kL2Rows + q] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        });
        if (ok)
            ok = umma_layer<20, 18, kL2Blocks>(sm, sm.a2, kL2Rows, 1, phase, sm.b12[1], [&](int q, const uint32_t(&pk)[8]) {
                // layer 2: 18 x 18, into a1 in the head's layout
                *(uint4 *)(sm.a1 + q * 8 + phys_half(q, 0) * 4) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                *(uint4 *)(sm.a1 + q * 8 + phys_half(q, 1) * 4) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            });
        if (__syncthreads_or(!ok)) {
            broken = true;
            if (tid == 0) b.pred[gt] = INFINITY;
            continue;
        }
        // layer 3: 16 -> 1 on 16 x 16 (tensor cores), then the tile mean (a fixed order of additions)
        const float s = mma_head(sm.a1, b.frags + kNetFrags12);
        if ((tid & 31) == 0) sm.part[tid >> 5] = s;
        __syncthreads();
        if (tid == 0) b.pred[gt] = ((sm.part[0] + sm.part[1]) + (sm.part[2] + sm.part[3])) / 256.0f + sm.w3[144];
    }
    if (broken) mbar_wait(&sm.bar, phase ^ 1u);  // once more, bounded, for the products that did not complete
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem), "r"(kTmemCols));
}

// ---------------------------------------------------------------------------------------------------------------
// Proposal and audit of a frame step.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    // SplitMix64's finaliser (Steele, Lea and Flood 2014)
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void __launch_bounds__(256) propose_kernel(const __grid_constant__ ProposeBatch b)
{
    const unsigned long long frame = *b.frame;
    for (int gt = blockIdx.x * 256 + threadIdx.x; gt < b.total_tiles; gt += gridDim.x * 256) {
        const int j = find_job(b.njobs, gt, [&](int k) { return b.job[k].first_tile; });
        const ProposeJob &J = b.job[j];
        const int tile = gt - J.first_tile, tx = tile % J.tiles_x, ty = tile / J.tiles_x;
        uint8_t kind = kTileRun;
        if (J.scale < 2) {
            const int s = J.scale;
            float best = -INFINITY;
            for (int y = ty << s; y < min((ty + 1) << s, J.pred_tiles_y); y++)
                for (int x = tx << s; x < min((tx + 1) << s, J.pred_tiles_x); x++)
                    best = fmaxf(best, b.pred[J.pred_first + y * J.pred_tiles_x + x]);
            if (best == -INFINITY) {
                kind = kTileEmpty;  // scale 0: nothing to compute; scale 1: left to the fallback, unaudited
            } else if (best < (b.pic_threshold ? b.pic_threshold[J.picture] : b.threshold)) {
                const unsigned long long hsh = mix64(frame * 0x100000001B3ull ^ ((unsigned long long)J.picture << 40) ^
                                                     ((unsigned long long)s << 36) ^ (unsigned long long)tile);
                kind = (unsigned)(hsh % 1000ull) < b.audit_permille[s] ? kTileAudit : kTileSkip;
            }
            if (kind == kTileAudit) atomicAdd(&b.n_audit[j], 1u);
            if (kind == kTileSkip) atomicAdd(&b.n_skip[j], 1u);
        }
        b.kind[gt] = kind;
        if (kind == kTileRun || kind == kTileAudit) b.list_a[atomicAdd(b.count_a, 1u)] = (unsigned)gt;
        else if (kind == kTileSkip || (kind == kTileEmpty && J.scale == 1)) b.list_b[atomicAdd(b.count_b, 1u)] = (unsigned)gt;
    }
}

// One block per picture: the largest skip threshold whose skipped scale-0 tiles are predicted to change the score by
// at most the budget. Predicted contributions are binned by prediction (kBudgetBinsPerUnit bins per unit from 0, the
// last bin open above) in fixed point (2^-40 of a score point), so the result does not depend on the order of adds.
__global__ void __launch_bounds__(kBudgetBins) budget_kernel(const __grid_constant__ BudgetBatch b)
{
    __shared__ unsigned long long bins[kBudgetBins];
    __shared__ unsigned long long warp_sums[kBudgetBins / 32];
    const BudgetJob &J = b.job[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    bins[tid] = 0;
    __syncthreads();
    const int tiles = J.tiles_x * J.tiles_y;
    for (int t = tid; t < tiles; t += kBudgetBins) {
        const float p = b.pred[J.pred_first + t];
        if (p == -INFINITY) continue;  // nothing to compute in the tile
        const int tx = t % J.tiles_x, ty = t / J.tiles_x;
        const int px = min(kCvTX, J.w - tx * kCvTX) * min(kCvTY, J.h - ty * kCvTY);
        const double c = J.scale * expm1((double)fmaxf(p, 0.0f)) * (double)px;
        const double fx = fmin(c * 1099511627776.0, 2.0e15);  // 2^40 units; 8192 tiles at the cap stay below 2^64
        const int bin = min(kBudgetBins - 1, max(0, (int)(p * kBudgetBinsPerUnit)));
        atomicAdd(&bins[bin], (unsigned long long)fx);
    }
    __syncthreads();
    // inclusive prefix over the bins: bin `tid` in thread tid
    unsigned long long v = bins[tid];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long u = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long u = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += u;
        }
        warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const unsigned long long incl = v + (warp ? warp_sums[warp - 1] : 0ull);
    const unsigned long long budget = (unsigned long long)fmin(b.budget * 1099511627776.0, 1.8e19);
    // bins 0 .. n - 1 fit the budget; the threshold is the lower edge of bin n
    const int n = __syncthreads_count(incl <= budget);
    if (tid == 0) {
        const float t = n >= kBudgetBins ? INFINITY : (float)n / kBudgetBinsPerUnit;
        b.pic_threshold[J.picture] = fmaxf(t, b.threshold);
    }
}

// One block per picture: the audited tiles' c-value mass, scaled up to the skipped tiles, as a change of the score.
__global__ void __launch_bounds__(256) audit_kernel(const __grid_constant__ AuditBatch b)
{
    __shared__ unsigned long long part[8];
    __shared__ unsigned part_run[8];
    const AuditJob &J = b.job[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double weight[2] = {16.0, 8.0};
    double est = 0.0;
    ProposalStats st{};
    for (int s = 0; s < 2; s++) {
        unsigned long long mass = 0;
        unsigned run = 0;
        for (int t = threadIdx.x; t < J.tiles[s]; t += 256) {
            const int gt = J.first_tile[s] + t;
            const uint8_t k = b.kind[gt];
            if (k == kTileAudit) mass += b.tile_mass[gt];
            run += k == kTileRun || k == kTileAudit;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            mass += __shfl_xor_sync(kFull, mass, o);
            run += __shfl_xor_sync(kFull, run, o);
        }
        if (lane == 0) {
            part[warp] = mass;
            part_run[warp] = run;
        }
        __syncthreads();
        unsigned long long total = 0;
        unsigned runs = 0;
        for (int k = 0; k < 8; k++) {
            total += part[k];
            runs += part_run[k];
        }
        __syncthreads();
        const unsigned na = b.n_audit[J.job[s]], ns = b.n_skip[J.job[s]];
        st.run[s] = runs - na;
        st.audited[s] = na;
        st.skipped[s] = ns;
        if (na > 0 && ns > 0) {
            const double missing = (double)total / 16777216.0 * ((double)ns / (double)na);
            est += weight[s] * missing / J.k[s] / ((double)J.window * (double)J.window);
        }
    }
    if (threadIdx.x == 0) {
        const int fb = est > b.tolerance;
        b.run[blockIdx.x] = fb;
        st.estimate = (float)est;
        st.fallback = fb;
        b.stats[blockIdx.x] = st;
    }
}

// B fragments of layers 1 and 2 from the rounded parameters: word [l][k][j][r][lane] holds, for output channel
// n = 8 j + lane / 4 and input channels c = 2 (lane % 4) + 8 r and c + 1, the two weights of tap k (low half: c).
__global__ void net_pack_kernel(const float *R, uint32_t *frags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kNetFrags) return;
    if (i >= kNetFrags3) {  // layer 0: word [ks][j][r][lane]: n = 8 j + lane / 4, k rows 16 ks + 2 (lane % 4) + 8 r, + 1
        const int q = i - kNetFrags3, lane = q & 31, r = (q >> 5) & 1, j = (q >> 6) & 1, ks = q >> 7;
        const int n = 8 * j + (lane >> 2), tap = 4 * ks + 2 * r + ((lane & 3) >> 1);  // k = 4 tap + 2 part + channel
        const float *W = R + net_w(0);
        frags[i] = tap < 9 ? pack_bf16(W[(n * 2 + 0) * 9 + tap], W[(n * 2 + 1) * 9 + tap]) : 0u;
        return;
    }
    if (i >= kNetFrags12) {  // layer 3: word [k][r][lane], column n = lane / 4 holds the weights when n == 0, else 0
        const int q = i - kNetFrags12, lane = q & 31, r = (q >> 5) & 1, k = q >> 6;
        const int n = lane >> 2, c = 2 * (lane & 3) + 8 * r;
        const float *W = R + net_w(3);
        frags[i] = n == 0 ? pack_bf16(W[c * 9 + k], W[(c + 1) * 9 + k]) : 0u;
        return;
    }
    const int lane = i & 31, r = (i >> 5) & 1, j = (i >> 6) & 1, k = (i >> 7) % 9, l = 1 + (i >> 7) / 9;
    const int n = 8 * j + (lane >> 2), c = 2 * (lane & 3) + 8 * r;
    const float *W = R + net_w(l);
    frags[i] = pack_bf16(W[(n * 16 + c) * 9 + k], W[(n * 16 + c + 1) * 9 + k]);
}

unsigned grid_for(size_t total) { return (unsigned)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16); }

}  // namespace

cudaError_t launch_predict(PredBatch &b, cudaStream_t s)
{
    if (b.total_tiles <= 0) return cudaSuccess;
    int blocks = 0;
    for (int j = 0; j < b.njobs; j++) {
        b.job[j].first_block = blocks;
        blocks += (int)((feature_map_size(b.job[j].w, b.job[j].h) + 255) / 256);
    }
    if (b.features_ready) {  // only the tile counter after the need flags
        cudaError_t e = cudaMemsetAsync(b.need + b.total_tiles, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) return e;
    } else {
        cudaError_t e = cudaMemsetAsync(b.need, 0, sizeof(unsigned) * (b.total_tiles + 1), s);
        if (e != cudaSuccess) return e;
        {
            LaunchTimer t("proposal_features", s);
            feature_map_kernel<<<blocks, 256, 0, s>>>(b);
        }
        e = after_launch();
        if (e != cudaSuccess) return e;
    }
    LaunchTimer t("proposal_predict", s);
    predict_kernel<<<b.total_tiles < kPredBlocks ? b.total_tiles : kPredBlocks, kPT, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_net_features(const uint16_t *word, int w, int h, const int *xy, int n, int fw, int fh, float *out,
                                cudaStream_t s)
{
    const size_t total = (size_t)fw * fh * n;
    if (!total) return cudaSuccess;
    LaunchTimer t("proposal_features", s);
    net_features_kernel<<<grid_for(total), 256, 0, s>>>(word, w, h, xy, n, fw, fh, out);
    return after_launch();
}

cudaError_t launch_net_forward(int layer, const float *in, int n, int h, int w, const float *params, float *out, cudaStream_t s)
{
    const size_t total = (size_t)(h - 2) * (w - 2) * n;
    if (!total) return cudaSuccess;
    LaunchTimer t("proposal_train_forward", s);
    const unsigned g = grid_for(total);
    switch (layer) {
    case 0: conv_fwd_kernel<2, 16><<<g, 256, 0, s>>>(in, n, h, w, params, net_w(0), net_b(0), true, out); break;
    case 1: conv_fwd_kernel<16, 16><<<g, 256, 0, s>>>(in, n, h, w, params, net_w(1), net_b(1), true, out); break;
    case 2: conv_fwd_kernel<16, 16><<<g, 256, 0, s>>>(in, n, h, w, params, net_w(2), net_b(2), true, out); break;
    case 3: conv_fwd_kernel<16, 1><<<g, 256, 0, s>>>(in, n, h, w, params, net_w(3), net_b(3), false, out); break;
    default: return cudaErrorInvalidValue;
    }
    return after_launch();
}

cudaError_t launch_net_backward(int layer, const float *gout, const float *in, int n, int h, int w, const float *params,
                                float *gin, float *grads, cudaStream_t s)
{
    LaunchTimer t("proposal_train_backward", s);
    const unsigned g = grid_for((size_t)h * w * n);
    switch (layer) {
    case 0: conv_bwd_weight_kernel<2, 16><<<16 * 2, 256, 0, s>>>(gout, in, n, h, w, grads, net_w(0), net_b(0)); break;
    case 1:
        conv_bwd_weight_kernel<16, 16><<<256, 256, 0, s>>>(gout, in, n, h, w, grads, net_w(1), net_b(1));
        count_launch();
        conv_bwd_data_kernel<16, 16><<<g, 256, 0, s>>>(gout, in, n, h, w, params, net_w(1), gin);
        break;
    case 2:
        conv_bwd_weight_kernel<16, 16><<<256, 256, 0, s>>>(gout, in, n, h, w, grads, net_w(2), net_b(2));
        count_launch();
        conv_bwd_data_kernel<16, 16><<<g, 256, 0, s>>>(gout, in, n, h, w, params, net_w(2), gin);
        break;
    case 3:
        conv_bwd_weight_kernel<16, 1><<<16, 256, 0, s>>>(gout, in, n, h, w, grads, net_w(3), net_b(3));
        count_launch();
        conv_bwd_data_kernel<16, 1><<<g, 256, 0, s>>>(gout, in, n, h, w, params, net_w(3), gin);
        break;
    default: return cudaErrorInvalidValue;
    }
    return after_launch();
}

cudaError_t launch_net_loss(const float *z, const float *labels, int n, int ta, int tb, float *gz, float *loss_parts, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    LaunchTimer t("proposal_train_loss", s);
    net_loss_kernel<<<n, 256, 0, s>>>(z, labels, n, ta, tb, gz, loss_parts);
    return after_launch();
}

cudaError_t launch_net_adam(float *params, float *rounded, const float *grads, float *m, float *v, int count, float lr, float b1,
                            float b2, float eps, int t, cudaStream_t s)
{
    LaunchTimer tm("proposal_train_adam", s);
    net_adam_kernel<<<(count + 255) / 256, 256, 0, s>>>(params, rounded, grads, m, v, count, lr, b1, b2, eps, t);
    return after_launch();
}

cudaError_t launch_net_pack(const float *rounded, uint32_t *frags, cudaStream_t s)
{
    LaunchTimer t("proposal_pack", s);
    net_pack_kernel<<<(kNetFrags + 255) / 256, 256, 0, s>>>(rounded, frags);
    return after_launch();
}

cudaError_t launch_propose(const ProposeBatch &b, cudaStream_t s)
{
    if (b.total_tiles <= 0) return cudaSuccess;
    LaunchTimer t("proposal_lists", s);
    propose_kernel<<<(b.total_tiles + 255) / 256, 256, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_budget(const BudgetBatch &b, cudaStream_t s)
{
    if (b.njobs <= 0) return cudaSuccess;
    LaunchTimer t("proposal_budget", s);
    budget_kernel<<<b.njobs, kBudgetBins, 0, s>>>(b);
    return after_launch();
}

cudaError_t launch_audit(const AuditBatch &b, cudaStream_t s)
{
    if (b.njobs <= 0) return cudaSuccess;
    LaunchTimer t("proposal_audit", s);
    audit_kernel<<<b.njobs, 256, 0, s>>>(b);
    return after_launch();
}

}  // namespace es
