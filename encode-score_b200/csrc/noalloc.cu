// es_cambi_score_noalloc: the CAMBI score of one plane with no device allocation at all.
//
// Some callers must not allocate device memory when they score a picture: plugins whose host application owns the
// device memory budget, and latency-critical paths where cudaMalloc's implicit device synchronization is not
// acceptable. This entry point runs the same kernels as es_cambi_launch / es_cambi_finish, but every buffer they use
// -- the five scale planes, the per-scale lists of positive c-values, the counters and the reciprocal table -- lives
// in one file-scope device array of kScratchBytes (20 MiB), which every GPU that loads the library holds until the
// process exits. The caller passes the input plane and a device double for the output.
//
// Host code cannot use the array's name as a device address (in host code it names a host-side stand-in). A device
// symbol's address belongs to a CUDA context, and a program may call from more than one context on a device (the
// primary one, or one it made with cuCtxCreate), so every call looks the address up again with cudaGetSymbolAddress in
// the context current on the calling thread, and every call rewrites the reciprocal table in its first kernel: no
// address or table state is kept on the host. A context's first call may load the library's kernels into it, so make
// it before any stream capture. Every call shares the array: each call clears what must start at zero, and calls whose
// work overlaps on the GPU race.
#include "es_internal.h"

namespace es {
namespace {

constexpr size_t kScratchBytes = (size_t)20 << 20;
constexpr int kNoAllocMaxPad = 32;                                                  // windows up to 65
constexpr int kLutEntries = (2 * kNoAllocMaxPad + 1) * (2 * kNoAllocMaxPad + 1) + 1;  // 4226

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

struct Carve {
    size_t slots, score, lut, words[kScales], lists[kScales], end;
    int sw[kScales], sh[kScales];
};

Carve carve(int w, int h)
{
    Carve c{};
    size_t at = 0;
    c.slots = at;
    at = align256(at + kScales * sizeof(CvSlot));
    c.score = at;
    at = align256(at + (1 + kScales) * sizeof(double));
    c.lut = at;
    at = align256(at + kLutEntries * sizeof(float));
    c.sw[0] = w;
    c.sh[0] = h;
    for (int s = 1; s < kScales; s++) {
        c.sw[s] = (c.sw[s - 1] + 1) >> 1;
        c.sh[s] = (c.sh[s - 1] + 1) >> 1;
    }
    for (int s = 0; s < kScales; s++) {
        c.words[s] = at;
        at = align256(at + (size_t)c.sw[s] * c.sh[s] * sizeof(uint16_t));
    }
    for (int s = 0; s < kScales; s++) {
        c.lists[s] = at;
        at = align256(at + (size_t)c.sw[s] * c.sh[s] * sizeof(float));
    }
    c.end = at;
    return c;
}

struct SlotSetup {
    float *list[kScales];
    unsigned long long n[kScales], k[kScales];
};

constexpr int kLutBlocks = 4;

// Blocks 0 .. kScales - 1 clear the five counter slots and point them at their lists (blockIdx.x = scale); the other
// kLutBlocks blocks write the reciprocal table lut[i] = 1/i as float for i < kLutEntries (entry 0 unused), the same
// correctly rounded values as reciprocal_table().
__global__ void noalloc_setup_kernel(CvSlot *slots, float *lut, const __grid_constant__ SlotSetup st)
{
    if (blockIdx.x >= kScales) {
        for (int i = (blockIdx.x - kScales) * blockDim.x + threadIdx.x; i < kLutEntries; i += kLutBlocks * blockDim.x)
            lut[i] = i ? __double2float_rn(__ddiv_rn(1.0, (double)i)) : 0.0f;
        return;
    }
    CvSlot &S = slots[blockIdx.x];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) S.hist[i] = 0;
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) S.dsum[i] = 0;
    if (threadIdx.x == 0) {
        S.sum_fx = S.count = S.list_n = 0;
        S.n = st.n[blockIdx.x];
        S.k = st.k[blockIdx.x];
        S.remaining = S.k;
        S.above_fx = S.above_n = 0;
        S.prefix = S.mask = 0;
        S.list = st.list[blockIdx.x];
    }
}

// The array's device address in the CUDA context current on the calling thread.
unsigned char *scratch_in_current_context()
{
    void *p = nullptr;
    cuda_check(cudaGetSymbolAddress(&p, g_scratch), "finding the no-allocation scratch array");
    return (unsigned char *)p;
}

}  // namespace
}  // namespace es

using namespace es;

extern "C" int es_cambi_score_noalloc(uint64_t img, int pitch, int w, int h, int depth, double *score, void *stream)
{
    return guarded([&] {
        require(img != 0 && score != nullptr, "es_cambi_score_noalloc: NULL plane or output");
        require(w > 1 && h > 1, "es_cambi_score_noalloc: CAMBI needs a picture of at least 2 x 2 pixels");
        require(depth == 8 || depth == 10, "es_cambi_score_noalloc: CAMBI takes 8- or 10-bit planes");
        require(pitch >= w, "es_cambi_score_noalloc: pitch is smaller than the width");
        const Carve c = carve(w, h);
        if (c.end > kScratchBytes)
            throw Error(ES_ERR_INVALID, "es_cambi_score_noalloc: a " + std::to_string(w) + " x " + std::to_string(h) +
                                            " picture needs " + std::to_string(c.end) + " bytes of scratch; the fixed array holds " +
                                            std::to_string(kScratchBytes) + " (about 1920 x 1080 at most)");
        const es_cambi_params p = derive_params(w, h);
        require(p.pad <= kNoAllocMaxPad, "es_cambi_score_noalloc: window wider than 65");
        require(p.band_size > 0 && p.band_size <= kMaxBand, "es_cambi_score_noalloc: band out of range");
        unsigned char *base = scratch_in_current_context();
        cudaStream_t s = (cudaStream_t)stream;
        CvSlot *slots = (CvSlot *)(base + c.slots);
        double *rec = (double *)(base + c.score);

        SlotSetup st{};
        for (int k = 0; k < kScales; k++) {
            st.list[k] = (float *)(base + c.lists[k]);
            st.n[k] = (unsigned long long)c.sw[k] * c.sh[k];
            st.k[k] = topk_count(st.n[k], p.topk);
        }
        noalloc_setup_kernel<<<kScales + kLutBlocks, 256, 0, s>>>(slots, (float *)(base + c.lut), st);
        cuda_check(cudaGetLastError(), "clearing the counters");

        Prep0Batch pb{};
        pb.njobs = 1;
        Prep0Job &pj = pb.job[0];
        pj.img = (const uint16_t *)img;
        pj.pitch = pitch;
        pj.w = w;
        pj.h = h;
        pj.depth = depth;
        pj.mask_index = p.mask_index;
        pj.word = (uint16_t *)(base + c.words[0]);
        pj.word1 = (uint16_t *)(base + c.words[1]);
        pj.w1 = c.sw[1];
        pj.h1 = c.sh[1];
        cuda_check(launch_prep0(pb, s), "cambi scales 0 and 1");
        for (int k = 2; k < kScales; k++) {
            DecBatch db{};
            db.njobs = 1;
            db.job[0] = DecJob{(const uint16_t *)(base + c.words[k - 1]), c.sw[k - 1], c.sh[k - 1], (uint16_t *)(base + c.words[k]),
                               c.sw[k], c.sh[k], 0};
            db.total_blocks = (c.sw[k] * c.sh[k] + 255) / 256;
            cuda_check(launch_decimate_mode(db, s), "cambi scales");
        }
        CvBatch cb{};
        cb.njobs = kScales;
        int tiles = 0;
        for (int k = 0; k < kScales; k++) {
            CvJob &j = cb.job[k];
            j.word = (const uint16_t *)(base + c.words[k]);
            j.w = c.sw[k];
            j.h = c.sh[k];
            j.pad = p.pad;
            j.tile_cols = cv_default_tile_cols(k);
            j.tiles_x = (j.w + j.tile_cols - 1) / j.tile_cols;
            j.first_tile = tiles;
            j.slot = k;
            j.plane = nullptr;
            tiles += j.tiles_x * ((j.h + kCvTY - 1) / kCvTY);
        }
        cb.total_tiles = tiles;
        cb.max_pad = p.pad;
        cb.band = Band{p.band_base, p.band_size, p.vlt, {p.tvi[0], p.tvi[1], p.tvi[2], p.tvi[3]},
                       {p.weight[0], p.weight[1], p.weight[2], p.weight[3]}};
        cb.lut = (const float *)(base + c.lut);
        cb.slots = slots;
        cuda_check(launch_cvalues(cb, s), "cambi c-values");
        cuda_check(launch_topk(slots, kScales, s), "cambi top-k");
        ScoreBatch sb{};
        sb.njobs = 1;
        sb.job[0].first_slot = 0;
        sb.job[0].window = p.window;
        sb.job[0].score = rec;
        sb.slots = slots;
        cuda_check(launch_score(sb, s), "cambi score");
        cuda_check(cudaMemcpyAsync(score, rec, sizeof(double), cudaMemcpyDeviceToDevice, s), "writing the score");
    });
}
