// es_cambi: CAMBI of one plane per launch, the C-ABI form of class Cambi (src/cambi.hpp:9-21, src/cambi.cpp:31-184).
//
// launch() queues the fused scale-0 kernel on the caller's stream (it reads the caller's plane, which is then free to
// be overwritten), then the scales, c-values, device-side top-k selection and score on the instance's own stream,
// ending with one 48-byte copy of the score and per-scale pooled values to page-locked memory. finish() only waits.
#include <cstring>
#include <vector>

#include "es_internal.h"

namespace es {
const void *kernel_entry_cvalues();
}

using namespace es;

struct es_cambi {
    int w = 0, h = 0, depth = 10;
    es_cambi_params p{};
    int sw[kScales], sh[kScales];
    DeviceBuffer<uint16_t> words[kScales];
    DeviceBuffer<float> lists[kScales];
    DeviceBuffer<CvSlot> slots;
    DeviceBuffer<unsigned long long> slot_n, slot_k;
    DeviceBuffer<float> lut;
    DeviceBuffer<double> score;  // score, then pooled per scale
    PinnedBuffer<double> host;
    Stream stream{true};  // CAMBI is the longer chain of a frame step: it runs at the higher priority
    Event copied, finished;
    float *planes[kScales] = {};
    unsigned long long *tile_mass = nullptr;
    bool pending = false, done = false;
};

namespace {

void init_cambi(es_cambi *c, int w, int h, int depth, const es_cambi_params &p)
{
    require(w > 1 && h > 1, "CAMBI needs a picture of at least 2 x 2 pixels");
    require(depth == 8 || depth == 10, "CAMBI takes 8- or 10-bit planes");
    require(p.pad >= 0 && p.pad <= kMaxPad && p.window == 2 * p.pad + 1, "CAMBI window must be odd and at most 129");
    require(p.band_size > 0 && p.band_size <= kMaxBand && p.band_base >= 0 && p.band_base + p.band_size <= kMaxBand + 8,
            "CAMBI band out of range");
    require(p.topk > 0 && p.topk <= 1, "CAMBI topk must be in (0, 1]");
    c->w = w;
    c->h = h;
    c->depth = depth;
    c->p = p;
    c->sw[0] = w;
    c->sh[0] = h;
    for (int s = 1; s < kScales; s++) {
        c->sw[s] = (c->sw[s - 1] + 1) >> 1;
        c->sh[s] = (c->sh[s - 1] + 1) >> 1;
    }
    unsigned long long n[kScales], k[kScales];
    for (int s = 0; s < kScales; s++) {
        const size_t m = (size_t)c->sw[s] * c->sh[s];
        c->words[s].reset(m);
        c->lists[s].reset(m);
        n[s] = m;
        k[s] = topk_count(m, p.topk);
    }
    c->slots.reset(kScales);
    c->slot_n.reset(kScales);
    c->slot_k.reset(kScales);
    cuda_check(cudaMemcpy(c->slot_n.ptr, n, sizeof n, cudaMemcpyHostToDevice), "cambi set-up");
    cuda_check(cudaMemcpy(c->slot_k.ptr, k, sizeof k, cudaMemcpyHostToDevice), "cambi set-up");
    const size_t lut_n = (size_t)(2 * p.pad + 1) * (2 * p.pad + 1) + 1;
    std::vector<float> lut(lut_n);
    reciprocal_table(p.pad, lut.data(), lut_n);
    c->lut.reset(lut_n);
    cuda_check(cudaMemcpy(c->lut.ptr, lut.data(), lut_n * sizeof(float), cudaMemcpyHostToDevice), "cambi set-up");
    c->score.reset(1 + kScales);
    c->host.reset(1 + kScales);
    std::memset(c->host.ptr, 0, sizeof(double) * (1 + kScales));
}

void queue_cambi(es_cambi *c, uint64_t img, int pitch, cudaStream_t caller)
{
    const es_cambi_params &p = c->p;
    // scale 0 on the caller's stream: it consumes the caller's plane
    Prep0Batch pb{};
    pb.njobs = 1;
    Prep0Job &pj = pb.job[0];
    pj.img = (const uint16_t *)img;
    pj.pitch = pitch;
    pj.w = c->w;
    pj.h = c->h;
    pj.depth = c->depth;
    pj.mask_index = p.mask_index;
    pj.word = c->words[0].ptr;
    pj.word1 = c->words[1].ptr;
    pj.w1 = c->sw[1];
    pj.h1 = c->sh[1];
    cuda_check(launch_prep0(pb, caller), "cambi scales 0 and 1");
    cuda_check(cudaEventRecord(c->copied.e, caller), "cambi event");
    cudaStream_t s = serial_streams() ? caller : c->stream.s;
    cuda_check(cudaStreamWaitEvent(s, c->copied.e, 0), "cambi event");
    cuda_check(launch_slots_reset(c->slots.ptr, kScales, c->slot_n.ptr, c->slot_k.ptr, s), "cambi reset");
    for (int sc = 2; sc < kScales; sc++) {
        DecBatch db{};
        db.njobs = 1;
        DecJob &dj = db.job[0];
        dj.src = c->words[sc - 1].ptr;
        dj.sw = c->sw[sc - 1];
        dj.sh = c->sh[sc - 1];
        dj.dst = c->words[sc].ptr;
        dj.w = c->sw[sc];
        dj.h = c->sh[sc];
        dj.first_block = 0;
        db.total_blocks = (dj.w * dj.h + 255) / 256;
        cuda_check(launch_decimate_mode(db, s), "cambi scales");
    }
    CvBatch cb{};
    cb.njobs = kScales;
    int tiles = 0;
    for (int sc = 0; sc < kScales; sc++) {
        CvJob &j = cb.job[sc];
        j.word = c->words[sc].ptr;
        j.w = c->sw[sc];
        j.h = c->sh[sc];
        j.pad = p.pad;
        j.tile_cols = c->tile_mass ? kCvTX : cv_default_tile_cols(sc);  // per-tile masses are counted on 64 x 64 tiles
        j.tiles_x = (j.w + j.tile_cols - 1) / j.tile_cols;
        j.first_tile = tiles;
        j.slot = sc;
        j.plane = c->planes[sc];
        tiles += j.tiles_x * ((j.h + kCvTY - 1) / kCvTY);
    }
    cb.total_tiles = tiles;
    cb.max_pad = p.pad;
    cb.band.band_base = p.band_base;
    cb.band.band_size = p.band_size;
    cb.band.vlt = p.vlt;
    for (int d = 0; d < kDiffs; d++) {
        cb.band.tvi[d] = p.tvi[d];
        cb.band.weight[d] = p.weight[d];
    }
    cb.lut = c->lut.ptr;
    cb.slots = c->slots.ptr;
    cb.tile_mass = c->tile_mass;
    // the slots carry their list buffers
    {
        static_assert(sizeof(CvSlot) % 8 == 0, "slot layout");
    }
    cuda_check(launch_cvalues(cb, s), "cambi c-values");
    cuda_check(launch_topk(c->slots.ptr, kScales, s), "cambi top-k");
    ScoreBatch sb{};
    sb.njobs = 1;
    sb.job[0].first_slot = 0;
    sb.job[0].window = p.window;
    sb.job[0].score = c->score.ptr;
    sb.slots = c->slots.ptr;
    cuda_check(launch_score(sb, s), "cambi score");
    cuda_check(cudaMemcpyAsync(c->host.ptr, c->score.ptr, sizeof(double) * (1 + kScales), cudaMemcpyDeviceToHost, s),
               "reading the score");
    cuda_check(cudaEventRecord(c->finished.e, s), "cambi event");
}

void set_lists(es_cambi *c)
{
    // each slot's list pointer lives in device memory; write them once
    std::vector<CvSlot> init(kScales);
    std::memset(init.data(), 0, sizeof(CvSlot) * kScales);
    for (int s = 0; s < kScales; s++) init[s].list = c->lists[s].ptr;
    cuda_check(cudaMemcpy(c->slots.ptr, init.data(), sizeof(CvSlot) * kScales, cudaMemcpyHostToDevice), "cambi set-up");
}

}  // namespace

void cambi_join(es_cambi *c, cudaStream_t stream)
{
    cuda_check(cudaStreamWaitEvent(stream, c->finished.e, 0), "cambi event");
}

extern "C" {

int es_cambi_create_with(const es_module *m, int w, int h, int depth, const es_cambi_params *params, es_cambi **out)
{
    return guarded([&] {
        require(m != nullptr && params != nullptr && out != nullptr, "es_cambi_create: NULL argument");
        require(params->w == w && params->h == h, "es_cambi_create_with: parameters are for another picture size");
        auto *c = new es_cambi;
        try {
            init_cambi(c, w, h, depth, *params);
            set_lists(c);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int es_cambi_create(const es_module *m, int w, int h, int depth, es_cambi **out)
{
    return guarded([&] {
        require(w > 0 && h > 0, "es_cambi_create: picture size must be positive");
        const es_cambi_params p = derive_params(w, h);
        const int r = es_cambi_create_with(m, w, h, depth, &p, out);
        if (r != ES_OK) throw Error(r, es_last_error());
    });
}

int es_cambi_get_params(const es_cambi *c, es_cambi_params *out)
{
    return guarded([&] {
        require(c != nullptr && out != nullptr, "es_cambi_get_params: NULL argument");
        *out = c->p;
    });
}

int es_cambi_launch(es_cambi *c, uint64_t img, int pitch, void *stream)
{
    return guarded([&] {
        require(c != nullptr, "es_cambi_launch: NULL instance");
        require(img != 0, "es_cambi_launch: NULL plane");
        require(pitch >= c->w, "es_cambi_launch: pitch is smaller than the width");
        if (c->pending) throw Error(ES_ERR_STATE, "es_cambi_launch: the previous launch has not been finished");
        queue_cambi(c, img, pitch, (cudaStream_t)stream);
        c->pending = true;
    });
}

int es_cambi_finish(es_cambi *c, double *score)
{
    return guarded([&] {
        require(c != nullptr && score != nullptr, "es_cambi_finish: NULL argument");
        if (!c->pending) throw Error(ES_ERR_STATE, "es_cambi_finish: nothing was launched");
        c->pending = false;
        cuda_check(cudaEventSynchronize(c->finished.e), "cambi");
        c->done = true;
        *score = c->host.ptr[0];
    });
}

int es_cambi_scale_stats(const es_cambi *c, double pooled[5], uint64_t sums_fx[5], uint64_t counts[5])
{
    return guarded([&] {
        require(c != nullptr, "es_cambi_scale_stats: NULL instance");
        if (!c->done) throw Error(ES_ERR_STATE, "es_cambi_scale_stats: no finished launch");
        std::vector<CvSlot> s(kScales);
        cuda_check(cudaMemcpy(s.data(), c->slots.ptr, sizeof(CvSlot) * kScales, cudaMemcpyDeviceToHost), "reading CAMBI sums");
        for (int k = 0; k < kScales; k++) {
            if (pooled) pooled[k] = c->host.ptr[1 + k];
            if (sums_fx) sums_fx[k] = s[k].sum_fx;
            if (counts) counts[k] = s[k].count;
        }
    });
}

int es_cambi_read_scale(const es_cambi *c, int s, uint16_t *image, uint8_t *mask)
{
    return guarded([&] {
        require(c != nullptr, "es_cambi_read_scale: NULL instance");
        require(s >= 0 && s < kScales, "es_cambi_read_scale: scale out of range");
        if (!c->done) throw Error(ES_ERR_STATE, "es_cambi_read_scale: no finished launch");
        const size_t n = (size_t)c->sw[s] * c->sh[s];
        std::vector<uint16_t> words(n);
        cuda_check(cudaMemcpy(words.data(), c->words[s].ptr, n * 2, cudaMemcpyDeviceToHost), "reading a CAMBI scale");
        for (size_t i = 0; i < n; i++) {
            if (image) image[i] = words[i] & 0x7FFF;
            if (mask) mask[i] = (words[i] & kMaskBit) ? 1 : 0;
        }
    });
}

int es_cambi_set_cvalue_planes(es_cambi *c, float *const dev_planes[5])
{
    return guarded([&] {
        require(c != nullptr, "es_cambi_set_cvalue_planes: NULL instance");
        for (int s = 0; s < kScales; s++) c->planes[s] = dev_planes ? dev_planes[s] : nullptr;
    });
}

int es_cambi_tile_count(int w, int h, int *count)
{
    return guarded([&] {
        require(w > 0 && h > 0 && count != nullptr, "es_cambi_tile_count: bad argument");
        int n = 0;
        for (int s = 0; s < kScales; s++) {
            n += ((w + kCvTX - 1) / kCvTX) * ((h + kCvTY - 1) / kCvTY);
            w = (w + 1) >> 1;
            h = (h + 1) >> 1;
        }
        *count = n;
    });
}

int es_cambi_set_tile_mass(es_cambi *c, uint64_t *dev_mass)
{
    return guarded([&] {
        require(c != nullptr, "es_cambi_set_tile_mass: NULL instance");
        c->tile_mass = (unsigned long long *)dev_mass;
    });
}

int es_cambi_scale_words(const es_cambi *c, int s, uint64_t *address)
{
    return guarded([&] {
        require(c != nullptr && address != nullptr, "es_cambi_scale_words: NULL argument");
        require(s >= 0 && s < kScales, "es_cambi_scale_words: scale out of range");
        *address = (uint64_t)c->words[s].ptr;
    });
}

void es_cambi_destroy(es_cambi *c)
{
    if (!c) return;
    if (c->pending) cudaEventSynchronize(c->finished.e);
    delete c;
}

}  // extern "C"
