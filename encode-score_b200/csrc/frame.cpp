// es_frame: the per-frame measures of one source against its encodes, the queue / collect pair of
// src/main.cpp:518-643 behind a C ABI.
//
// Frame f's GPU work is queued on the caller's stream (CAMBI continues on its instances' own streams) and its figures
// arrive in page-locked memory; collect(f) waits for them and adds them to the caller's accumulators while the GPU
// works on frame f + 1. Like the reference, whatever a frame's figures are read from comes in two, used by f % 2.
//
// Device state per run: the source's luma for the last 14 frames (the lasting texture needs frames f-13 .. f), each
// encode's luma for the last 7 (its texture is measured at f - 6), the running even / odd luma sums of the source
// around the centre frame (double-buffered), and the structure masks of the last 7 frames.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "es_internal.h"

using namespace es;

namespace {
constexpr int kRing = 14, kEncRing = 7, kRadius = 6, kStats = 8, kPersist = 5, kBinArrays = 6;
}

struct es_frame {
    int w = 0, h = 0, pd = 10, nenc = 0, ww = 0, wh = 0, windows = 0;
    size_t n = 0;
    size_t slot = 0;  // elements between ring slots: n rounded up to 128, so every plane starts 256-byte aligned
    DeviceBuffer<uint16_t> src_ring, src_u, src_v;
    std::vector<std::unique_ptr<DeviceBuffer<uint16_t>>> enc_ring, enc_u, enc_v;
    DeviceBuffer<uint16_t> run_e[2], run_o[2];
    DeviceBuffer<float> stats[2], persist[2];  // [nenc][windows][8 | 5]
    DeviceBuffer<uint8_t> masks;               // [kEncRing][windows]
    DeviceBuffer<unsigned long long> sums[2];  // sse [nenc][3], then color [nenc + 1][3]
    DeviceBuffer<FrameFigures> figs[2];
    DeviceBuffer<uint16_t> bins[2];            // [nenc][6][windows]
    DeviceBuffer<float> threshold;             // the frame's structure threshold (scratch)
    DeviceBuffer<double> partials;             // per-block sums of the per-frame reduction (scratch)
    PinnedBuffer<unsigned long long> h_sums[2];
    PinnedBuffer<FrameFigures> h_figs[2];
    PinnedBuffer<uint16_t> h_bins[2];
    es_cambi *src_cambi[2] = {nullptr, nullptr};
    std::vector<es_cambi *> enc_cambi[2];
    Event done[2];
    bool source_cambi[2] = {false, false};
    long queued[2] = {-1, -1};
    long next = 0, last_collected = -1;

    ~es_frame()
    {
        for (int i = 0; i < 2; i++) {
            es_cambi_destroy(src_cambi[i]);
            for (es_cambi *c : enc_cambi[i]) es_cambi_destroy(c);
        }
    }
    uint16_t *src_plane(long f) const { return src_ring.ptr + (size_t)(f % kRing) * slot; }
    uint16_t *enc_plane(int e, long f) const { return enc_ring[e]->ptr + (size_t)(f % kEncRing) * slot; }
};

namespace {

FrameViewDev view_of(const es_frame_view &v)
{
    FrameViewDev d;
    d.y = v.y;
    d.u = v.u;
    d.v = v.v;
    d.ypitch = v.ypitch;
    d.cpitch = v.cpitch;
    d.semi = v.semi;
    d.bytes = v.bytes;
    d.shift = v.shift;
    d.depth = v.depth;
    return d;
}

void check_view(const es_frame_view &v, int pd, const char *what)
{
    require(v.y != nullptr && v.u != nullptr && (v.semi || v.v != nullptr), std::string(what) + ": missing plane");
    require(v.bytes == 1 || v.bytes == 2, std::string(what) + ": samples must be 1 or 2 bytes");
    require(v.depth == 8 || v.depth == 10, std::string(what) + ": depth must be 8 or 10");
    require(v.depth <= pd, std::string(what) + ": deeper than the pipeline");
    require(v.shift >= 0 && v.shift < 16, std::string(what) + ": bad shift");
}

void queue_frame(es_frame *fr, long f, const es_frame_view *source, int sx, int sy, int source_cambi,
                 const es_frame_view *encodes, const int *ex, const int *ey, cudaStream_t s)
{
    const int at = (int)(f % 2), up = 10 - fr->pd;
    // unpack every picture of the step in one launch
    UnpackBatch ub{};
    const int blocks = unpack_blocks(fr->w, fr->h);
    int first = 0;
    for (int p = 0; p <= fr->nenc; p++) {
        UnpackJob &j = ub.job[p];
        if (p == 0) {
            j.f = view_of(*source);
            j.x0 = sx;
            j.y0 = sy;
            j.y16 = fr->src_plane(f);
            j.u16 = fr->src_u.ptr;
            j.v16 = fr->src_v.ptr;
        } else {
            j.f = view_of(encodes[p - 1]);
            j.x0 = ex ? ex[p - 1] : 0;
            j.y0 = ey ? ey[p - 1] : 0;
            j.y16 = fr->enc_plane(p - 1, f);
            j.u16 = fr->enc_u[p - 1]->ptr;
            j.v16 = fr->enc_v[p - 1]->ptr;
        }
        j.w = fr->w;
        j.h = fr->h;
        j.pd = fr->pd;
        j.first_block = first;
        first += blocks;
    }
    ub.njobs = fr->nenc + 1;
    ub.total_blocks = first;
    cuda_check(launch_unpack(ub, s), "unpacking frames");

    // CAMBI of the source (unless cached) and of each encode; each continues on its own stream
    fr->source_cambi[at] = source_cambi != 0;
    if (source_cambi) {
        const int r = es_cambi_launch(fr->src_cambi[at], (uint64_t)fr->src_plane(f), fr->w, s);
        if (r) throw Error(r, es_last_error());
    }
    for (int e = 0; e < fr->nenc; e++) {
        const int r = es_cambi_launch(fr->enc_cambi[at][e], (uint64_t)fr->enc_plane(e, f), fr->w, s);
        if (r) throw Error(r, es_last_error());
    }

    // PSNR squared errors and color sums
    cuda_check(cudaMemsetAsync(fr->sums[at].ptr, 0, fr->sums[at].bytes(), s), "clearing");
    PairSumsJob pj{};
    pj.ry = fr->src_plane(f);
    pj.ru = fr->src_u.ptr;
    pj.rv = fr->src_v.ptr;
    for (int e = 0; e < fr->nenc; e++) {
        pj.dy[e] = fr->enc_plane(e, f);
        pj.du[e] = fr->enc_u[e]->ptr;
        pj.dv[e] = fr->enc_v[e]->ptr;
    }
    pj.sse = fr->sums[at].ptr;
    pj.color = fr->sums[at].ptr + 3 * fr->nenc;
    pj.nenc = fr->nenc;
    pj.w = fr->w;
    pj.h = fr->h;
    pj.up = up;
    PairSumsBatch pb{};
    pb.job[0] = pj;
    pb.njobs = 1;
    cuda_check(launch_pair_sums(pb, s), "squared errors and colors");

    // detail window figures of frame f
    WindowJob wj{};
    wj.yr = fr->src_plane(f);
    for (int e = 0; e < fr->nenc; e++) {
        wj.yd[e] = fr->enc_plane(e, f);
        wj.stats[e] = fr->stats[at].ptr + (size_t)e * fr->windows * kStats;
    }
    wj.nenc = fr->nenc;
    wj.w = fr->w;
    wj.h = fr->h;
    wj.up = up;
    WindowBatch wb{};
    wb.job[0] = wj;
    wb.njobs = 1;
    cuda_check(launch_window_stats(wb, s), "window figures");

    // lasting texture of frame f - 6, once frames f - 12 .. f are in
    const bool texture = f >= 2 * kRadius;
    PersistJob qj{};
    const int cur = at;
    qj.e_old = fr->run_e[cur ^ 1].ptr;
    qj.o_old = fr->run_o[cur ^ 1].ptr;
    qj.e_new = fr->run_e[cur].ptr;
    qj.o_new = fr->run_o[cur].ptr;
    qj.y_m13 = f >= 13 ? fr->src_plane(f - 13) : nullptr;
    qj.y_m7 = f >= 7 ? fr->src_plane(f - 7) : nullptr;
    qj.y_c = f >= 6 ? fr->src_plane(f - 6) : nullptr;
    qj.y_f = fr->src_plane(f);
    for (int e = 0; e < fr->nenc; e++) {
        qj.yd[e] = f >= 6 ? fr->enc_plane(e, f - 6) : nullptr;
        qj.out[e] = fr->persist[at].ptr + (size_t)e * fr->windows * kPersist;
    }
    qj.nenc = fr->nenc;
    qj.w = fr->w;
    qj.h = fr->h;
    qj.up = up;
    qj.stats = texture ? 1 : 0;
    PersistBatch qb{};
    qb.job[0] = qj;
    qb.njobs = 1;
    cuda_check(launch_persist(qb, s), "lasting texture");

    // per-frame reduction on the device
    CollectJob cj{};
    for (int e = 0; e < fr->nenc; e++) {
        cj.stats[e] = wj.stats[e];
        cj.persist[e] = texture ? qj.out[e] : nullptr;
        cj.fig[e] = fr->figs[at].ptr + e;
        cj.bins[e] = fr->bins[at].ptr + (size_t)e * kBinArrays * fr->windows;
        cj.bin_n[e] = bin_counts(fr->bins[at].ptr, fr->windows, fr->nenc) + 2 * e;
    }
    cj.centre_mask = fr->masks.ptr + (size_t)((f + kEncRing - kRadius) % kEncRing) * fr->windows;
    cj.mask = fr->masks.ptr + (size_t)(f % kEncRing) * fr->windows;
    cj.nenc = fr->nenc;
    cj.windows = fr->windows;
    cj.threshold = fr->threshold.ptr;
    cj.partials = fr->partials.ptr;
    if (fr->windows > 0) {
        CollectBatch cb{};
        cb.job[0] = cj;
        cb.njobs = 1;
        cuda_check(cudaMemsetAsync(cj.bin_n[0], 0, 8 * (size_t)fr->nenc, s), "clearing");
        cuda_check(launch_collect(cb, s), "collecting figures");
    }

    cuda_check(cudaMemcpyAsync(fr->h_sums[at].ptr, fr->sums[at].ptr, fr->sums[at].bytes(), cudaMemcpyDeviceToHost, s), "reading figures");
    if (fr->windows > 0) {
        cuda_check(cudaMemcpyAsync(fr->h_figs[at].ptr, fr->figs[at].ptr, fr->figs[at].bytes(), cudaMemcpyDeviceToHost, s), "reading figures");
        cuda_check(cudaMemcpyAsync(fr->h_bins[at].ptr, fr->bins[at].ptr, fr->bins[at].bytes(), cudaMemcpyDeviceToHost, s), "reading figures");
    }
    // the frame is done when the CAMBI streams are too
    if (source_cambi) cambi_join(fr->src_cambi[at], s);
    for (int e = 0; e < fr->nenc; e++) cambi_join(fr->enc_cambi[at][e], s);
    cuda_check(cudaEventRecord(fr->done[at].e, s), "event");
    fr->queued[at] = f;
}

// the n bins the collect kernel wrote (only those that count)
void add_bins(es_histogram &hist, const uint16_t *bins, unsigned n)
{
    for (unsigned i = 0; i < n; i++) hist.bins[bins[i]]++;
    hist.n += n;
}

}  // namespace

// src/main.cpp:584-641 for one encode of a collected frame step.
es_frame_result es::collect_encode(const EncodeFigures &in, es_accum *frame_acc, es_accum *centre_acc)
{
    const size_t cn = in.n / 4;
    auto color_of = [](const unsigned long long *c, int i) { return i < 2 ? (double)c[i] : (double)c[2] * (1.0 / 1073741824.0); };
    const FrameFigures &fg = *in.fig;
    es_frame_result res{};
    res.cambi = in.banding;
    res.cambi_source = in.source_banding;
    res.psnr[0] = es_psnr(in.sse[0], in.n, in.pd);
    res.psnr[1] = es_psnr(in.sse[1], cn, in.pd);
    res.psnr[2] = es_psnr(in.sse[2], cn, in.pd);
    for (int i = 0; i < 3; i++) {
        res.color_source[i] = color_of(in.source_color, i) / (double)cn;
        res.color_encode[i] = color_of(in.encode_color, i) / (double)cn;
    }
    res.texture = in.texture;
    res.structure_windows = in.windows > 0 ? fg.n_structure : 0;
    res.lasting_windows = in.texture && in.windows > 0 ? fg.n_lasting : 0;
    if (frame_acc) {
        es_accum &acc = *frame_acc;
        acc.frames++;
        acc.cambi += in.banding;
        acc.cambi_source += in.source_banding;
        for (int i = 0; i < 3; i++) {
            acc.psnr[i] += res.psnr[i];
            acc.color_r[i] += color_of(in.source_color, i) / (double)cn;
            acc.color_d[i] += color_of(in.encode_color, i) / (double)cn;
        }
        if (in.windows > 0) {
            for (int k = 0; k < 3; k++) {
                acc.all_r[k] += fg.all_r[k];
                acc.all_d[k] += fg.all_d[k];
                acc.st_r[k] += fg.st_r[k];
                acc.st_d[k] += fg.st_d[k];
            }
            for (int k = 0; k < 2; k++) {
                acc.sh_all_r[k] += fg.all_r[k];
                acc.sh_all_x[k] += fg.sh_all_x[k];
                acc.sh_st_r[k] += fg.st_r[k];
                acc.sh_st_x[k] += fg.sh_st_x[k];
            }
            for (int k = 0; k < 3; k++) add_bins(acc.amount[k], in.bins + (size_t)k * in.windows, in.bin_n[0]);
            for (int k = 0; k < 2; k++) add_bins(acc.matching[k], in.bins + (size_t)(3 + k) * in.windows, in.bin_n[0]);
        }
    }
    if (in.texture && in.windows > 0 && centre_acc) {
        es_accum &cacc = *centre_acc;
        cacc.own += fg.own;
        cacc.mine += fg.mine;
        add_bins(cacc.lasting, in.bins + (size_t)5 * in.windows, in.bin_n[1]);
    }
    return res;
}

extern "C" {

int es_frame_create(const es_module *m, int w, int h, int pd, int n_encodes, es_frame **out)
{
    return guarded([&] {
        require(m != nullptr && out != nullptr, "es_frame_create: NULL argument");
        require(w >= 16 && h >= 16 && w % 2 == 0 && h % 2 == 0, "es_frame_create: the picture must be even and at least 16 x 16");
        require(pd == 8 || pd == 10, "es_frame_create: pipeline depth must be 8 or 10");
        require(n_encodes >= 1 && n_encodes <= kMaxEncodes, "es_frame_create: 1 to 16 encodes");
        auto fr = std::make_unique<es_frame>();
        fr->w = w;
        fr->h = h;
        fr->pd = pd;
        fr->nenc = n_encodes;
        fr->n = (size_t)w * h;
        fr->slot = (fr->n + 127) & ~(size_t)127;
        fr->ww = w / kWin;
        fr->wh = h / kWin;
        fr->windows = fr->ww * fr->wh;
        const size_t n = fr->n, cn = n / 4, win = (size_t)fr->windows;
        fr->src_ring.reset(fr->slot * kRing);
        fr->src_u.reset(cn);
        fr->src_v.reset(cn);
        for (int e = 0; e < n_encodes; e++) {
            fr->enc_ring.push_back(std::make_unique<DeviceBuffer<uint16_t>>(fr->slot * kEncRing));
            fr->enc_u.push_back(std::make_unique<DeviceBuffer<uint16_t>>(cn));
            fr->enc_v.push_back(std::make_unique<DeviceBuffer<uint16_t>>(cn));
        }
        for (int i = 0; i < 2; i++) {
            fr->run_e[i].reset(n);
            fr->run_o[i].reset(n);
            cuda_check(cudaMemset(fr->run_e[i].ptr, 0, n * 2), "clearing");
            cuda_check(cudaMemset(fr->run_o[i].ptr, 0, n * 2), "clearing");
            fr->stats[i].reset(std::max<size_t>(1, win * kStats * n_encodes));
            fr->persist[i].reset(std::max<size_t>(1, win * kPersist * n_encodes));
            fr->sums[i].reset((size_t)3 * n_encodes + 3 * (n_encodes + 1));
            fr->figs[i].reset(n_encodes);
            fr->bins[i].reset(win * kBinArrays * n_encodes + 4 * (size_t)n_encodes);  // the arrays, then 2 counts per encode
            fr->h_sums[i].reset(fr->sums[i].count);
            fr->h_figs[i].reset(n_encodes);
            fr->h_bins[i].reset(fr->bins[i].count);
            std::memset(fr->h_figs[i].ptr, 0, sizeof(FrameFigures) * n_encodes);
            for (int r = 0; r < 1 + n_encodes; r++) {
                es_cambi *c = nullptr;
                const int st = es_cambi_create(m, w, h, pd, &c);
                if (st) throw Error(st, es_last_error());
                if (r == 0) fr->src_cambi[i] = c;
                else fr->enc_cambi[i].push_back(c);
            }
        }
        fr->threshold.reset(1);
        fr->partials.reset(std::max<size_t>(1, (size_t)n_encodes * collect_blocks(fr->windows) * kCollectSums));
        fr->masks.reset(std::max<size_t>(1, win * kEncRing));
        cuda_check(cudaMemset(fr->masks.ptr, 0, fr->masks.bytes()), "clearing");
        cuda_check(cudaDeviceSynchronize(), "frame set-up");
        *out = fr.release();
    });
}

int es_frame_queue(es_frame *fr, long f, const es_frame_view *source, int sx, int sy, int source_cambi,
                   const es_frame_view *encodes, const int *ex, const int *ey, void *stream)
{
    return guarded([&] {
        require(fr != nullptr && source != nullptr && encodes != nullptr, "es_frame_queue: NULL argument");
        require(f == fr->next, "es_frame_queue: frames must be queued in order from 0");
        require(sx >= 0 && sy >= 0 && (sx % 2) == 0 && (sy % 2) == 0, "es_frame_queue: crop offsets must be even and >= 0");
        check_view(*source, fr->pd, "source");
        for (int e = 0; e < fr->nenc; e++) {
            check_view(encodes[e], fr->pd, "encode");
            if (ex) require(ex[e] >= 0 && ex[e] % 2 == 0, "es_frame_queue: crop offsets must be even and >= 0");
            if (ey) require(ey[e] >= 0 && ey[e] % 2 == 0, "es_frame_queue: crop offsets must be even and >= 0");
        }
        const int at = (int)(f % 2);
        if (fr->queued[at] > fr->last_collected)
            throw Error(ES_ERR_STATE, "es_frame_queue: frame " + std::to_string(fr->queued[at]) + " has not been collected");
        queue_frame(fr, f, source, sx, sy, source_cambi, encodes, ex, ey, (cudaStream_t)stream);
        fr->next = f + 1;
    });
}

int es_frame_collect(es_frame *fr, long f, const double *cached_source_cambi, es_accum *const *frame_acc,
                     es_accum *const *centre_acc, es_frame_result *out)
{
    return guarded([&] {
        require(fr != nullptr, "es_frame_collect: NULL frame");
        const int at = (int)(f % 2);
        if (fr->queued[at] != f) throw Error(ES_ERR_STATE, "es_frame_collect: frame " + std::to_string(f) + " was not queued");
        if (f <= fr->last_collected) throw Error(ES_ERR_STATE, "es_frame_collect: frame collected twice");
        cuda_check(cudaEventSynchronize(fr->done[at].e), "waiting for a frame");
        double source_banding = 0;
        if (fr->source_cambi[at]) {
            const int r = es_cambi_finish(fr->src_cambi[at], &source_banding);
            if (r) throw Error(r, es_last_error());
        } else {
            require(cached_source_cambi != nullptr, "es_frame_collect: the source's CAMBI was skipped and no cached value given");
            source_banding = *cached_source_cambi;
        }
        const bool texture = f >= 2 * kRadius;
        const unsigned long long *sse = fr->h_sums[at].ptr, *color = sse + 3 * fr->nenc;
        const unsigned long long *scol = color + 3 * fr->nenc;
        for (int e = 0; e < fr->nenc; e++) {
            double banding = 0;
            const int r = es_cambi_finish(fr->enc_cambi[at][e], &banding);
            if (r) throw Error(r, es_last_error());
            const es_frame_result res = collect_encode(
                EncodeFigures{banding, source_banding, sse + 3 * e, scol, color + 3 * e, fr->n, fr->pd, fr->windows,
                              &fr->h_figs[at].ptr[e], fr->h_bins[at].ptr + (size_t)e * kBinArrays * fr->windows,
                              bin_counts(fr->h_bins[at].ptr, fr->windows, fr->nenc) + 2 * e, texture},
                frame_acc ? frame_acc[e] : nullptr, centre_acc ? centre_acc[e] : nullptr);
            if (out) out[e] = res;
        }
        fr->last_collected = f;
    });
}

int es_frame_read_windows(es_frame *fr, int encode, float *stats, float *persist)
{
    return guarded([&] {
        require(fr != nullptr, "es_frame_read_windows: NULL frame");
        require(encode >= 0 && encode < fr->nenc, "es_frame_read_windows: encode out of range");
        if (fr->last_collected < 0) throw Error(ES_ERR_STATE, "es_frame_read_windows: no frame collected");
        const int at = (int)(fr->last_collected % 2);
        const size_t win = (size_t)fr->windows;
        if (stats && win)
            cuda_check(cudaMemcpy(stats, fr->stats[at].ptr + (size_t)encode * win * kStats, win * kStats * 4, cudaMemcpyDeviceToHost), "reading");
        if (persist && win) {
            require(fr->last_collected >= 2 * kRadius, "es_frame_read_windows: no lasting texture before frame 12");
            cuda_check(cudaMemcpy(persist, fr->persist[at].ptr + (size_t)encode * win * kPersist, win * kPersist * 4, cudaMemcpyDeviceToHost), "reading");
        }
    });
}

int es_frame_luma(const es_frame *fr, int p, long f, uint64_t *address)
{
    return guarded([&] {
        require(fr != nullptr && address != nullptr, "es_frame_luma: NULL argument");
        require(p >= 0 && p <= fr->nenc, "es_frame_luma: picture out of range");
        const long ring = p == 0 ? kRing : kEncRing;
        if (f < 0 || f >= fr->next || f + ring < fr->next)
            throw Error(ES_ERR_STATE, "es_frame_luma: frame " + std::to_string(f) + " is not in the ring");
        *address = (uint64_t)(p == 0 ? fr->src_plane(f) : fr->enc_plane(p - 1, f));
    });
}

int es_to_pictures(const es_picture_copy *copies, int n, void *stream)
{
    return guarded([&] {
        require(copies != nullptr && n >= 1 && n <= kPictureMaxJobs, "es_to_pictures: 1 to 64 copies");
        PictureBatch pb{};
        for (int i = 0; i < n; i++) {
            const es_picture_copy &c = copies[i];
            require(c.src != 0 && c.dst != 0, "es_to_pictures: NULL plane or picture");
            require(c.w > 0 && c.h > 0, "es_to_pictures: empty plane");
            require(c.bytes == 1 || c.bytes == 2, "es_to_pictures: samples must be 1 or 2 bytes");
            require(c.pitch >= c.w * c.bytes, "es_to_pictures: pitch is smaller than a row");
            pb.job[pb.njobs++] = PictureJob{(const uint16_t *)c.src, (void *)c.dst, c.w, c.h, c.pitch, c.bytes, 0};
        }
        cuda_check(launch_to_pictures(pb, (cudaStream_t)stream), "copying pictures");
    });
}

void es_frame_destroy(es_frame *fr)
{
    if (!fr) return;
    cudaDeviceSynchronize();
    delete fr;
}

}  // extern "C"
