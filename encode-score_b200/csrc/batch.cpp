// es_batch: the per-frame measures of several sources at once, each with its own encodes, picture size and depth.
//
// The reference scores one source per process, with one launch per kernel and picture and a host round trip per
// top-k radix round (src/main.cpp:518-643, src/cambi.cpp:88-184). Here a frame step of every source is one launch per
// stage for all pictures: unpacking, scale 0, the decimation of each scale, the c-values of every scale of every
// picture, the top-k rounds of every slot and the scores form one chain; PSNR / color, window figures, lasting texture
// and the per-frame reduction of every source form a second chain that runs beside it. Once a source's rings are full
// (frame 14 on), a step is replayed from a CUDA graph captured per ring phase, so queueing a step costs one small copy
// of the input addresses and one graph launch.
//
// Per source the device state is that of es_frame (luma rings, running texture sums, structure masks, figures); per
// picture the CAMBI state is one word plane and one positive c-value list per scale. The figures of step f are copied
// to page-locked memory indexed by f % 2, so collect(f) reads them while step f + 1 runs.
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "es_internal.h"

using namespace es;

const float *proposal_net_rounded(es_proposal_net *net, cudaStream_t s);
const uint32_t *proposal_net_frags(const es_proposal_net *net);

namespace {
constexpr int kRing = 14, kEncRing = 7, kRadius = 6, kStats = 8, kPersist = 5, kBinArrays = 6;
constexpr int kMaxBatchPictures = kMaxJobs / kScales;  // c-value jobs of one launch

struct Source {
    int w = 0, h = 0, pd = 10, nenc = 0, ww = 0, wh = 0, windows = 0;
    size_t n = 0, slot = 0;
    int picture = 0;  // index of its own picture; its encodes' pictures follow
    DeviceBuffer<uint16_t> src_ring, src_u, src_v;
    std::vector<std::unique_ptr<DeviceBuffer<uint16_t>>> enc_ring, enc_u, enc_v;
    DeviceBuffer<uint16_t> run_e[2], run_o[2];
    DeviceBuffer<float> stats[2], persist[2];
    DeviceBuffer<uint8_t> masks;
    DeviceBuffer<unsigned long long> sums[2];
    DeviceBuffer<FrameFigures> figs[2];
    DeviceBuffer<uint16_t> bins[2];
    DeviceBuffer<float> threshold;
    DeviceBuffer<double> partials;
    PinnedBuffer<unsigned long long> h_sums[2];
    PinnedBuffer<FrameFigures> h_figs[2];
    PinnedBuffer<uint16_t> h_bins[2];
    uint16_t *src_plane(long f) const { return src_ring.ptr + (size_t)(f % kRing) * slot; }
    uint16_t *enc_plane(int e, long f) const { return enc_ring[e]->ptr + (size_t)(f % kEncRing) * slot; }
};

struct Picture {
    int source = 0, encode = -1;  // encode -1: the source's own picture
    int w = 0, h = 0, depth = 10;
    int tile_rows[kScales] = {64, 64, 64, 64, 64};  // c-value tile rows per scale
    int tile_cols[kScales] = {64, 64, 64, 64, 64};  // c-value tile columns per scale
    float *cv_plane[kScales] = {};                   // optional: every computed c-value at its pixel (tests)
    es_cambi_params p{};
    int sw[kScales], sh[kScales];
    DeviceBuffer<uint16_t> words[kScales];
    DeviceBuffer<float> lists[kScales];
};
}  // namespace

struct es_batch {
    std::vector<std::unique_ptr<Source>> sources;
    std::vector<std::unique_ptr<Picture>> pictures;
    int max_pad = 0;
    DeviceBuffer<CvSlot> slots;  // pictures x kScales
    DeviceBuffer<unsigned long long> slot_n, slot_k;
    DeviceBuffer<float> lut;
    DeviceBuffer<double> scores;  // pictures x (1 + kScales): score, then pooled per scale
    PinnedBuffer<double> h_scores[2];
    DeviceBuffer<UnpackView> views;
    PinnedBuffer<UnpackView> h_views[2];
    // the CAMBI chain, the longer one, runs at the higher priority; the texture chain fills the SMs beside it
    Stream main{true}, side{false}, aux{true};  // aux: the proposal's lists beside the decimation
    Stream side2{false};                          // the structure threshold beside the lasting texture
    Event start, fork, join, done[2], fork_aux, join_aux, fork_thr, join_thr;
    bool use_graphs = true;
    struct Step {
        cudaGraphExec_t exec;
        long long kernels;  // kernel nodes of the graph, counted as launches at each replay
    };
    std::map<std::pair<int, uint32_t>, Step> graphs;  // (ring phase, skipped sources) -> step
    uint32_t skipped[2] = {0, 0};
    long queued[2] = {-1, -1};
    long next = 0, last_collected = -1;
    uint64_t graph_launches = 0;

    // learned tile proposal (off while net is null)
    es_proposal_net *net = nullptr;
    es_proposal_options popt{};
    const float *net_params = nullptr;
    const uint32_t *net_frags = nullptr;
    int total_tiles = 0, total_tiles0 = 0;   // c-value tiles of every scale / of scale 0, all pictures
    DeviceBuffer<float> pred;                // per scale-0 tile
    DeviceBuffer<unsigned> need;             // per scale-0 tile
    DeviceBuffer<float2> feat;               // feature maps, picture by picture
    std::vector<size_t> feat_at;             // each picture's map offset
    DeviceBuffer<uint8_t> kind;              // per tile
    DeviceBuffer<unsigned> lists;            // list_a, then list_b (total_tiles each)
    DeviceBuffer<unsigned> counters;         // count_a, count_b, next_a, next_b, n_audit[kMaxJobs], n_skip[kMaxJobs]
    DeviceBuffer<unsigned long long> tile_mass, frame;
    DeviceBuffer<int> run_flags;
    DeviceBuffer<float> pic_threshold;       // per picture, budget mode
    DeviceBuffer<ProposalStats> stats;
    PinnedBuffer<ProposalStats> h_stats[2];
    PinnedBuffer<unsigned long long> h_frame[2];

    ~es_batch()
    {
        for (auto &g : graphs) cudaGraphExecDestroy(g.second.exec);
    }
    int encode_picture(int s, int e) const { return sources[s]->picture + 1 + e; }
};

namespace {

Band band_of(const es_cambi_params &p)
{
    Band bd{};
    bd.band_base = p.band_base;
    bd.band_size = p.band_size;
    bd.vlt = p.vlt;
    for (int d = 0; d < kDiffs; d++) {
        bd.tvi[d] = p.tvi[d];
        bd.weight[d] = p.weight[d];
    }
    return bd;
}

void check_view(const es_frame_view &v, int pd, const char *what)
{
    require(v.y != nullptr && v.u != nullptr && (v.semi || v.v != nullptr), std::string(what) + ": missing plane");
    require(v.bytes == 1 || v.bytes == 2, std::string(what) + ": samples must be 1 or 2 bytes");
    require(v.depth == 8 || v.depth == 10, std::string(what) + ": depth must be 8 or 10");
    require(v.depth <= pd, std::string(what) + ": deeper than the pipeline");
    require(v.shift >= 0 && v.shift < 16, std::string(what) + ": bad shift");
}

void init_source(Source &S, const es_batch_source &d)
{
    S.w = d.w;
    S.h = d.h;
    S.pd = d.pd;
    S.nenc = d.n_encodes;
    S.n = (size_t)d.w * d.h;
    S.slot = (S.n + 127) & ~(size_t)127;
    S.ww = d.w / kWin;
    S.wh = d.h / kWin;
    S.windows = S.ww * S.wh;
    const size_t n = S.n, cn = n / 4, win = (size_t)S.windows;
    S.src_ring.reset(S.slot * kRing);
    S.src_u.reset(cn);
    S.src_v.reset(cn);
    for (int e = 0; e < S.nenc; e++) {
        S.enc_ring.push_back(std::make_unique<DeviceBuffer<uint16_t>>(S.slot * kEncRing));
        S.enc_u.push_back(std::make_unique<DeviceBuffer<uint16_t>>(cn));
        S.enc_v.push_back(std::make_unique<DeviceBuffer<uint16_t>>(cn));
    }
    for (int i = 0; i < 2; i++) {
        S.run_e[i].reset(n);
        S.run_o[i].reset(n);
        cuda_check(cudaMemset(S.run_e[i].ptr, 0, n * 2), "clearing");
        cuda_check(cudaMemset(S.run_o[i].ptr, 0, n * 2), "clearing");
        S.stats[i].reset(std::max<size_t>(1, win * kStats * S.nenc));
        S.persist[i].reset(std::max<size_t>(1, win * kPersist * S.nenc));
        S.sums[i].reset((size_t)3 * S.nenc + 3 * (S.nenc + 1));
        S.figs[i].reset(S.nenc);
        S.bins[i].reset(win * kBinArrays * S.nenc + 4 * (size_t)S.nenc);  // the arrays, then 2 counts per encode
        S.h_sums[i].reset(S.sums[i].count);
        S.h_figs[i].reset(S.nenc);
        S.h_bins[i].reset(S.bins[i].count);
        std::memset(S.h_figs[i].ptr, 0, sizeof(FrameFigures) * S.nenc);
    }
    S.threshold.reset(1);
    S.partials.reset(std::max<size_t>(1, (size_t)S.nenc * collect_blocks(S.windows) * kCollectSums));
    S.masks.reset(std::max<size_t>(1, win * kEncRing));
    cuda_check(cudaMemset(S.masks.ptr, 0, S.masks.bytes()), "clearing");
}

void init_cambi(es_batch &b)
{
    const int P = (int)b.pictures.size();
    std::vector<unsigned long long> n(P * kScales), k(P * kScales);
    std::vector<CvSlot> init(P * kScales);
    std::memset(init.data(), 0, sizeof(CvSlot) * init.size());
    for (int i = 0; i < P; i++) {
        Picture &pic = *b.pictures[i];
        pic.sw[0] = pic.w;
        pic.sh[0] = pic.h;
        for (int s = 1; s < kScales; s++) {
            pic.sw[s] = (pic.sw[s - 1] + 1) >> 1;
            pic.sh[s] = (pic.sh[s - 1] + 1) >> 1;
        }
        for (int s = 0; s < kScales; s++) {
            const size_t m = (size_t)pic.sw[s] * pic.sh[s];
            pic.words[s].reset(m);
            pic.lists[s].reset(m);
            n[i * kScales + s] = m;
            k[i * kScales + s] = topk_count(m, pic.p.topk);
            init[i * kScales + s].list = pic.lists[s].ptr;
        }
        b.max_pad = std::max(b.max_pad, pic.p.pad);
    }
    b.slots.reset(init.size());
    b.slot_n.reset(n.size());
    b.slot_k.reset(k.size());
    cuda_check(cudaMemcpy(b.slots.ptr, init.data(), sizeof(CvSlot) * init.size(), cudaMemcpyHostToDevice), "batch set-up");
    cuda_check(cudaMemcpy(b.slot_n.ptr, n.data(), n.size() * 8, cudaMemcpyHostToDevice), "batch set-up");
    cuda_check(cudaMemcpy(b.slot_k.ptr, k.data(), k.size() * 8, cudaMemcpyHostToDevice), "batch set-up");
    const size_t lut_n = (size_t)(2 * b.max_pad + 1) * (2 * b.max_pad + 1) + 1;
    std::vector<float> lut(lut_n);
    reciprocal_table(b.max_pad, lut.data(), lut_n);
    b.lut.reset(lut_n);
    cuda_check(cudaMemcpy(b.lut.ptr, lut.data(), lut_n * 4, cudaMemcpyHostToDevice), "batch set-up");
    b.scores.reset((size_t)P * (1 + kScales));
    for (int i = 0; i < 2; i++) {
        b.h_scores[i].reset((size_t)P * (1 + kScales));
        std::memset(b.h_scores[i].ptr, 0, sizeof(double) * P * (1 + kScales));
        b.h_views[i].reset(P);
    }
    b.views.reset(P);
}

uint16_t *luma_of(const es_batch &b, int picture, long f)
{
    const Picture &pic = *b.pictures[picture];
    const Source &S = *b.sources[pic.source];
    return pic.encode < 0 ? S.src_plane(f) : S.enc_plane(pic.encode, f);
}

// The c-values of a step with the learned proposal: predictions of every scale-0 tile, the tile lists, the proposed
// and audited tiles, the audit, then the skipped tiles of the pictures whose audit asks for the fallback. `run` lists
// the pictures whose CAMBI runs; cb is the step's c-value job table (scales 0-4 of each, in that order).
// The proposal of a step up to its tile lists: features come with scale 0, then the prediction, the optional budget
// and the lists. Needs scale 0 only, so it runs beside the decimation of scales 1-4. Returns the audit's table.
AuditBatch record_proposal_lists(es_batch &b, const std::vector<int> &run, CvBatch &cb, cudaStream_t s)
{
    const int np = (int)run.size();
    unsigned *count_a = b.counters.ptr, *count_b = count_a + 1;
    unsigned *n_audit = count_a + 4, *n_skip = n_audit + kMaxJobs;
    cuda_check(cudaMemsetAsync(b.counters.ptr, 0, b.counters.bytes(), s), "clearing proposal counters");
    PredBatch pb{};
    int t0 = 0;
    for (int r = 0; r < np; r++) {
        const Picture &pic = *b.pictures[run[r]];
        PredJob &j = pb.job[pb.njobs++];
        j.word = pic.words[0].ptr;
        j.w = pic.w;
        j.h = pic.h;
        j.tiles_x = (pic.w + kCvTX - 1) / kCvTX;
        j.tiles_y = (pic.h + kCvTY - 1) / kCvTY;
        j.first_tile = t0;
        j.feat = b.feat.ptr + b.feat_at[run[r]];
        t0 += j.tiles_x * j.tiles_y;
    }
    pb.total_tiles = t0;
    pb.need = b.need.ptr;
    pb.band = cb.band;
    pb.params = b.net_params;
    pb.frags = b.net_frags;
    pb.pred = b.pred.ptr;
    pb.features_ready = 1;  // made by the scale-0 launch
    cuda_check(launch_predict(pb, s), "tile predictions");
    const bool budget = b.popt.budget > 0;
    if (budget) {
        BudgetBatch bb{};
        for (int r = 0; r < np; r++) {
            const Picture &pic = *b.pictures[run[r]];
            BudgetJob &j = bb.job[bb.njobs++];
            j.pred_first = pb.job[r].first_tile;
            j.tiles_x = pb.job[r].tiles_x;
            j.tiles_y = pb.job[r].tiles_y;
            j.w = pic.w;
            j.h = pic.h;
            j.picture = run[r];
            const double k0 = (double)topk_count((unsigned long long)pic.sw[0] * pic.sh[0], pic.p.topk);
            j.scale = 16.0 / (k0 * (double)pic.p.window * (double)pic.p.window);
        }
        bb.pred = b.pred.ptr;
        bb.threshold = b.popt.threshold;
        bb.budget = b.popt.budget;
        bb.pic_threshold = b.pic_threshold.ptr;
        cuda_check(launch_budget(bb, s), "tile budget");
    }
    ProposeBatch qb{};
    AuditBatch ab{};
    for (int r = 0; r < np; r++) {
        const Picture &pic = *b.pictures[run[r]];
        AuditJob &aj = ab.job[ab.njobs++];
        aj.window = pic.p.window;
        for (int sc = 0; sc < kScales; sc++) {
            const int ji = r * kScales + sc;
            CvJob &cj = cb.job[ji];
            cj.run_index = r;
            ProposeJob &pj = qb.job[qb.njobs++];
            pj.first_tile = cj.first_tile;
            pj.tiles_x = cj.tiles_x;
            pj.tiles_y = (cj.h + cj.tile_rows - 1) / cj.tile_rows;
            pj.scale = sc;
            pj.picture = run[r];
            pj.pred_first = pb.job[r].first_tile;
            pj.pred_tiles_x = pb.job[r].tiles_x;
            pj.pred_tiles_y = pb.job[r].tiles_y;
            if (sc < 2) {
                aj.job[sc] = ji;
                aj.first_tile[sc] = cj.first_tile;
                aj.tiles[sc] = pj.tiles_x * pj.tiles_y;
                aj.k[sc] = (double)topk_count((unsigned long long)pic.sw[sc] * pic.sh[sc], pic.p.topk);
            }
        }
    }
    qb.total_tiles = cb.total_tiles;
    qb.pred = b.pred.ptr;
    qb.threshold = b.popt.threshold;
    qb.pic_threshold = budget ? b.pic_threshold.ptr : nullptr;
    qb.audit_permille[0] = (unsigned)b.popt.audit_permille[0];
    qb.audit_permille[1] = (unsigned)b.popt.audit_permille[1];
    qb.frame = b.frame.ptr;
    qb.list_a = b.lists.ptr;
    qb.list_b = b.lists.ptr + b.total_tiles;
    qb.count_a = count_a;
    qb.count_b = count_b;
    qb.kind = b.kind.ptr;
    qb.n_audit = n_audit;
    qb.n_skip = n_skip;
    cuda_check(launch_propose(qb, s), "tile proposal");
    return ab;
}

// The c-values of the proposed and audited tiles, the audit, and the skipped tiles of the pictures that fall back.
void record_proposal_cvalues(es_batch &b, const CvBatch &cb, AuditBatch ab, cudaStream_t s)
{
    unsigned *count_a = b.counters.ptr, *count_b = count_a + 1, *next_a = count_a + 2, *next_b = count_a + 3;
    unsigned *n_audit = count_a + 4, *n_skip = n_audit + kMaxJobs;
    CvBatch ca = cb;
    ca.tiles = b.lists.ptr;
    ca.tile_count = count_a;
    ca.tile_next = next_a;
    ca.tile_mass = b.tile_mass.ptr;
    cuda_check(launch_cvalues(ca, s), "proposed c-values");
    ab.tile_mass = b.tile_mass.ptr;
    ab.kind = b.kind.ptr;
    ab.n_audit = n_audit;
    ab.n_skip = n_skip;
    ab.tolerance = b.popt.tolerance;
    ab.run = b.run_flags.ptr;
    ab.stats = b.stats.ptr;
    cuda_check(launch_audit(ab, s), "tile audit");
    CvBatch cf = cb;
    cf.tiles = b.lists.ptr + b.total_tiles;
    cf.tile_count = count_b;
    cf.tile_next = next_b;
    cf.run = b.run_flags.ptr;
    cuda_check(launch_cvalues(cf, s), "fallback c-values");
}

// The CAMBI chain of step f for the pictures whose CAMBI runs, on stream s.
void record_cambi(es_batch &b, long f, uint32_t skip, cudaStream_t s)
{
    std::vector<int> run;
    for (int i = 0; i < (int)b.pictures.size(); i++) {
        const Picture &pic = *b.pictures[i];
        if (pic.encode >= 0 || !((skip >> pic.source) & 1u)) run.push_back(i);
    }
    if (run.empty()) return;
    const Band band = band_of(b.pictures[0]->p);
    Prep0Batch pb{};
    int pred_tiles = 0;  // with the proposal, scale 0 also makes the feature maps and the tiles' need flags
    for (int i : run) {
        const Picture &pic = *b.pictures[i];
        Prep0Job &j = pb.job[pb.njobs++];
        j.img = luma_of(b, i, f);
        j.pitch = pic.w;
        j.w = pic.w;
        j.h = pic.h;
        j.depth = pic.depth;
        j.mask_index = pic.p.mask_index;
        j.word = pic.words[0].ptr;
        j.word1 = pic.words[1].ptr;
        j.w1 = pic.sw[1];
        j.h1 = pic.sh[1];
        if (b.net) {
            j.feat = b.feat.ptr + b.feat_at[i];
            j.need = b.need.ptr + pred_tiles;
            pred_tiles += ((pic.w + kCvTX - 1) / kCvTX) * ((pic.h + kCvTY - 1) / kCvTY);
        }
    }
    pb.band = band;
    cuda_check(launch_prep0(pb, s), "batch scales 0 and 1");
    CvBatch cb{};
    int tiles = 0;
    for (int i : run) {
        const Picture &pic = *b.pictures[i];
        for (int sc = 0; sc < kScales; sc++) {
            CvJob &j = cb.job[cb.njobs++];
            j.word = pic.words[sc].ptr;
            j.w = pic.sw[sc];
            j.h = pic.sh[sc];
            j.pad = pic.p.pad;
            j.tile_cols = b.net ? kCvTX : pic.tile_cols[sc];  // the proposal maps 64-column tiles
            j.tiles_x = (j.w + j.tile_cols - 1) / j.tile_cols;
            j.first_tile = tiles;
            j.slot = i * kScales + sc;
            j.plane = pic.cv_plane[sc];
            j.tile_rows = (b.net && sc < 2) ? 64 : pic.tile_rows[sc];  // the proposal maps 64-row tiles of scales 0, 1
            tiles += j.tiles_x * ((j.h + j.tile_rows - 1) / j.tile_rows);
        }
    }
    cb.total_tiles = tiles;
    cb.max_pad = b.max_pad;
    cb.band = band;
    cb.lut = b.lut.ptr;
    cb.slots = b.slots.ptr;
    // with the proposal, its lists are made beside the decimation (they need scale 0 only)
    const bool split = !serial_streams();
    AuditBatch ab{};
    if (b.net) {
        cudaStream_t a = split ? b.aux.s : s;
        if (split) {
            cuda_check(cudaEventRecord(b.fork_aux.e, s), "event");
            cuda_check(cudaStreamWaitEvent(a, b.fork_aux.e, 0), "event");
        }
        ab = record_proposal_lists(b, run, cb, a);
        if (split) cuda_check(cudaEventRecord(b.join_aux.e, a), "event");
    }
    const int nslots = (int)b.pictures.size() * kScales;
    cuda_check(launch_slots_reset(b.slots.ptr, nslots, b.slot_n.ptr, b.slot_k.ptr, s), "batch reset");
    for (int sc = 2; sc < kScales; sc++) {
        DecBatch db{};
        int blocks = 0;
        for (int i : run) {
            const Picture &pic = *b.pictures[i];
            DecJob &dj = db.job[db.njobs++];
            dj.src = pic.words[sc - 1].ptr;
            dj.sw = pic.sw[sc - 1];
            dj.sh = pic.sh[sc - 1];
            dj.dst = pic.words[sc].ptr;
            dj.w = pic.sw[sc];
            dj.h = pic.sh[sc];
            dj.first_block = blocks;
            blocks += (dj.w * dj.h + 255) / 256;
        }
        db.total_blocks = blocks;
        cuda_check(launch_decimate_mode(db, s), "batch scales");
    }
    if (!b.net) {
        cuda_check(launch_cvalues(cb, s), "batch c-values");
    } else {
        if (split) cuda_check(cudaStreamWaitEvent(s, b.join_aux.e, 0), "event");
        record_proposal_cvalues(b, cb, ab, s);
    }
    cuda_check(launch_topk(b.slots.ptr, nslots, s), "batch top-k");
    ScoreBatch sb{};
    for (int i : run) {
        ScoreJob &j = sb.job[sb.njobs++];
        j.first_slot = i * kScales;
        j.window = b.pictures[i]->p.window;
        j.score = b.scores.ptr + (size_t)i * (1 + kScales);
    }
    sb.slots = b.slots.ptr;
    cuda_check(launch_score(sb, s), "batch score");
    cuda_check(cudaMemcpyAsync(b.h_scores[f % 2].ptr, b.scores.ptr, b.scores.bytes(), cudaMemcpyDeviceToHost, s),
               "reading scores");
    if (b.net)
        cuda_check(cudaMemcpyAsync(b.h_stats[f % 2].ptr, b.stats.ptr, b.stats.bytes(), cudaMemcpyDeviceToHost, s), "reading proposal stats");
}

// The texture chain of step f (PSNR / color, window figures, lasting texture, reduction) for every source.
void record_texture(es_batch &b, long f, cudaStream_t s, cudaStream_t s2)
{
    const int at = (int)(f % 2);
    const bool texture = f >= 2 * kRadius;
    PairSumsBatch pb{};
    WindowBatch wb{};
    PersistBatch qb{};
    CollectBatch cb{};
    for (auto &sp : b.sources) {
        Source &S = *sp;
        const int up = 10 - S.pd;
        cuda_check(cudaMemsetAsync(S.sums[at].ptr, 0, S.sums[at].bytes(), s), "clearing");
        PairSumsJob &pj = pb.job[pb.njobs++];
        pj.ry = S.src_plane(f);
        pj.ru = S.src_u.ptr;
        pj.rv = S.src_v.ptr;
        for (int e = 0; e < S.nenc; e++) {
            pj.dy[e] = S.enc_plane(e, f);
            pj.du[e] = S.enc_u[e]->ptr;
            pj.dv[e] = S.enc_v[e]->ptr;
        }
        pj.sse = S.sums[at].ptr;
        pj.color = S.sums[at].ptr + 3 * S.nenc;
        pj.nenc = S.nenc;
        pj.w = S.w;
        pj.h = S.h;
        pj.up = up;

        WindowJob &wj = wb.job[wb.njobs++];
        wj.yr = S.src_plane(f);
        for (int e = 0; e < S.nenc; e++) {
            wj.yd[e] = S.enc_plane(e, f);
            wj.stats[e] = S.stats[at].ptr + (size_t)e * S.windows * kStats;
        }
        wj.nenc = S.nenc;
        wj.w = S.w;
        wj.h = S.h;
        wj.up = up;

        PersistJob &qj = qb.job[qb.njobs++];
        qj.e_old = S.run_e[at ^ 1].ptr;
        qj.o_old = S.run_o[at ^ 1].ptr;
        qj.e_new = S.run_e[at].ptr;
        qj.o_new = S.run_o[at].ptr;
        qj.y_m13 = f >= 13 ? S.src_plane(f - 13) : nullptr;
        qj.y_m7 = f >= 7 ? S.src_plane(f - 7) : nullptr;
        qj.y_c = f >= 6 ? S.src_plane(f - 6) : nullptr;
        qj.y_f = S.src_plane(f);
        for (int e = 0; e < S.nenc; e++) {
            qj.yd[e] = f >= 6 ? S.enc_plane(e, f - 6) : nullptr;
            qj.out[e] = S.persist[at].ptr + (size_t)e * S.windows * kPersist;
        }
        qj.nenc = S.nenc;
        qj.w = S.w;
        qj.h = S.h;
        qj.up = up;
        qj.stats = texture ? 1 : 0;

        if (S.windows > 0) {
            CollectJob &cj = cb.job[cb.njobs++];
            for (int e = 0; e < S.nenc; e++) {
                cj.stats[e] = wj.stats[e];
                cj.persist[e] = texture ? qj.out[e] : nullptr;
                cj.fig[e] = S.figs[at].ptr + e;
                cj.bins[e] = S.bins[at].ptr + (size_t)e * kBinArrays * S.windows;
                cj.bin_n[e] = bin_counts(S.bins[at].ptr, S.windows, S.nenc) + 2 * e;
            }
            cj.centre_mask = S.masks.ptr + (size_t)((f + kEncRing - kRadius) % kEncRing) * S.windows;
            cj.mask = S.masks.ptr + (size_t)(f % kEncRing) * S.windows;
            cj.nenc = S.nenc;
            cj.windows = S.windows;
            cj.threshold = S.threshold.ptr;
            cj.partials = S.partials.ptr;
        }
    }
    cuda_check(launch_pair_sums(pb, s), "batch squared errors and colors");
    cuda_check(launch_window_stats(wb, s), "batch window figures");
    // the structure threshold needs only the window figures, so on a stream of its own it runs beside the lasting
    // texture (one block, otherwise alone at the end of the chain)
    const bool fork = cb.njobs && s2 != nullptr;
    if (fork) {
        cuda_check(cudaEventRecord(b.fork_thr.e, s), "event");
        cuda_check(cudaStreamWaitEvent(s2, b.fork_thr.e, 0), "event");
        cuda_check(launch_collect_threshold(cb, s2), "batch structure threshold");
        cuda_check(cudaEventRecord(b.join_thr.e, s2), "event");
    }
    cuda_check(launch_persist(qb, s), "batch lasting texture");
    if (cb.njobs) {
        if (fork) cuda_check(cudaStreamWaitEvent(s, b.join_thr.e, 0), "event");
        else cuda_check(launch_collect_threshold(cb, s), "batch structure threshold");
        for (auto &sp : b.sources)
            if (sp->windows > 0)
                cuda_check(cudaMemsetAsync(bin_counts(sp->bins[at].ptr, sp->windows, sp->nenc), 0, 8 * (size_t)sp->nenc, s), "clearing");
        cuda_check(launch_collect_sums(cb, s), "batch collecting figures");
    }
    for (auto &sp : b.sources) {
        Source &S = *sp;
        cuda_check(cudaMemcpyAsync(S.h_sums[at].ptr, S.sums[at].ptr, S.sums[at].bytes(), cudaMemcpyDeviceToHost, s), "reading figures");
        if (S.windows > 0) {
            cuda_check(cudaMemcpyAsync(S.h_figs[at].ptr, S.figs[at].ptr, S.figs[at].bytes(), cudaMemcpyDeviceToHost, s), "reading figures");
            cuda_check(cudaMemcpyAsync(S.h_bins[at].ptr, S.bins[at].ptr, S.bins[at].bytes(), cudaMemcpyDeviceToHost, s), "reading figures");
        }
    }
}

// The whole step f on b.main: unpacking, then the CAMBI chain on main beside the texture chain on side.
void record_step(es_batch &b, long f, uint32_t skip)
{
    cudaStream_t s = b.main.s;
    UnpackBatch ub{};
    ub.views = b.views.ptr;
    int first = 0;
    for (int i = 0; i < (int)b.pictures.size(); i++) {
        const Picture &pic = *b.pictures[i];
        const Source &S = *b.sources[pic.source];
        UnpackJob &j = ub.job[ub.njobs++];
        j.y16 = luma_of(b, i, f);
        j.u16 = pic.encode < 0 ? S.src_u.ptr : S.enc_u[pic.encode]->ptr;
        j.v16 = pic.encode < 0 ? S.src_v.ptr : S.enc_v[pic.encode]->ptr;
        j.w = S.w;
        j.h = S.h;
        j.pd = S.pd;
        j.first_block = first;
        first += unpack_blocks(S.w, S.h);
    }
    ub.total_blocks = first;
    cuda_check(launch_unpack(ub, s), "batch unpacking");
    const bool split = !serial_streams();
    cudaStream_t t = split ? b.side.s : s;
    if (split) {
        cuda_check(cudaEventRecord(b.fork.e, s), "event");
        cuda_check(cudaStreamWaitEvent(t, b.fork.e, 0), "event");
    }
    record_cambi(b, f, skip, s);
    record_texture(b, f, t, split ? b.side2.s : nullptr);
    if (split) {
        cuda_check(cudaEventRecord(b.join.e, t), "event");
        cuda_check(cudaStreamWaitEvent(s, b.join.e, 0), "event");
    }
}

void queue_step(es_batch &b, long f, uint32_t skip)
{
    const bool graph = b.use_graphs && f >= kRing && !kernel_timing_on();
    if (!graph) {
        record_step(b, f, skip);
        return;
    }
    const auto key = std::make_pair((int)(f % kRing), skip);
    auto it = b.graphs.find(key);
    if (it == b.graphs.end()) {
        cudaGraph_t g = nullptr;
        const unsigned long long counted = es_launch_count();
        cuda_check(cudaStreamBeginCapture(b.main.s, cudaStreamCaptureModeThreadLocal), "capturing a step");
        try {
            record_step(b, f, skip);
        } catch (...) {
            cudaStreamEndCapture(b.main.s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        count_launches(-(long long)(es_launch_count() - counted));  // recorded, not launched
        cuda_check(cudaStreamEndCapture(b.main.s, &g), "capturing a step");
        size_t n = 0;
        long long kernels = 0;
        cudaError_t e = cudaGraphGetNodes(g, nullptr, &n);
        if (e == cudaSuccess && n) {
            std::vector<cudaGraphNode_t> nodes(n);
            e = cudaGraphGetNodes(g, nodes.data(), &n);
            for (size_t i = 0; e == cudaSuccess && i < n; i++) {
                cudaGraphNodeType type;
                if (cudaGraphNodeGetType(nodes[i], &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) kernels++;
            }
        }
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        cuda_check(e, "instantiating a step graph");
        it = b.graphs.emplace(key, es_batch::Step{exec, kernels}).first;
    }
    cuda_check(cudaGraphLaunch(it->second.exec, b.main.s), "launching a step graph");
    count_launches(it->second.kernels);
    b.graph_launches++;
}

}  // namespace

extern "C" {

int es_batch_create(const es_module *m, int n_sources, const es_batch_source *sources, const es_batch_options *options,
                    es_batch **out)
{
    return guarded([&] {
        require(m != nullptr && sources != nullptr && out != nullptr, "es_batch_create: NULL argument");
        require(n_sources >= 1 && n_sources <= kMaxSources, "es_batch_create: 1 to 32 sources");
        int pictures = 0;
        for (int i = 0; i < n_sources; i++) {
            const es_batch_source &d = sources[i];
            require(d.w >= 16 && d.h >= 16 && d.w % 2 == 0 && d.h % 2 == 0,
                    "es_batch_create: every picture must be even and at least 16 x 16");
            require(d.pd == 8 || d.pd == 10, "es_batch_create: pipeline depth must be 8 or 10");
            require(d.n_encodes >= 1 && d.n_encodes <= kMaxEncodes, "es_batch_create: 1 to 16 encodes per source");
            pictures += 1 + d.n_encodes;
        }
        require(pictures <= kMaxBatchPictures, "es_batch_create: at most 64 pictures (sources and encodes) per batch");
        check_device();
        auto b = std::make_unique<es_batch>();
        if (options) b->use_graphs = options->use_graphs != 0;
        for (int i = 0; i < n_sources; i++) {
            auto S = std::make_unique<Source>();
            init_source(*S, sources[i]);
            S->picture = (int)b->pictures.size();
            const es_cambi_params p = derive_params(sources[i].w, sources[i].h);
            for (int e = -1; e < sources[i].n_encodes; e++) {
                auto pic = std::make_unique<Picture>();
                pic->source = i;
                pic->encode = e;
                pic->w = sources[i].w;
                pic->h = sources[i].h;
                pic->depth = sources[i].pd;
                pic->p = p;
                for (int sc = 0; sc < kScales; sc++) {
                    const int r = sources[i].cv_tile_rows[sc];
                    require(r == 0 || r == 16 || r == 32 || r == 64, "es_batch_create: c-value tile rows must be 0, 16, 32 or 64");
                    pic->tile_rows[sc] = r ? r : 64;
                    const int c = sources[i].cv_tile_cols[sc];
                    require(c == 0 || c == 64 || c == 128, "es_batch_create: c-value tile columns must be 0, 64 or 128");
                    pic->tile_cols[sc] = c ? c : cv_default_tile_cols(sc);
                }
                b->pictures.push_back(std::move(pic));
            }
            b->sources.push_back(std::move(S));
        }
        init_cambi(*b);
        cuda_check(cudaDeviceSynchronize(), "batch set-up");
        *out = b.release();
    });
}

int es_batch_queue(es_batch *b, long f, const es_frame_view *views, const int *crops, const int *source_cambi,
                   void *stream)
{
    return guarded([&] {
        require(b != nullptr && views != nullptr, "es_batch_queue: NULL argument");
        require(f == b->next, "es_batch_queue: frames must be queued in order from 0");
        const int at = (int)(f % 2);
        if (b->queued[at] > b->last_collected)
            throw Error(ES_ERR_STATE, "es_batch_queue: frame " + std::to_string(b->queued[at]) + " has not been collected");
        uint32_t skip = 0;
        const int P = (int)b->pictures.size();
        for (int i = 0; i < P; i++) {
            const Picture &pic = *b->pictures[i];
            check_view(views[i], b->sources[pic.source]->pd, pic.encode < 0 ? "source" : "encode");
            UnpackView &u = b->h_views[at].ptr[i];
            u.f = FrameViewDev{views[i].y, views[i].u, views[i].v, views[i].ypitch, views[i].cpitch, views[i].semi,
                               views[i].bytes, views[i].shift, views[i].depth};
            u.x0 = crops ? crops[2 * i] : 0;
            u.y0 = crops ? crops[2 * i + 1] : 0;
            require(u.x0 >= 0 && u.y0 >= 0 && u.x0 % 2 == 0 && u.y0 % 2 == 0, "es_batch_queue: crop offsets must be even and >= 0");
        }
        for (int s = 0; s < (int)b->sources.size(); s++)
            if (source_cambi && !source_cambi[s]) skip |= 1u << s;
        cudaStream_t caller = (cudaStream_t)stream;
        cuda_check(cudaEventRecord(b->start.e, caller), "event");
        cuda_check(cudaStreamWaitEvent(b->main.s, b->start.e, 0), "event");
        cuda_check(cudaMemcpyAsync(b->views.ptr, b->h_views[at].ptr, sizeof(UnpackView) * P, cudaMemcpyHostToDevice, b->main.s),
                   "input addresses");
        if (b->net) {
            b->h_frame[at].ptr[0] = (unsigned long long)f;
            cuda_check(cudaMemcpyAsync(b->frame.ptr, b->h_frame[at].ptr, 8, cudaMemcpyHostToDevice, b->main.s), "frame number");
        }
        queue_step(*b, f, skip);
        cuda_check(cudaEventRecord(b->done[at].e, b->main.s), "event");
        cuda_check(cudaStreamWaitEvent(caller, b->done[at].e, 0), "event");
        b->skipped[at] = skip;
        b->queued[at] = f;
        b->next = f + 1;
    });
}

int es_batch_collect(es_batch *b, long f, const double *cached_source_cambi, es_accum *const *frame_acc,
                     es_accum *const *centre_acc, es_frame_result *out)
{
    return guarded([&] {
        require(b != nullptr, "es_batch_collect: NULL batch");
        const int at = (int)(f % 2);
        if (b->queued[at] != f) throw Error(ES_ERR_STATE, "es_batch_collect: frame " + std::to_string(f) + " was not queued");
        if (f <= b->last_collected) throw Error(ES_ERR_STATE, "es_batch_collect: frame collected twice");
        cuda_check(cudaEventSynchronize(b->done[at].e), "waiting for a frame step");
        const bool texture = f >= 2 * kRadius;
        const double *sc = b->h_scores[at].ptr;
        int k = 0;
        for (int s = 0; s < (int)b->sources.size(); s++) {
            const Source &S = *b->sources[s];
            double source_banding;
            if ((b->skipped[at] >> s) & 1u) {
                require(cached_source_cambi != nullptr, "es_batch_collect: a source's CAMBI was skipped and no cached value given");
                source_banding = cached_source_cambi[s];
            } else {
                source_banding = sc[(size_t)S.picture * (1 + kScales)];
            }
            const unsigned long long *sse = S.h_sums[at].ptr, *color = sse + 3 * S.nenc, *scol = color + 3 * S.nenc;
            for (int e = 0; e < S.nenc; e++, k++) {
                const double banding = sc[(size_t)b->encode_picture(s, e) * (1 + kScales)];
                const es_frame_result res = collect_encode(
                    EncodeFigures{banding, source_banding, sse + 3 * e, scol, color + 3 * e, S.n, S.pd, S.windows,
                                  &S.h_figs[at].ptr[e], S.h_bins[at].ptr + (size_t)e * kBinArrays * S.windows,
                                  bin_counts(S.h_bins[at].ptr, S.windows, S.nenc) + 2 * e, texture},
                    frame_acc ? frame_acc[k] : nullptr, centre_acc ? centre_acc[k] : nullptr);
                if (out) out[k] = res;
            }
        }
        b->last_collected = f;
    });
}

int es_batch_read_windows(es_batch *b, int source, int encode, float *stats, float *persist)
{
    return guarded([&] {
        require(b != nullptr, "es_batch_read_windows: NULL batch");
        require(source >= 0 && source < (int)b->sources.size(), "es_batch_read_windows: source out of range");
        const Source &S = *b->sources[source];
        require(encode >= 0 && encode < S.nenc, "es_batch_read_windows: encode out of range");
        if (b->last_collected < 0) throw Error(ES_ERR_STATE, "es_batch_read_windows: no frame collected");
        const int at = (int)(b->last_collected % 2);
        const size_t win = (size_t)S.windows;
        if (stats && win)
            cuda_check(cudaMemcpy(stats, S.stats[at].ptr + (size_t)encode * win * kStats, win * kStats * 4, cudaMemcpyDeviceToHost), "reading");
        if (persist && win) {
            require(b->last_collected >= 2 * kRadius, "es_batch_read_windows: no lasting texture before frame 12");
            cuda_check(cudaMemcpy(persist, S.persist[at].ptr + (size_t)encode * win * kPersist, win * kPersist * 4, cudaMemcpyDeviceToHost), "reading");
        }
    });
}

int es_batch_luma(const es_batch *b, int picture, long f, uint64_t *address)
{
    return guarded([&] {
        require(b != nullptr && address != nullptr, "es_batch_luma: NULL argument");
        require(picture >= 0 && picture < (int)b->pictures.size(), "es_batch_luma: picture out of range");
        const long ring = b->pictures[picture]->encode < 0 ? kRing : kEncRing;
        if (f < 0 || f >= b->next || f + ring < b->next)
            throw Error(ES_ERR_STATE, "es_batch_luma: frame " + std::to_string(f) + " is not in the ring");
        *address = (uint64_t)luma_of(*b, picture, f);
    });
}

int es_batch_scale_pooled(es_batch *b, int picture, double pooled[5])
{
    return guarded([&] {
        require(b != nullptr && pooled != nullptr, "es_batch_scale_pooled: NULL argument");
        require(picture >= 0 && picture < (int)b->pictures.size(), "es_batch_scale_pooled: picture out of range");
        if (b->last_collected < 0) throw Error(ES_ERR_STATE, "es_batch_scale_pooled: no frame collected");
        const double *sc = b->h_scores[b->last_collected % 2].ptr + (size_t)picture * (1 + kScales);
        for (int s = 0; s < kScales; s++) pooled[s] = sc[1 + s];
    });
}

int es_batch_set_cvalue_planes(es_batch *b, int picture, float *const dev_planes[5])
{
    return guarded([&] {
        require(b != nullptr, "es_batch_set_cvalue_planes: NULL batch");
        require(picture >= 0 && picture < (int)b->pictures.size(), "es_batch_set_cvalue_planes: picture out of range");
        if (b->queued[0] > b->last_collected || b->queued[1] > b->last_collected)
            throw Error(ES_ERR_STATE, "es_batch_set_cvalue_planes: collect every queued step first");
        cuda_check(cudaStreamSynchronize(b->main.s), "es_batch_set_cvalue_planes");
        for (auto &g : b->graphs) cudaGraphExecDestroy(g.second.exec);  // captured steps hold the old addresses
        b->graphs.clear();
        Picture &pic = *b->pictures[picture];
        for (int s = 0; s < kScales; s++) pic.cv_plane[s] = dev_planes ? dev_planes[s] : nullptr;
    });
}

int es_batch_set_proposal(es_batch *b, es_proposal_net *net, const es_proposal_options *options)
{
    return guarded([&] {
        require(b != nullptr, "es_batch_set_proposal: NULL batch");
        if (b->queued[0] > b->last_collected || b->queued[1] > b->last_collected)
            throw Error(ES_ERR_STATE, "es_batch_set_proposal: collect every queued step first");
        es_proposal_options o{};
        o.threshold = 0.05f;
        o.audit_permille[0] = 50;
        o.audit_permille[1] = 200;
        o.tolerance = 0.025;
        if (options) o = *options;
        require(o.audit_permille[0] >= 0 && o.audit_permille[0] <= 1000 && o.audit_permille[1] >= 0 && o.audit_permille[1] <= 1000,
                "es_batch_set_proposal: audit rates are per mille, 0 to 1000");
        require(o.tolerance >= 0, "es_batch_set_proposal: tolerance must be >= 0");
        require(o.budget >= 0, "es_batch_set_proposal: budget must be >= 0");
        cuda_check(cudaStreamSynchronize(b->main.s), "es_batch_set_proposal");
        for (auto &g : b->graphs) cudaGraphExecDestroy(g.second.exec);  // captured steps belong to the old setting
        b->graphs.clear();
        b->net = net;
        b->popt = o;
        if (!net) return;
        b->net_params = proposal_net_rounded(net, b->main.s);
        b->net_frags = proposal_net_frags(net);
        if (!b->pred.ptr) {
            int tiles = 0, tiles0 = 0;
            for (auto &pp : b->pictures) {
                const Picture &pic = *pp;
                for (int sc = 0; sc < kScales; sc++) {
                    const int tr = sc < 2 ? 64 : pic.tile_rows[sc];
                    const int t = ((pic.sw[sc] + kCvTX - 1) / kCvTX) * ((pic.sh[sc] + tr - 1) / tr);
                    tiles += t;
                    if (sc == 0) tiles0 += t;
                }
            }
            b->total_tiles = tiles;
            b->total_tiles0 = tiles0;
            const int P = (int)b->pictures.size();
            b->pred.reset(tiles0);
            b->need.reset(tiles0 + 1);  // + predict_kernel's tile counter
            size_t fs = 0;
            b->feat_at.clear();
            for (auto &pp : b->pictures) {
                b->feat_at.push_back(fs);
                fs += feature_map_size(pp->w, pp->h);
            }
            b->feat.reset(fs);
            b->kind.reset(tiles);
            b->lists.reset(2 * (size_t)tiles);
            b->counters.reset(4 + 2 * kMaxJobs);
            b->tile_mass.reset(tiles);
            b->frame.reset(1);
            b->run_flags.reset(P);
            b->pic_threshold.reset(P);
            b->stats.reset(P);
            for (int i = 0; i < 2; i++) {
                b->h_stats[i].reset(P);
                std::memset(b->h_stats[i].ptr, 0, sizeof(ProposalStats) * P);
                b->h_frame[i].reset(1);
            }
        }
        cuda_check(cudaStreamSynchronize(b->main.s), "es_batch_set_proposal");
    });
}

int es_batch_proposal_stats(es_batch *b, int picture, es_proposal_stats *out)
{
    return guarded([&] {
        require(b != nullptr && out != nullptr, "es_batch_proposal_stats: NULL argument");
        require(picture >= 0 && picture < (int)b->pictures.size(), "es_batch_proposal_stats: picture out of range");
        require(b->net != nullptr, "es_batch_proposal_stats: the proposal is off");
        if (b->last_collected < 0) throw Error(ES_ERR_STATE, "es_batch_proposal_stats: no frame collected");
        // the stats array is in the order of the pictures whose CAMBI ran
        const int at = (int)(b->last_collected % 2);
        int r = 0;
        for (int i = 0; i < picture; i++) {
            const Picture &pic = *b->pictures[i];
            if (pic.encode >= 0 || !((b->skipped[at] >> pic.source) & 1u)) r++;
        }
        const Picture &me = *b->pictures[picture];
        if (me.encode < 0 && ((b->skipped[at] >> me.source) & 1u)) throw Error(ES_ERR_STATE, "es_batch_proposal_stats: that CAMBI was skipped");
        const ProposalStats &st = b->h_stats[at].ptr[r];
        out->estimate = st.estimate;
        out->fallback = st.fallback;
        for (int k = 0; k < 2; k++) {
            out->run[k] = st.run[k];
            out->audited[k] = st.audited[k];
            out->skipped[k] = st.skipped[k];
        }
    });
}

uint64_t es_batch_graph_launches(const es_batch *b) { return b ? b->graph_launches : 0; }

void es_batch_destroy(es_batch *b)
{
    if (!b) return;
    cudaDeviceSynchronize();
    delete b;
}

}  // extern "C"
