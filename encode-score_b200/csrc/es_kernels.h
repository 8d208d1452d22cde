// Job descriptors and launchers shared by the host code (C++) and the kernels (CUDA).
//
// Kernels take their work as tables of jobs passed by value in the kernel parameters (up to 32 KB since CUDA 12.1),
// so that one launch covers any mix of pictures and scales: the single-picture Cambi path and the batched frame step
// use the same kernels. Each launcher returns the cudaError_t of the launch.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace es {

// Every launcher below ends with after_launch(): it counts the launch (es_launch_count) and returns its error.
void count_launch();
// Adds n (which may be negative) to the launch count: a graph replay counts its kernel nodes, a capture takes back
// the launches its recording counted.
void count_launches(long long n);
inline cudaError_t after_launch()
{
    count_launch();
    return cudaGetLastError();
}

// Brackets a launcher's kernel launch with CUDA events on its stream while kernel timing is switched on
// (es_kernel_timing); a no-op otherwise.
struct LaunchTimer {
    int slot = -1;
    cudaStream_t stream;
    LaunchTimer(const char *name, cudaStream_t s);
    ~LaunchTimer();
    LaunchTimer(const LaunchTimer &) = delete;
};
// True while es_kernel_timing(2) is in force: CAMBI instances then queue all their work on the caller's stream, so
// that nothing runs beside a timed kernel and its events bracket that kernel alone.
bool serial_streams();
// True while es_kernel_timing is on (its events need plain launches, so graphs are not used then).
bool kernel_timing_on();

constexpr int kScales = 5;
constexpr int kDiffs = 4;
constexpr uint16_t kNone = 0xFFFF;
constexpr uint16_t kMaskBit = 0x8000;  // a scale's plane holds value | mask << 15
constexpr int kMaxBand = 1024;         // codes of a 10-bit pipeline
constexpr int kMaxPad = 64;            // window 129
constexpr int kMaxPictures = 64;       // pictures in one batched launch
constexpr int kMaxJobs = kMaxPictures * 5;  // pictures x scales in one c-value launch
constexpr int kWin = 16;               // detail window side (src/kernels.cu:331)

#ifdef __CUDACC__
// The job whose range of blocks or tiles holds t: the last job j with first(j) <= t, by binary search over a job
// table whose first blocks do not decrease (a job without blocks shares its first with the next).
template <typename First>
__device__ __forceinline__ int find_job(int njobs, int t, First first)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t >= first(mid)) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
#endif

// CAMBI's band parameters (src/kernels.cu:65-69 CambiParams without the per-scale size).
struct Band {
    int band_base, band_size, vlt;
    int tvi[kDiffs];
    int weight[kDiffs];
};

// ---- scales 0 and 1: preprocessing, zero-derivative mask and mode filter of one plane, then its first decimation --
struct Prep0Job {
    const uint16_t *img;  // input plane, `pitch` pixels per row
    int pitch, w, h, depth, mask_index;
    uint16_t *word;       // out: w x h, mode-filtered value | mask << 15
    int tiles_x, first_tile;  // set by the launcher
    // optional (the tile proposal): the feature map of the words, ceil(h / 4) x ceil(w / 4) (mean, mask share) pairs
    // as the proposal's feature kernel makes it, and per 64 x 64 tile whether a pixel needs a c-value (0 or 1)
    float2 *feat;
    unsigned *need;
    // optional: scale 1 (w1 x h1 = the halved size, rounded up) made in the same pass; nullptr: scale 0 only
    uint16_t *word1;
    int w1, h1;
};
constexpr int kPrep0MaxJobs = kMaxPictures;
struct Prep0Batch {
    Prep0Job job[kPrep0MaxJobs];
    int njobs, total_tiles;  // total_tiles: set by the launcher
    Band band;               // the codes that need c-values, for the need flags
    int need_lo, need_span;  // set by the launcher: the needed values are need_lo .. need_lo + need_span when they
                             // form one range (need_span >= 0), else need_span = -1 and the band's bits decide
};
cudaError_t launch_prep0(Prep0Batch &b, cudaStream_t s);

// ---- scales 1..4: decimation and mode filter ------------------------------------------------------------------------
struct DecJob {
    const uint16_t *src;  // previous scale's words, sw x sh
    int sw, sh;
    uint16_t *dst;        // this scale's words, w x h
    int w, h;
    int first_block;      // set by the launcher: the job's first 64 x 16 output tile
};
constexpr int kDecMaxJobs = kMaxPictures;
struct DecBatch {
    DecJob job[kDecMaxJobs];
    int njobs, total_blocks;  // total_blocks: set by the launcher
};
cudaError_t launch_decimate_mode(DecBatch &b, cudaStream_t s);

// ---- c-values --------------------------------------------------------------------------------------------------------
// Per picture-scale counters in device memory. The c-values are exact multiples of 2^-24 (they are at least 0.5), so
// their sum is kept exactly as an integer in those units; the order of additions does not matter.
// The c-value kernel also counts the positive values by the top 11 bits of their floats (the first radix digit of the
// top-k selection): at least 0.5 and below 2^13, so those digits lie in kCvDigit0 .. kCvDigit0 + 55.
constexpr unsigned kCvDigit0 = 0x3F000000u >> 21, kCvDigits = 64;
struct CvSlot {
    unsigned long long sum_fx, count;  // positive c-values: sum in 2^-24 units, number
    unsigned long long list_n;         // values appended to `list`
    unsigned long long n, k;           // pixels of the scale, top-k count
    unsigned long long remaining, above_fx, above_n;
    unsigned prefix, mask;             // radix select state
    float *list;                       // positive c-values (capacity n)
    unsigned hist[2048];               // counts of the current radix digit
    unsigned long long dsum[1024];     // last round: sums (2^-24 units) of the values of each last digit
};

struct CvJob {
    const uint16_t *word;
    int w, h, pad;
    int tiles_x, first_tile;
    int slot;       // index into the CvSlot array
    float *plane;   // optional: every computed c-value at its pixel
    int run_index;  // the entry of CvBatch::run that gates this job (with a run table)
    int tile_rows;  // rows of this job's tiles: 64 (0 means 64), 32 or 16; tiles are numbered row by row
    int tile_cols;  // columns of this job's tiles: 64 (0 means 64) or 128 (tiles_x counts tiles of this width)
};
struct CvBatch {
    CvJob job[kMaxJobs];
    int njobs, total_tiles, max_pad;
    Band band;
    const float *lut;  // lut[i] = 1/i as float, i < (2 max_pad + 1)^2 + 1
    CvSlot *slots;
    // Optional tile list: the launch then has a fixed grid whose blocks take tiles[*tile_next++] (global tile ids, job
    // by job as first_tile numbers them) while the counter is below *tile_count; *tile_next must be 0 at launch.
    const unsigned *tiles;
    const unsigned *tile_count;
    unsigned *tile_next;
    // Optional: per global tile, the exact sum of its positive c-values in 2^-24 units (0 for a tile with none).
    unsigned long long *tile_mass;
    // Optional: run[job.run_index] == 0 skips the job's tiles.
    const int *run;
    int need_lo, need_span;  // set by the launcher: as Prep0Batch's
};
// Blocks of a tile-list launch.
constexpr int kCvListBlocks = 148 * 4;
constexpr int kCvTX = 64, kCvTY = 64, kCvThreads = 256, kCvBins = 32;
size_t cvalues_smem_bytes(int max_pad, int tile_cols);
// The c-value tile width of a scale when nothing else asks for one: 64 columns (128-column tiles stage less margin per
// output pixel, but two 512-thread blocks per SM measured slower than four 256-thread ones at every scale of a 4K
// picture; the autotuner may still pick them).
inline int cv_default_tile_cols(int /*scale*/) { return 64; }
cudaError_t launch_cvalues(const CvBatch &b, cudaStream_t s);

// ---- top-k pooling and score -------------------------------------------------------------------------------------
// Clears the counters of slots [0, nslots) and sets each slot's n and k.
cudaError_t launch_slots_reset(CvSlot *slots, int nslots, const unsigned long long *n, const unsigned long long *k,
                               cudaStream_t s);
// The exact k-th largest c-value, and the sum and count of the values above it, of every slot whose positive count
// exceeds k, after the c-value launches (which leave the first digit's counts in each slot): three radix rounds of 11,
// 11 and 10 bits over the slots' lists, the last one also summing what lies above the selected value.
cudaError_t launch_topk(CvSlot *slots, int nslots, cudaStream_t s);
struct ScoreJob {
    int first_slot;  // kScales consecutive slots
    int window;
    double *score;   // out
};
constexpr int kScoreMaxJobs = kMaxPictures;
struct ScoreBatch {
    ScoreJob job[kScoreMaxJobs];
    int njobs;
    const CvSlot *slots;
};
cudaError_t launch_score(const ScoreBatch &b, cudaStream_t s);

// ---- frame unpacking ---------------------------------------------------------------------------------------------
struct FrameViewDev {
    const void *y, *u, *v;
    int ypitch, cpitch, semi, bytes, shift, depth;
};
struct UnpackJob {
    FrameViewDev f;
    int x0, y0;
    uint16_t *y16, *u16, *v16;  // w x h, w/2 x h/2
    int w, h, pd;               // common picture area and pipeline depth of this picture's source
    int first_block;            // in blocks of unpack_blocks(w, h)
};
constexpr int kUnpackMaxJobs = kMaxPictures;
// Blocks of 256 threads for one picture of w x h: a thread takes 4 consecutive 2 x 2 groups of a chroma row.
inline int unpack_blocks(int w, int h) { return (int)(((size_t)((w / 2 + 3) / 4) * (h / 2) + 255) / 256); }
struct UnpackView {
    FrameViewDev f;
    int x0, y0;
};
struct UnpackBatch {
    UnpackJob job[kUnpackMaxJobs];
    int njobs, total_blocks;
    // optional: job j's frame view and crop are views[j] in device memory instead of job[j].f, x0, y0 (so a captured
    // graph can take new input addresses each step)
    const UnpackView *views;
};
cudaError_t launch_unpack(const UnpackBatch &b, cudaStream_t s);

// ---- the VMAF picture feed (src/kernels.cu:537-545) -------------------------------------------------------------
struct PictureJob {
    const uint16_t *src;  // w x h values, rows of w
    void *dst;            // rows of `pitch` bytes, `bytes` (1 or 2) per sample
    int w, h, pitch, bytes;
    int first_block;      // set by the launcher
};
constexpr int kPictureMaxJobs = kMaxPictures;
struct PictureBatch {
    PictureJob job[kPictureMaxJobs];
    int njobs;
};
cudaError_t launch_to_pictures(PictureBatch &b, cudaStream_t s);

// ---- detail window statistics ------------------------------------------------------------------------------------
constexpr int kMaxEncodes = 16;
struct WindowJob {
    const uint16_t *yr;                 // source luma (pipeline depth)
    const uint16_t *yd[kMaxEncodes];    // encode luma
    float *stats[kMaxEncodes];          // per encode: windows x 8
    int nenc, w, h, up;
    int first_block;                    // set by the launcher
};
// Per-source work of a frame step for up to kMaxSources sources in one launch.
constexpr int kMaxSources = 32;
struct WindowBatch {
    WindowJob job[kMaxSources];
    int njobs;
};
cudaError_t launch_window_stats(WindowBatch &b, cudaStream_t s);

// ---- lasting texture ------------------------------------------------------------------------------------------------
// Running sums of the source's luma over the even and odd frame offsets of the centre frame c = f - 6:
//   E(c) = sum y(c + k), k = +-2, +-4, +-6;   O(c) = sum y(c + k), k = +-1, +-3, +-5
// with E(c) = O(c-1) - y(c) + y(c+6) and O(c) = E(c-1) - y(c-7) + y(c-1); missing frames count as 0.
struct PersistJob {
    const uint16_t *e_old, *o_old;  // 10-bit scale, w x h
    uint16_t *e_new, *o_new;
    const uint16_t *y_m13, *y_m7, *y_c, *y_f;  // frames f-13, f-7, f-6 (= centre), f; nullptr = zero
    const uint16_t *yd[kMaxEncodes];           // encodes' luma at the centre frame
    float *out[kMaxEncodes];                   // per encode: windows x 5
    int nenc, w, h, up;
    int stats;  // 0: only advance the running sums
    int first_block;  // set by the launcher
};
struct PersistBatch {
    PersistJob job[kMaxSources];
    int njobs;
};
cudaError_t launch_persist(PersistBatch &b, cudaStream_t s);

// ---- PSNR squared errors and color sums --------------------------------------------------------------------------
struct PairSumsJob {
    const uint16_t *ry, *ru, *rv;  // source planes (pipeline depth)
    const uint16_t *dy[kMaxEncodes], *du[kMaxEncodes], *dv[kMaxEncodes];
    unsigned long long *sse;       // [nenc][3]
    unsigned long long *color;     // [nenc + 1][3]: sum U, sum V, strength in 2^-30 units; source last
    int nenc, w, h, up;
    int first_pic;  // set by the launcher: this job's pictures are grid rows first_pic .. first_pic + nenc
};
struct PairSumsBatch {
    PairSumsJob job[kMaxSources];
    int njobs;
};
cudaError_t launch_pair_sums(PairSumsBatch &b, cudaStream_t s);

// ---- per-frame reduction of the window figures (src/main.cpp:606-641) -------------------------------------------
struct FrameFigures {
    double all_r[3], all_d[3], st_r[3], st_d[3];
    double sh_all_x[2], sh_st_x[2];
    double own, mine;
    unsigned n_structure, n_lasting;
    float threshold;
    unsigned pad_;
};
struct CollectJob {
    const float *stats[kMaxEncodes];    // windows x 8
    const float *persist[kMaxEncodes];  // windows x 5, centre frame (nullptr: no lasting texture this frame)
    const uint8_t *centre_mask;         // structure mask of the centre frame
    uint8_t *mask;                      // out: structure mask of this frame
    FrameFigures *fig[kMaxEncodes];
    uint16_t *bins[kMaxEncodes];        // out: 6 arrays of up to `windows` bins (amount 0-2, matching 0-1, lasting),
                                        // only those that count, from the start of each array in no fixed order
    unsigned *bin_n[kMaxEncodes];       // out (cleared by the caller): [0] bins in each of the first five arrays
                                        // (the structure windows), [1] in the lasting array
    float *threshold;                   // scratch: the frame's structure threshold
    double *partials;                   // scratch: [nenc][collect_blocks(windows)][kCollectSums]
    int nenc, windows;
    int first_enc;  // set by the launcher: this job's encodes are grid rows first_enc .. first_enc + nenc - 1
};
struct CollectBatch {
    CollectJob job[kMaxSources];
    int njobs;
};
constexpr int kCollectSums = 20;  // 18 double sums and 2 counts per block
int collect_blocks(int windows);
cudaError_t launch_collect(CollectBatch &b, cudaStream_t s);
// the same in two parts: the structure threshold and mask (needs the window figures only), then the windows' bins and
// sums (needs the lasting figures too)
cudaError_t launch_collect_threshold(CollectBatch &b, cudaStream_t s);
cudaError_t launch_collect_sums(CollectBatch &b, cudaStream_t s);

// ---- temporal alignment (src/kernels.cu:502-520, src/main.cpp:336-353) -------------------------------------------
constexpr int kThumbW = 64, kThumbH = 36, kThumbPixels = kThumbW * kThumbH;
constexpr int kThumbFrames = 64;  // frames of one thumbnail launch
struct ThumbBatch {
    FrameViewDev f[kThumbFrames];
    int n, x0, y0, w, h;  // frames; the crop of every frame
    float *out;           // [frame][kThumbH][kThumbW]
};
cudaError_t launch_thumbnails(const ThumbBatch &b, cudaStream_t s);
cudaError_t launch_offset_totals(const float *ref, const float *probe, int n_probe, int lags, double *totals, cudaStream_t s);

// ---- learned tile proposal -------------------------------------------------------------------------------------
// A 4-layer network of valid 3 x 3 convolutions (2 -> 16 -> 16 -> 16 -> 1, ReLU after the first three) on 4 x 4
// block features of scale 0 predicts log1p(mean positive c-value) of each 64 x 64 scale-0 tile. Parameters are one
// float array: per layer the weights [co][ci][3][3], then the biases.
constexpr int kNetParams = 5089;
__host__ __device__ constexpr int net_w(int l) { return l == 0 ? 0 : l == 1 ? 304 : l == 2 ? 2624 : 4944; }   // weights of layer l
__host__ __device__ constexpr int net_b(int l) { return l == 0 ? 288 : l == 1 ? 2608 : l == 2 ? 4928 : 5088; }  // its biases
constexpr int kFeatTile = 24;  // feature pixels per side around one tile (16 + 2 x 4 halo)
// mma B fragments: layers 1 and 2 (16 -> 16) [layer][tap][n tile][register][lane], then layer 3 (16 -> 1, its one
// output channel in column 0 of an 8-wide n tile) [tap][register][lane], then layer 0 (2 -> 16, k = 4 tap + 2 part +
// input channel, 36 of 3 k-steps of 16 used) [k-step][n tile][register][lane]
constexpr int kNetFrags12 = 2 * 9 * 2 * 2 * 32;
constexpr int kNetFrags3 = kNetFrags12 + 9 * 2 * 32;
constexpr int kNetFrags = kNetFrags3 + 3 * 2 * 2 * 32;

struct PredJob {
    const uint16_t *word;  // scale-0 words of a picture
    int w, h, tiles_x, tiles_y, first_tile;
    float2 *feat;          // its feature map: ceil(h / 4) x ceil(w / 4) (mean, mask share) pairs
    int first_block;       // set by the features launcher
};
struct PredBatch {
    PredJob job[kMaxPictures];
    int njobs, total_tiles;
    Band band;
    const float *params;    // bfloat16-rounded parameters (as floats)
    const uint32_t *frags;  // B fragments of layers 1, 2 and 3
    unsigned *need;         // per scale-0 tile: non-zero when a pixel of it needs a c-value, then a tile counter
                            // (total_tiles + 1 words, zeroed by the launcher unless features_ready)
    int features_ready;     // the feature maps and need flags were made with scale 0 (prep0): only predict
    float *pred;            // per scale-0 tile: the prediction, -inf where no pixel needs a c-value
};
// Both kernels of a prediction: the feature maps (and need flags) of every picture, then the network per tile.
cudaError_t launch_predict(PredBatch &b, cudaStream_t s);
inline size_t feature_map_size(int w, int h) { return (size_t)((w + 3) / 4) * ((h + 3) / 4); }

// Features of n crops: crop i covers scale-0 pixels from (xy[2 i], xy[2 i + 1]) on, fw x fh feature pixels of 4 x 4.
cudaError_t launch_net_features(const uint16_t *word, int w, int h, const int *xy, int n, int fw, int fh, float *out,
                                cudaStream_t s);
// Training on crops (NCHW float): forward of layer l (input n x ci x h x w, output n x co x (h - 2) x (w - 2), ReLU
// for l < 3); backward of layer l (gradients of its weights and biases into grads and, for l > 0, the gradient of its
// input times the ReLU mask of that input into gin); the tile loss of the last layer (n x 1 x 16a x 16b against
// n x a x b labels: per-tile squared differences into loss_parts, the gradient of the last layer's output into gz);
// and Adam (master weights, their bfloat16-rounded copy, moments).
cudaError_t launch_net_forward(int layer, const float *in, int n, int h, int w, const float *params, float *out,
                               cudaStream_t s);
cudaError_t launch_net_backward(int layer, const float *gout, const float *in, int n, int h, int w, const float *params,
                                float *gin, float *grads, cudaStream_t s);
cudaError_t launch_net_loss(const float *z, const float *labels, int n, int ta, int tb, float *gz, float *loss_parts,
                            cudaStream_t s);
cudaError_t launch_net_adam(float *params, float *rounded, const float *grads, float *m, float *v, int count, float lr,
                            float b1, float b2, float eps, int t, cudaStream_t s);
// The mma B fragments of layers 1 and 2 (kNetFrags words) from the bfloat16-rounded parameters.
cudaError_t launch_net_pack(const float *rounded, uint32_t *frags, cudaStream_t s);

// The proposal of one frame step over the c-value job table: which tiles of scales 0 and 1 run now (proposed or
// audited) and which wait for the fallback; scales 2-4 always run.
constexpr uint8_t kTileSkip = 0, kTileRun = 1, kTileAudit = 2, kTileEmpty = 3;
struct ProposeJob {
    int first_tile, tiles_x, tiles_y, scale, picture;
    int pred_first, pred_tiles_x, pred_tiles_y;  // the picture's scale-0 tile predictions
};
struct ProposeBatch {
    ProposeJob job[kMaxJobs];
    int njobs, total_tiles;
    const float *pred;
    float threshold;
    const float *pic_threshold;           // per picture (budget mode), else null: threshold for all
    unsigned audit_permille[2];           // per scale 0, 1
    const unsigned long long *frame;      // device: the step's frame number (seeds the audit sample)
    unsigned *list_a, *count_a;           // tiles to run now
    unsigned *list_b, *count_b;           // tiles of the fallback
    uint8_t *kind;                        // per global tile
    unsigned *n_audit, *n_skip;           // per job (zeroed before the launch, with the counts)
};
cudaError_t launch_propose(const ProposeBatch &b, cudaStream_t s);
// Budget mode: per picture, the skip threshold T >= `threshold` of the predictions such that the predicted score
// contribution of the scale-0 tiles below T, sum of scale * expm1(pred) * pixels, stays within `budget`.
constexpr int kBudgetBins = 1024;
constexpr float kBudgetBinsPerUnit = 128.0f;  // bins cover predictions 0 .. 8
struct BudgetJob {
    int pred_first, tiles_x, tiles_y, w, h, picture;
    double scale;  // score per unit of scale-0 c-value mass: 16 / (k0 window^2)
};
struct BudgetBatch {
    BudgetJob job[kMaxPictures];
    int njobs;
    const float *pred;
    float threshold;
    double budget;
    float *pic_threshold;  // out, by picture
};
cudaError_t launch_budget(const BudgetBatch &b, cudaStream_t s);
struct AuditJob {
    int job[2];         // the picture's scale-0 and scale-1 jobs in the propose table
    int first_tile[2];  // their global tile ranges
    int tiles[2];
    double k[2];        // their top-k counts
    int window;
};
struct ProposalStats {
    float estimate;     // estimated change of the score from the skipped tiles
    int fallback;       // 1: the skipped tiles ran too
    unsigned run[2], audited[2], skipped[2];
};
struct AuditBatch {
    AuditJob job[kMaxPictures];
    int njobs;
    const unsigned long long *tile_mass;
    const uint8_t *kind;
    const unsigned *n_audit, *n_skip;
    double tolerance;
    int *run;                 // out: per picture, 1 when the fallback runs
    ProposalStats *stats;     // out: per picture
};
cudaError_t launch_audit(const AuditBatch &b, cudaStream_t s);

}  // namespace es
