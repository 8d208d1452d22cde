/*
 * es_b200.h -- C ABI of the B200 (sm_100a) implementation of encode-score's per-frame measurement path.
 *
 * Every function returns an int status (ES_OK = 0) unless noted; es_last_error() gives the message of the calling
 * thread's last failure. Device memory is passed as plain addresses (uint64_t, a CUdeviceptr), streams as void*
 * (a CUstream / cudaStream_t). No function falls back to the CPU: without an sm_100 device they fail with
 * ES_ERR_DEVICE.
 *
 * Reference interfaces replaced (paths inside the encode-score project):
 *   es_module_*      Kernels::load / get / launch, src/gpu.hpp:15-23, src/gpu.cpp:6-19
 *   es_cambi_*       class Cambi, src/cambi.hpp:9-21, src/cambi.cpp:31-184
 *   es_frame_*       the per-frame queue / collect of src/main.cpp:518-643 (which launches frame_planes,
 *                    window_stats, persist_stats, plane_sse and color_sums by name, src/main.cpp:229-234)
 *   es_accum_*, es_histogram_*   struct Histogram / Accum / score, src/stats.hpp:10-83
 *   es_thumbnails, es_offset_totals, es_find_offset   the offset search between a source and its encodes:
 *                    tiny_luma (src/kernels.cu:502-520), thumbnails() and find_offset() (src/main.cpp:301-353)
 */
#ifndef ES_B200_H
#define ES_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ES_OK 0
#define ES_ERR_INVALID 1 /* an argument is out of range */
#define ES_ERR_CUDA 2    /* a CUDA call failed */
#define ES_ERR_ALLOC 3   /* device or pinned memory could not be allocated */
#define ES_ERR_STATE 4   /* a call out of order, such as finish() without launch() */
#define ES_ERR_DEVICE 5  /* no sm_100 device, or the kernels do not load on it */
#define ES_ERR_NO_MATCH 6 /* es_find_offset: the probe matches the reference at no lag */

/* The message of the calling thread's last failure ("" if none). The pointer stays valid until the thread's next
 * call into this library. */
const char *es_last_error(void);
/* Library version as MAJOR * 10000 + MINOR * 100 + PATCH. */
int es_version(void);
/* Diagnostics with no counterpart in the reference: the number of kernels this library has launched in this process
 * (all threads), so a caller can check how many GPU launches a piece of work took. */
uint64_t es_launch_count(void);
/* Diagnostics with no counterpart in the reference: with on != 0, each later kernel launch of the library is
 * bracketed by CUDA events on the stream it is launched on (and earlier totals are cleared); 0 stops it. With on == 2
 * the CAMBI work of es_cambi_launch and es_frame_queue also stays on the caller's stream instead of each instance's
 * own, so kernels run one at a time and each event pair times one kernel alone. */
int es_kernel_timing(int on);
/* Waits for the device, then writes per kernel (up to `max` kernels): its name in names[32 i .. 32 i + 31]
 * (NUL-terminated), the summed event time in total_ms[i] and the number of timed launches in launches[i];
 * *count receives the number of kernels timed so far. Any output pointer but count may be NULL. */
int es_kernel_times(char *names, double *total_ms, uint64_t *launches, int max, int *count);

/* ---------------------------------------------------------------------------------------------------------------
 * Kernel module. Replaces Kernels (src/gpu.hpp:15-23): load() checks the current device and the kernels' image,
 * get(name) returns a CUfunction of one of this library's kernels, launch() runs a 2-D kernel in 32 x 8 blocks.
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct es_module es_module;
/* Kernels::load (src/gpu.cpp:6): binds to the current CUDA context's device; fails unless it is sm_100. */
int es_module_load(es_module **out);
void es_module_unload(es_module *m);
/* Kernels::get (src/gpu.cpp:8-13): the CUfunction of a kernel by name, written to *function. */
int es_module_get(const es_module *m, const char *name, void **function);
/* Kernels::launch (src/gpu.cpp:15-19): grid ceil(w/32) x ceil(h/8) of 32 x 8 threads. */
int es_module_launch(void *function, unsigned w, unsigned h, void **args, void *stream);

/* ---------------------------------------------------------------------------------------------------------------
 * CAMBI of one luma plane. Replaces class Cambi (src/cambi.hpp:9-21): create = Cambi(k, w, h, depth), launch =
 * Cambi::launch, finish = Cambi::finish. launch() reads the plane on the caller's stream (after the work already
 * queued there), then continues on the instance's own stream, so the caller may overwrite the plane with work it
 * queues on its stream afterwards; each launch() must be followed by its finish() before the next launch().
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct es_cambi es_cambi;

/* The parameters src/cambi.cpp:39-53 derives from the picture size; tvi[] in cambi.c's "+4" adjusted space. */
typedef struct {
    int w, h;       /* picture size */
    int window;     /* odd window side (cambi.c adjust_window_size) */
    int pad;        /* window >> 1 */
    int mask_index; /* more than this many flat pixels in the 7x7 square put a pixel in the mask */
    int band_base, band_size, vlt;
    int tvi[4];
    int weight[4];
    double topk; /* share of each scale's pixels pooled (0.6) */
} es_cambi_params;

/* Cambi::Cambi (src/cambi.cpp:31-77): `depth` is the bit depth of the planes launch() will get, 8 or 10. */
int es_cambi_create(const es_module *m, int w, int h, int depth, es_cambi **out);
/* As es_cambi_create with the derived parameters replaced by *params (w and h must match); window up to 129. */
int es_cambi_create_with(const es_module *m, int w, int h, int depth, const es_cambi_params *params, es_cambi **out);
/* The parameters src/cambi.cpp:39-53 would derive for a w x h picture. */
int es_cambi_derive_params(int w, int h, es_cambi_params *out);
int es_cambi_get_params(const es_cambi *c, es_cambi_params *out);
/* Cambi::launch (src/cambi.cpp:88-135): `img` is a device plane of w x h values at `depth` bits, `pitch` in
 * pixels. */
int es_cambi_launch(es_cambi *c, uint64_t img, int pitch, void *stream);
/* Cambi::finish (src/cambi.cpp:172-184): waits and gives the score, capped at 1000. */
int es_cambi_finish(es_cambi *c, double *score);
void es_cambi_destroy(es_cambi *c);

/* Introspection for tests and tools (no counterpart in the reference, whose buffers are private). After a finish():
 * per scale, the pooled value, the exact sum of the positive c-values in units of 2^-24 and their count. */
int es_cambi_scale_stats(const es_cambi *c, double pooled[5], uint64_t sums_fx[5], uint64_t counts[5]);
/* After a finish(): copies scale s's picture (mode-filtered values, u16) and mask (u8) to host memory. */
int es_cambi_read_scale(const es_cambi *c, int s, uint16_t *image, uint8_t *mask);
/* With dev_planes[s] device buffers of scale s's size (float, zeroed by the caller), later launches also write every
 * computed c-value there (the buffer kernels.cu's cambi_cvalues fills). NULL entries switch it off per scale. */
int es_cambi_set_cvalue_planes(es_cambi *c, float *const dev_planes[5]);

/* Introspection with no counterpart in the reference: the number of 64 x 64 c-value tiles of all five scales of a
 * w x h picture (scale 0's first, row by row, then scale 1's, ...). */
int es_cambi_tile_count(int w, int h, int *count);
/* With dev_mass a device array of es_cambi_tile_count entries, later launches write each tile's exact sum of positive
 * c-values there, in units of 2^-24 (the labels of the tile-proposal network); NULL switches it off. */
int es_cambi_set_tile_mass(es_cambi *c, uint64_t *dev_mass);
/* The device address of scale s's words (value | mask << 15, sw x sh): valid until the instance's next launch. */
int es_cambi_scale_words(const es_cambi *c, int s, uint64_t *address);

/* No counterpart in the reference. The CAMBI score of one plane, like es_cambi_create + es_cambi_launch +
 * es_cambi_finish, for callers that must not allocate device memory when they score a picture: plugins whose host
 * application owns the device memory budget, and latency-critical paths where cudaMalloc's implicit device
 * synchronization is not acceptable. It allocates nothing: its scratch is one fixed 20 MiB device array inside the
 * library, which every GPU that loads the library holds until the process exits, so it takes pictures up to about
 * 1920 x 1080 (larger ones fail with ES_ERR_INVALID and the size they would need). `img` is a device plane of w x h
 * values at `depth` bits (8 or 10), `pitch` in pixels; the score is written to the device double `score`; all work is
 * queued on `stream` and the call returns without waiting. It runs in the CUDA context current on the calling thread
 * (the primary context, or one made with cuCtxCreate): each call looks the array's address up in that context and
 * rewrites its reciprocal table, so nothing is cached across contexts or device resets. A context's first call may
 * load the library's kernels into it, so it should come before any stream capture. Every call shares the array: calls
 * whose work overlaps on the GPU race, so serialize them (one stream, or events). */
int es_cambi_score_noalloc(uint64_t img, int pitch, int w, int h, int depth, double *score, void *stream);

/* ---------------------------------------------------------------------------------------------------------------
 * A decoded frame as the kernels read it: src/main.cpp:99-102 FrameView / src/kernels.cu:284-287 Frame. Planar or
 * semi-planar 4:2:0 (chroma interleaved in u when semi), `bytes` per sample (1 or 2), sample value >> shift (6 for
 * P010) with `depth` bits (8 or 10). Pitches in bytes. Device addresses.
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct {
    const void *y, *u, *v;
    int ypitch, cpitch, semi, bytes, shift, depth;
} es_frame_view;

/* ---------------------------------------------------------------------------------------------------------------
 * Histogram / Accum / score: src/stats.hpp:10-83, identical layout and arithmetic.
 * --------------------------------------------------------------------------------------------------------------- */
#define ES_HIST_BINS 20001
typedef struct {
    uint64_t bins[ES_HIST_BINS];
    uint64_t n;
} es_histogram;

typedef struct {
    uint64_t frames;
    double vmaf, vmaf_min, psnr[3], cambi, cambi_source;
    double color_r[3], color_d[3];
    double all_r[3], all_d[3], st_r[3], st_d[3];
    es_histogram amount[3];
    double sh_all_r[2], sh_all_x[2], sh_st_r[2], sh_st_x[2];
    es_histogram matching[2];
    double own, mine;
    es_histogram lasting;
} es_accum;

typedef struct { double fidelity, texture, banding, grain; } es_weights;          /* src/stats.hpp:34 */
typedef struct { double fidelity, texture, banding, grain, score; } es_parts;     /* src/stats.hpp:69 */

void es_histogram_add(es_histogram *hist, double pct);                  /* src/stats.hpp:14-19 */
double es_histogram_quantile(const es_histogram *hist, double q);       /* src/stats.hpp:20-30 */
void es_accum_init(es_accum *a);                                        /* Accum{} (vmaf_min = 1e9) */
void es_accum_merge(es_accum *a, const es_accum *o);                    /* src/stats.hpp:50-64 */
/* src/stats.hpp:70-82; weights NULL = {0.30, 0.30, 0.25, 0.15}. */
void es_accum_score(const es_accum *a, const es_weights *weights, es_parts *out);
/* The segment's JSON object as src/main.cpp:738-757 writes it; returns the length it needs (excluding the NUL),
 * writing at most `size` bytes. */
size_t es_accum_json(const es_accum *a, char *buf, size_t size);

/* The per_frame object of src/main.cpp:767-774 for n frames ({"vmaf": [...], "cambi": [...], "cambi_source": [...],
 * "psnr_y": [...]}, same digits); vmaf NULL writes "vmaf": null (VMAF is outside this library). Returns the length it
 * needs (excluding the NUL), writing at most `size` bytes. */
size_t es_per_frame_json(const double *vmaf, const double *cambi, const double *cambi_source, const double *psnr_y, long n,
                         char *buf, size_t size);

/* ---------------------------------------------------------------------------------------------------------------
 * Source-CAMBI cache: class CambiCache (src/cache.hpp:9-29, src/cache.cpp:13-88), same key and file format. The
 * source's CAMBI per frame, kept on disk so a later run against the same source skips it (es_frame_queue /
 * es_batch_queue with the source's CAMBI off and the cached value given to collect). Host only.
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct es_cambi_cache es_cambi_cache;
/* CambiCache(path, x0, y0, w, h, depth): `path` is the source file (its size and first and last MiB key the cache);
 * dir NULL = $XDG_CACHE_HOME/encode-score or $HOME/.cache/encode-score. A cache that cannot be opened works as an empty
 * one that stores nothing. */
int es_cambi_cache_open(const char *path, int x0, int y0, int w, int h, int depth, const char *dir, es_cambi_cache **out);
/* CambiCache::find: 1 and *score when frame `pts` is cached, else 0 (INT64_MIN, a frame without a timestamp, is never
 * cached). */
int es_cambi_cache_find(const es_cambi_cache *c, int64_t pts, double *score);
/* CambiCache::add: kept in memory, written every 240 scores and on close. */
int es_cambi_cache_add(es_cambi_cache *c, int64_t pts, double score);
/* CambiCache::file: the cache file's path ("" when there is none). */
const char *es_cambi_cache_file(const es_cambi_cache *c);
void es_cambi_cache_close(es_cambi_cache *c);

/* PSNR as src/main.cpp:272-277: 10 log10(peak^2 / mse) capped at 6 depth + 12. */
double es_psnr(uint64_t sse, uint64_t n, int depth);

/* ---------------------------------------------------------------------------------------------------------------
 * Per-frame measures of one source against n encodes: src/main.cpp:518-643. es_frame_queue queues frame f's GPU
 * work on `stream` (double-buffered by f % 2 like the reference), es_frame_collect(f) waits for it and adds the
 * figures into the caller's accumulators.
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct es_frame es_frame;

typedef struct {
    double cambi, cambi_source; /* this frame */
    double psnr[3];             /* Y, Cb, Cr */
    double color_source[3], color_encode[3]; /* mean Cb, Cr and color strength on a 10-bit scale */
    int texture;                /* 1 when the lasting texture of frame f - 6 was added */
    uint32_t structure_windows; /* windows in the structure mask of frame f */
    uint32_t lasting_windows;   /* lasting-texture windows of frame f - 6 (when texture) */
} es_frame_result;

/* `w` x `h` is the common picture area (even), `pd` the pipeline depth (8 or 10, src/main.cpp:377-382). */
int es_frame_create(const es_module *m, int w, int h, int pd, int n_encodes, es_frame **out);
/* Frame f (0, 1, 2, ... in order). source / encodes[i] are device frames cropped at (sx, sy) / (ex[i], ey[i]);
 * source_cambi = 0 skips the source's CAMBI (src/main.cpp:522-523, a cached value given to collect instead). */
int es_frame_queue(es_frame *fr, long f, const es_frame_view *source, int sx, int sy, int source_cambi,
                   const es_frame_view *encodes, const int *ex, const int *ey, void *stream);
/* Waits for frame f and adds its figures: frame_acc[i] receives encode i's figures of frame f, centre_acc[i] the
 * lasting texture of frame f - 6 (src/main.cpp:630-641; may equal frame_acc[i] or be NULL when f < 12). With
 * source_cambi = 0 at queue time, *cached_source_cambi is used (else ignored; may be NULL). out[i] may be NULL. */
int es_frame_collect(es_frame *fr, long f, const double *cached_source_cambi, es_accum *const *frame_acc,
                     es_accum *const *centre_acc, es_frame_result *out);
/* Introspection for tests: after collect(f), encode i's window figures of frame f (windows x 8 floats, the layout of
 * src/kernels.cu:340-341) and, when f >= 12, the lasting-texture figures of frame f - 6 (windows x 5 floats,
 * src/kernels.cu:434); either pointer may be NULL. */
int es_frame_read_windows(es_frame *fr, int encode, float *stats, float *persist);
void es_frame_destroy(es_frame *fr);
/* The device address of picture p's unpacked luma plane of frame f (p = 0: the source, 1 + e: encode e; w x h 16-bit
 * values at the pipeline depth, rows of w), as es_frame_queue left it: valid from that queue call until frame f + 14
 * (the source) or f + 7 (an encode) is queued. It is the plane src/main.cpp:506-512 hands to libvmaf (see
 * es_to_pictures). */
int es_frame_luma(const es_frame *fr, int p, long f, uint64_t *address);

/* ---------------------------------------------------------------------------------------------------------------
 * The VMAF picture feed: to_picture (src/kernels.cu:537-545) as src/main.cpp:506-512 uses it, copying each unpacked
 * luma plane into libvmaf's preallocated CUDA picture (data[0], stride[0]). libvmaf itself is not part of this
 * library; a caller that links it passes the picture's device address and row pitch.
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct {
    uint64_t src;   /* device plane: w x h 16-bit values, rows of w */
    uint64_t dst;   /* device picture: rows of `pitch` bytes */
    int w, h;
    int pitch;      /* bytes per picture row, at least w * bytes */
    int bytes;      /* 1 (an 8-bit pipeline: the low byte of each value, as the reference) or 2 */
} es_picture_copy;
/* Copies n planes (1 to 64) in one launch queued on `stream`. */
int es_to_pictures(const es_picture_copy *copies, int n, void *stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Texture window energies on larger windows, in three arithmetics (the precision study; no counterpart in the
 * reference, which sums FP32 box means over fixed 16 x 16 windows, src/kernels.cu:331-428). The 3 x 3 and 9 x 9 box
 * sums (edge pixels repeated) come from summed-area tables of each luma plane kept as int64, as FP32 with two-sum
 * compensation, and as plain FP32; pixel terms and their per-16 x 16-block sums follow in the same arithmetic (exact
 * int64 numerators; Neumaier-compensated FP32; plain FP32). A window of side 16 k sums k x k blocks and gives the
 * 8 figures of src/kernels.cu:340-341 (windows x 8 doubles, window (x, y) at index y * (w / window) + x).
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct es_windows es_windows;
int es_windows_create(int w, int h, es_windows **out);
/* src / enc: device luma planes (w x h uint16 at the pipeline depth); up = 10 - depth (0 or 2). */
int es_windows_compute(es_windows *p, uint64_t src, uint64_t enc, int up, void *stream);
/* mode 0: integer tables (exact, rounded once to double); 1: compensated FP32; 2: plain FP32. out: device doubles. */
int es_windows_figures(es_windows *p, int window, int mode, double *out, void *stream);
void es_windows_destroy(es_windows *p);

/* ---------------------------------------------------------------------------------------------------------------
 * Learned tile proposal: no counterpart in the reference, which computes the c-values of every tile. A network of
 * four valid 3 x 3 convolutions (2 -> 16 -> 16 -> 16 -> 1, ReLU after the first three, bfloat16 weights, FP32
 * accumulation) reads 4 x 4 block features of CAMBI's scale-0 words -- the mean value as (mean - 512) / 256 and the
 * share of masked pixels -- and predicts log1p(mean positive c-value) of each 64 x 64 scale-0 tile. Parameters are
 * ES_PROPOSAL_PARAMS floats: per layer the weights [co][ci][3][3], then the biases.
 * --------------------------------------------------------------------------------------------------------------- */
#define ES_PROPOSAL_PARAMS 5089
typedef struct es_proposal_net es_proposal_net;
/* params: ES_PROPOSAL_PARAMS host floats, or NULL for He-initialised weights drawn with `seed`. */
int es_proposal_net_create(const float *params, uint64_t seed, es_proposal_net **out);
/* Copies the FP32 master parameters to params (host, ES_PROPOSAL_PARAMS floats). */
int es_proposal_net_get(const es_proposal_net *net, float *params);
/* One training step on n crops: x (device, n x 2 x h x w floats of features, h and w = 8 + 16 k), labels (device,
 * n x (h - 8) / 16 x (w - 8) / 16 floats). Computes the loss (mean squared error of the tile means, written to *loss
 * when not NULL) and the gradients (copied to the host array grads when not NULL), then takes an Adam step
 * (b1 0.9, b2 0.999, eps 1e-8) when lr > 0. Waits for the stream when loss or grads is asked for. */
int es_proposal_net_train_step(es_proposal_net *net, const float *x, const float *labels, int n, int h, int w, float lr,
                               double *loss, float *grads, void *stream);
/* Features of n crops of a picture's scale-0 words (device, w x h): crop i starts at pixel (xy[2i], xy[2i+1]) (device
 * ints, may be negative) and has fw x fh feature pixels; out (device) receives n x 2 x fh x fw floats. */
int es_proposal_features(uint64_t words, int w, int h, const int *xy, int n, int fw, int fh, float *out, void *stream);
/* The prediction of every scale-0 tile of a picture's scale-0 words (device) by the fused inference kernel: pred
 * (device, ceil(h / 64) x ceil(w / 64) floats), -inf for tiles where no pixel needs a c-value. */
int es_proposal_predict(es_proposal_net *net, uint64_t words, int w, int h, float *pred, void *stream);
void es_proposal_net_destroy(es_proposal_net *net);

/* ---------------------------------------------------------------------------------------------------------------
 * Batched frame steps: no counterpart in the reference, which scores one source per process with one launch per
 * kernel and picture (src/main.cpp:518-643). A batch holds up to 32 sources, each with its own encodes, picture size
 * and pipeline depth (at most 64 pictures in all), and scores a frame step of all of them with one launch per stage;
 * CAMBI runs beside the texture figures, and from frame 14 on a step is replayed from a CUDA graph per ring phase.
 * queue / collect keep es_frame_queue / es_frame_collect's contract (double-buffered by f % 2, frames in order).
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct es_batch es_batch;
typedef struct {
    int w, h;      /* common picture area of the source and its encodes (even) */
    int pd;        /* pipeline depth, 8 or 10 */
    int n_encodes; /* 1 to 16 */
    int cv_tile_rows[5]; /* rows of the c-value tiles per scale: 64, 32 or 16 (0 = 64); an autotuner's choice. With
                          * the learned proposal on, scales 0 and 1 use 64. */
    int cv_tile_cols[5]; /* columns of the c-value tiles per scale: 64 or 128 (0 = 64);
                          * an autotuner's choice. With the learned proposal on, every scale uses 64. */
} es_batch_source;
typedef struct {
    int use_graphs; /* replay steps from CUDA graphs once the rings are full (frame 14 on) */
} es_batch_options;

/* options NULL = {use_graphs = 1}. Pictures are numbered source by source: the source, then its encodes. */
int es_batch_create(const es_module *m, int n_sources, const es_batch_source *sources, const es_batch_options *options,
                    es_batch **out);
/* views[i]: picture i's device frame (numbered as above); crops: (x, y) per picture (even), or NULL for none;
 * source_cambi: per source, 0 to skip its CAMBI this step (a cached value is given to collect), or NULL for all.
 * The step runs after the work already queued on `stream`, and `stream` waits for it. */
int es_batch_queue(es_batch *b, long f, const es_frame_view *views, const int *crops, const int *source_cambi,
                   void *stream);
/* Waits for step f and adds its figures; frame_acc / centre_acc / out are indexed by encode, numbered source by
 * source (any may be NULL or hold NULL entries); cached_source_cambi[s] is read for sources skipped at queue time. */
int es_batch_collect(es_batch *b, long f, const double *cached_source_cambi, es_accum *const *frame_acc,
                     es_accum *const *centre_acc, es_frame_result *out);
/* Introspection for tests: as es_frame_read_windows for encode `encode` of source `source`. */
int es_batch_read_windows(es_batch *b, int source, int encode, float *stats, float *persist);
/* As es_frame_luma for picture `picture` of the batch (numbered source by source: the source, then its encodes). */
int es_batch_luma(const es_batch *b, int picture, long f, uint64_t *address);
/* Introspection for tests: the pooled value of each scale of picture `picture` in the last collected step. */
int es_batch_scale_pooled(es_batch *b, int picture, double pooled[5]);
/* Introspection for tests: as es_cambi_set_cvalue_planes for picture `picture` of later steps (dev_planes NULL
 * switches it off). Steps already captured as CUDA graphs are dropped, so later ones capture the new setting. Every
 * queued step must have been collected. */
int es_batch_set_cvalue_planes(es_batch *b, int picture, float *const dev_planes[5]);
/* The learned tile proposal (no counterpart in the reference): with a network, later steps compute c-values of
 * scales 0 and 1 only on tiles whose prediction (or, at scale 1, the prediction of a scale-0 tile it covers) reaches
 * `threshold`, plus a random audit sample (per mille of the other tiles, per scale); scales 2-4 always run. From the
 * audited tiles' exact c-value sums the device estimates how much the skipped tiles would add to each picture's score;
 * above `tolerance` the skipped tiles run too (the fallback), so the score is then exact. Scale-0 tiles with no pixel
 * that needs a c-value are skipped in every mode (they add nothing). net NULL switches the proposal off. The network
 * must stay alive while the batch uses it; after training it further, call this again. Every queued step must have
 * been collected. options NULL = {threshold 0.05, audit 50 and 200 per mille, tolerance 0.025, no budget}. */
typedef struct {
    float threshold;       /* in the network's label space, log1p(mean c-value of the tile) */
    int audit_permille[2]; /* scales 0 and 1 */
    double tolerance;      /* estimated change of the score above which the fallback runs */
    double budget;         /* > 0: per picture, also skip the scale-0 tiles of lowest prediction while their predicted
                              contribution to the score, 16 expm1(prediction) pixels / (k window^2) summed, stays
                              within this budget (the threshold becomes a floor); 0: the threshold alone */
} es_proposal_options;
int es_batch_set_proposal(es_batch *b, es_proposal_net *net, const es_proposal_options *options);
typedef struct {
    float estimate;        /* the audit's estimate of the skipped tiles' share of the score */
    int fallback;          /* 1: the skipped tiles ran too */
    uint32_t run[2];       /* proposed tiles of scales 0 and 1 */
    uint32_t audited[2], skipped[2];
} es_proposal_stats;
/* The proposal's figures for picture `picture` in the last collected step. */
int es_batch_proposal_stats(es_batch *b, int picture, es_proposal_stats *out);
/* Diagnostics: how many steps were replayed from CUDA graphs. */
uint64_t es_batch_graph_launches(const es_batch *b);
void es_batch_destroy(es_batch *b);

/* ---------------------------------------------------------------------------------------------------------------
 * Temporal alignment: the offset between a source and an encode that start at different points, found from 64 x 36
 * luma thumbnails (src/kernels.cu:502-520, src/main.cpp:301-353).
 * --------------------------------------------------------------------------------------------------------------- */
#define ES_THUMB_W 64
#define ES_THUMB_H 36
/* Thumbnails of n frames in one launch: per frame, the box means of its luma cropped to w x h at (x0, y0), on a 10-bit
 * scale (samples << (10 - depth)), into out[frame * 2304 + row * 64 + column] (device floats). Cell (tx, ty) covers
 * columns x0 + tx w / 64 .. x0 + (tx + 1) w / 64 - 1 and rows alike; a cell with no pixel is NaN. Each cell's sum is
 * an exact integer divided once, so the means equal tiny_luma's wherever a cell's sum is below 2^24 (cells up to
 * 16,400 pixels: every picture up to 8K). views: host array of n views whose luma planes are in device memory. */
int es_thumbnails(const es_frame_view *views, int n, int x0, int y0, int w, int h, uint64_t out, void *stream);
/* For each lag l = 0 .. n_ref - n_probe: the sum over probe frames i and thumbnail pixels p, in that order, of
 * |ref[l + i][p] - probe[i][p]|, each difference in float and the sum in double, as src/main.cpp:342-346 adds them.
 * ref, probe: device thumbnails, 2304 floats per frame; totals: device doubles, one per lag. */
int es_offset_totals(uint64_t ref, int n_ref, uint64_t probe, int n_probe, uint64_t totals, void *stream);
/* find_offset (src/main.cpp:336-353): the offset to add to the probe's times so that its frames match the reference's,
 * ref_times[lag] - probe_times[0] at the first lag of least mean thumbnail difference (total / (n_probe 2304)). Fewer
 * than 24 probe frames, or more probe frames than reference frames, fail with ES_ERR_INVALID; a least mean difference
 * above 16 (10-bit code values; matching pictures are well under 5) fails with ES_ERR_NO_MATCH. best_mean (may be
 * NULL) receives the least mean in both cases. Thumbnails in device memory, times (seconds) in host memory; the call
 * waits for `stream`. */
int es_find_offset(uint64_t ref, const double *ref_times, int n_ref, uint64_t probe, const double *probe_times, int n_probe,
                   void *stream, double *offset, double *best_mean);

#ifdef __cplusplus
}
#endif
#endif
