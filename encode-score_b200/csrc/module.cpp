// The kernel module (Kernels of src/gpu.hpp:15-23 / src/gpu.cpp:6-19), error reporting, and CAMBI's derived
// parameters (src/cambi.cpp:21-53) with the luminance model restated from its published definitions.
#include <cuda.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "es_internal.h"

namespace es {

namespace {
thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(long long n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

// ---- kernel timing (diagnostics) -------------------------------------------------------------------------------------
namespace {
struct Timing {
    std::mutex m;
    std::atomic<bool> on{false}, serial{false};
    struct Pending {
        std::string name;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> free_pairs;
    std::map<std::string, std::pair<double, uint64_t>> totals;
};
Timing &timing()
{
    static Timing *t = new Timing;  // never destroyed: launches may outlive static destruction
    return *t;
}
}  // namespace

LaunchTimer::LaunchTimer(const char *name, cudaStream_t s) : stream(s)
{
    Timing &t = timing();
    if (!t.on.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lock(t.m);
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (!t.free_pairs.empty()) {
        ev = t.free_pairs.back();
        t.free_pairs.pop_back();
    } else if (cudaEventCreate(&ev.first) != cudaSuccess || cudaEventCreate(&ev.second) != cudaSuccess) {
        return;
    }
    if (cudaEventRecord(ev.first, s) != cudaSuccess) {
        t.free_pairs.push_back(ev);
        return;
    }
    slot = (int)t.pending.size();
    t.pending.push_back({name, ev.first, ev.second});
}

LaunchTimer::~LaunchTimer()
{
    if (slot < 0) return;
    Timing &t = timing();
    std::lock_guard<std::mutex> lock(t.m);
    if (slot < (int)t.pending.size()) cudaEventRecord(t.pending[slot].b, stream);
}

bool serial_streams() { return timing().serial.load(std::memory_order_relaxed); }
bool kernel_timing_on() { return timing().on.load(std::memory_order_relaxed); }

void set_last_error(const std::string &msg) { g_last_error = msg; }
void clear_last_error() { g_last_error.clear(); }

// The kernels the library registers, by the names Kernels::get accepts. Their entry points are looked up through
// the runtime from these host stubs.
struct NamedKernel {
    const char *name;
    const void *(*entry)();
};
const void *kernel_entry_prep0();
const void *kernel_entry_decimate_mode();
const void *kernel_entry_cvalues();
const void *kernel_entry_unpack();
const void *kernel_entry_window_stats();
const void *kernel_entry_persist();
const void *kernel_entry_pair_sums();
const void *kernel_entry_collect();

static const NamedKernel kKernels[] = {
    {"cambi_prep0", kernel_entry_prep0},           {"cambi_decimate_mode", kernel_entry_decimate_mode},
    {"cambi_cvalues", kernel_entry_cvalues},       {"frame_unpack", kernel_entry_unpack},
    {"window_stats", kernel_entry_window_stats},   {"persist_stats", kernel_entry_persist},
    {"pair_sums", kernel_entry_pair_sums},         {"frame_collect", kernel_entry_collect},
};

void check_device()
{
    // devices already found to be sm_100 with loadable kernels: reading all of a device's properties takes
    // milliseconds, too long for entry points called per batch of frames
    static std::atomic<uint64_t> verified{0};
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "finding the CUDA device");
    if (dev >= 0 && dev < 64 && ((verified.load(std::memory_order_acquire) >> dev) & 1u)) return;
    cudaDeviceProp prop;
    cuda_check(cudaGetDeviceProperties(&prop, dev), "reading the device's properties");
    if (prop.major != 10 || prop.minor != 0)
        throw Error(ES_ERR_DEVICE, std::string("device ") + prop.name + " is sm_" + std::to_string(prop.major) + std::to_string(prop.minor) +
                                       "; this library runs on sm_100 (B200) only");
    cudaFuncAttributes attr;
    cuda_check(cudaFuncGetAttributes(&attr, kernel_entry_cvalues()), "loading the kernels");
    if (dev >= 0 && dev < 64) verified.fetch_or(uint64_t(1) << dev, std::memory_order_acq_rel);
}

// ---- CAMBI parameters ---------------------------------------------------------------------------------------------
// ITU-R BT.1886 Annex 1 EOTF, L = a max(V + b, 0)^2.4, for a 300 cd/m2 white / 0.01 cd/m2 black reference display on
// 10-bit limited-range codes (64 .. 940); a step of d codes at code v is visible when L(v + d) - L(v) > 0.019 L(v)
// (CAMBI's Weber threshold).
namespace {
constexpr double kGamma = 2.4, kWhite = 300.0, kBlack = 0.01, kTvi = 0.019;
constexpr int kFoot = 64, kHead = 940;

double luminance(int code)
{
    const double lw = std::pow(kWhite, 1.0 / kGamma), lb = std::pow(kBlack, 1.0 / kGamma);
    const double a = std::pow(lw - lb, kGamma), b = lb / (lw - lb);
    double v = (double)(code - kFoot) / (double)(kHead - kFoot);
    v = v < 0 ? 0 : v > 1 ? 1 : v;
    return a * std::pow(v + b > 0 ? v + b : 0.0, kGamma);
}

int tvi_for_diff(int diff)
{
    int last = kFoot;
    for (int code = kFoot; code + diff <= kHead; code++) {
        const double l = luminance(code);
        if (luminance(code + diff) - l > kTvi * l) last = code;
    }
    return last;
}

int vlt_luma(double threshold)
{
    int last = kFoot;
    for (int code = kFoot; code <= kHead; code++)
        if (luminance(code) <= threshold) last = code;
    return last;
}

int ceil_log2(uint32_t n)
{
    int s = 0;
    for (uint32_t t = n ? n - 1 : 0; t; t >>= 1) s++;
    return s;
}
}  // namespace

struct LumaThresholds {
    int tvi[kDiffs], vlt;
    LumaThresholds()
    {
        for (int d = 0; d < kDiffs; d++) tvi[d] = tvi_for_diff(d + 1);
        vlt = vlt_luma(0.0);
    }
};

es_cambi_params derive_params(int w, int h)
{
    static const LumaThresholds thresholds;  // initialised once, thread-safely
    const int *tvi = thresholds.tvi, vlt = thresholds.vlt;
    es_cambi_params p;
    std::memset(&p, 0, sizeof p);
    p.w = w;
    p.h = h;
    p.window = ((65 * (w + h) / 375) >> 4) | 1;
    p.pad = p.window >> 1;
    p.mask_index = (49 + 3 * (ceil_log2((uint32_t)((w >> 6) * (h >> 6))) - 11) - 1) >> 1;
    for (int d = 0; d < kDiffs; d++) {
        p.tvi[d] = tvi[d] + kDiffs;
        p.weight[d] = d + 1;
    }
    p.vlt = vlt;
    p.band_base = vlt - 3 * kDiffs + 1 > 0 ? vlt - 3 * kDiffs + 1 : 0;
    p.band_size = p.tvi[kDiffs - 1] + 1 - p.band_base;
    p.topk = 0.6;
    return p;
}

void reciprocal_table(int pad, float *lut, size_t n)
{
    (void)pad;
    lut[0] = 0.0f;
    for (size_t i = 1; i < n; i++) lut[i] = (float)(1.0 / (double)i);
}

unsigned long long topk_count(unsigned long long n, double topk)
{
    const unsigned long long k = (unsigned long long)(int)(topk * (double)n);
    return k < 1 ? 1 : k > n ? n : k;
}

}  // namespace es

using namespace es;

extern "C" {

const char *es_last_error(void) { return g_last_error.c_str(); }

int es_version(void) { return 10000; }

uint64_t es_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int es_kernel_timing(int on)
{
    return guarded([&] {
        Timing &t = timing();
        std::lock_guard<std::mutex> lock(t.m);
        require(on >= 0 && on <= 2, "es_kernel_timing: on must be 0, 1 or 2");
        t.on = on != 0;
        t.serial = on == 2;
        if (on) t.totals.clear();
    });
}

int es_kernel_times(char *names, double *total_ms, uint64_t *launches, int max, int *count)
{
    return guarded([&] {
        require(count != nullptr, "es_kernel_times: count is NULL");
        cuda_check(cudaDeviceSynchronize(), "waiting for timed kernels");
        Timing &t = timing();
        std::lock_guard<std::mutex> lock(t.m);
        for (const Timing::Pending &p : t.pending) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                auto &e = t.totals[p.name];
                e.first += ms;
                e.second++;
            }
            t.free_pairs.push_back({p.a, p.b});
        }
        t.pending.clear();
        int i = 0;
        for (const auto &kv : t.totals) {
            if (i < max) {
                if (names) {
                    std::memset(names + (size_t)i * 32, 0, 32);
                    std::strncpy(names + (size_t)i * 32, kv.first.c_str(), 31);
                }
                if (total_ms) total_ms[i] = kv.second.first;
                if (launches) launches[i] = kv.second.second;
            }
            i++;
        }
        *count = i;
    });
}

int es_module_load(es_module **out)
{
    return guarded([&] {
        require(out != nullptr, "es_module_load: out is NULL");
        check_device();
        auto *m = new es_module;
        cuda_check(cudaGetDevice(&m->device), "finding the CUDA device");
        *out = m;
    });
}

void es_module_unload(es_module *m) { delete m; }

int es_module_get(const es_module *m, const char *name, void **function)
{
    return guarded([&] {
        require(m != nullptr && name != nullptr && function != nullptr, "es_module_get: NULL argument");
        for (const NamedKernel &k : kKernels)
            if (std::strcmp(k.name, name) == 0) {
                cudaFunction_t f;
                cuda_check(cudaGetFuncBySymbol(&f, k.entry()), name);
                *function = (void *)f;
                return;
            }
        throw Error(ES_ERR_INVALID, std::string(name) + ": named symbol not found");
    });
}

int es_module_launch(void *function, unsigned w, unsigned h, void **args, void *stream)
{
    return guarded([&] {
        require(function != nullptr, "es_module_launch: NULL function");
        // the driver's launch entry point, looked up through the runtime so the library does not link libcuda
        using Launch = CUresult (*)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                                    CUstream, void **, void **);
        using ErrorString = CUresult (*)(CUresult, const char **);
        static Launch launch = nullptr;
        static ErrorString error_string = nullptr;
        if (!launch) {
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            cuda_check(cudaGetDriverEntryPoint("cuLaunchKernel", &fn, cudaEnableDefault, &q), "finding cuLaunchKernel");
            require(q == cudaDriverEntryPointSuccess && fn, "cuLaunchKernel is not available");
            launch = (Launch)fn;
            fn = nullptr;
            if (cudaGetDriverEntryPoint("cuGetErrorString", &fn, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
                error_string = (ErrorString)fn;
        }
        const unsigned bx = 32, by = 8;
        const CUresult r = launch((CUfunction)function, (w + bx - 1) / bx, (h + by - 1) / by, 1, bx, by, 1, 0, (CUstream)stream, args, nullptr);
        if (r != CUDA_SUCCESS) {
            const char *msg = nullptr;
            if (error_string) error_string(r, &msg);
            throw Error(ES_ERR_CUDA, std::string("kernel launch: ") + (msg ? msg : "unknown CUDA error"));
        }
    });
}

int es_cambi_derive_params(int w, int h, es_cambi_params *out)
{
    return guarded([&] {
        require(out != nullptr, "es_cambi_derive_params: out is NULL");
        require(w > 0 && h > 0, "es_cambi_derive_params: picture size must be positive");
        *out = derive_params(w, h);
    });
}

}  // extern "C"
