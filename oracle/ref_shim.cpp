// TEST INFRASTRUCTURE, not product code: a C harness around the reference's own GPU implementation, compiled
// unmodified from the reference's src/cambi.cpp, src/gpu.cpp and src/kernels.cu into oracle/_ref/ (oracle/Makefile).
//
// It gives tests and measurement scripts:
//  * the reference's class Cambi (src/cambi.hpp:9-21) behind plain C functions;
//  * the reference's CAMBI kernels run step by step with the launch shapes of src/cambi.cpp:88-135, keeping every
//    scale's picture, mask and c-values for bit-exact comparison;
//  * frame_planes, window_stats, persist_stats, plane_sse and color_sums with the launch shapes of
//    src/main.cpp:502-566;
//  * tiny_luma with the launch shape of src/main.cpp:321;
//  * to_picture with the launch shape of src/main.cpp:511.
// The four libvmaf luminance functions src/cambi.cpp declares (lines 7-15) are supplied here from the same published
// model the product uses (BT.1886, 10-bit limited range, 300 / 0.01 cd/m2), so both sides share one parameter set.
#include <cuda.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "cambi.hpp"

namespace {
thread_local std::string g_error;

double bt1886(double v)
{
    const double g = 2.4, lw = std::pow(300.0, 1.0 / g), lb = std::pow(0.01, 1.0 / g);
    const double a = std::pow(lw - lb, g), b = lb / (lw - lb);
    return a * std::pow(v + b > 0 ? v + b : 0.0, g);
}

template <typename F>
int guarded(F &&f)
{
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

struct RefScales {
    CUdeviceptr img[5], mask[5], out[5];
    int w[5], h[5], first[6];
    CUdeviceptr sum, count;
};
struct RefParams {
    int w, h, pad, band_base, band_size, vlt;
    int tvi[4];
    int weight[4];
};
}  // namespace

extern "C" {

typedef struct { int foot, head; } VmafLumaRange;
typedef double (*VmafEOTF)(double);

int vmaf_luminance_init_luma_range(VmafLumaRange *range, int bitdepth, int pixel_range)
{
    // limited range: black at 16, white at 235, scaled to the bit depth
    const int shift = bitdepth - 8;
    range->foot = pixel_range ? 16 << shift : 0;
    range->head = pixel_range ? 235 << shift : (1 << bitdepth) - 1;
    return 0;
}

int vmaf_luminance_init_eotf(VmafEOTF *eotf, const char *name)
{
    if (std::strcmp(name, "bt1886") != 0) return -1;
    *eotf = bt1886;
    return 0;
}

static double luminance_of(int code, VmafLumaRange r, VmafEOTF eotf)
{
    double v = (double)(code - r.foot) / (double)(r.head - r.foot);
    v = v < 0 ? 0 : v > 1 ? 1 : v;
    return eotf(v);
}

int get_tvi_for_diff(int diff, double tvi_threshold, int bitdepth, VmafLumaRange range, VmafEOTF eotf)
{
    (void)bitdepth;
    int last = range.foot;
    for (int code = range.foot; code + diff <= range.head; code++) {
        const double l = luminance_of(code, range, eotf);
        if (luminance_of(code + diff, range, eotf) - l > tvi_threshold * l) last = code;
    }
    return last;
}

int get_vlt_luma(double threshold, VmafLumaRange range, VmafEOTF eotf)
{
    int last = range.foot;
    for (int code = range.foot; code <= range.head; code++)
        if (luminance_of(code, range, eotf) <= threshold) last = code;
    return last;
}

const char *ref_error(void) { return g_error.c_str(); }

int ref_init(void)
{
    return guarded([] {
        cu_check(cuInit(0), "cuInit");
        CUcontext ctx = nullptr;
        cu_check(cuCtxGetCurrent(&ctx), "cuCtxGetCurrent");
        if (!ctx) {
            CUdevice dev;
            cu_check(cuDeviceGet(&dev, 0), "cuDeviceGet");
            cu_check(cuDevicePrimaryCtxRetain(&ctx, dev), "cuDevicePrimaryCtxRetain");
            cu_check(cuCtxSetCurrent(ctx), "cuCtxSetCurrent");
        }
    });
}

void *ref_kernels(void)
{
    Kernels *k = new Kernels;
    if (guarded([&] { k->load(); })) {
        delete k;
        return nullptr;
    }
    return k;
}

void *ref_cambi_create(void *k, int w, int h, int depth)
{
    Cambi *c = nullptr;
    guarded([&] { c = new Cambi(*(Kernels *)k, w, h, depth); });
    return c;
}

int ref_cambi_launch(void *c, uint64_t img, int pitch, uint64_t stream)
{
    return guarded([&] { ((Cambi *)c)->launch((CUdeviceptr)img, pitch, (CUstream)stream); });
}

int ref_cambi_finish(void *c, double *score)
{
    return guarded([&] { *score = ((Cambi *)c)->finish(); });
}

void ref_cambi_destroy(void *c) { delete (Cambi *)c; }

// p: pad, band_base, band_size, vlt, tvi[4], weight[4], mask_index
int ref_cambi_steps(void *kp, uint64_t img, int pitch, int w, int h, int depth, const int *p, const uint64_t *images,
                    const uint64_t *masks, const uint64_t *cvalues, uint64_t scratch, uint64_t sums)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        CUdeviceptr s0 = (CUdeviceptr)scratch;
        CUdeviceptr in = (CUdeviceptr)img;
        int ww = w, hh = h;
        if (depth == 8) {
            void *a[] = {&in, &pitch, &ww, &hh, &s0};
            Kernels::launch(k.get("cambi_from8"), w, h, a, nullptr);
        } else {
            CUDA_MEMCPY2D m = {};
            m.srcMemoryType = m.dstMemoryType = CU_MEMORYTYPE_DEVICE;
            m.srcDevice = in;
            m.srcPitch = (size_t)pitch * 2;
            m.dstDevice = s0;
            m.dstPitch = (size_t)w * 2;
            m.WidthInBytes = (size_t)w * 2;
            m.Height = h;
            cu_check(cuMemcpy2D(&m), "copy");
        }
        int idx = p[12];
        CUdeviceptr m0 = (CUdeviceptr)masks[0];
        {
            void *a[] = {&s0, &ww, &hh, &idx, &m0};
            cu_check(cuLaunchKernel(k.get("cambi_mask"), (w + 127) / 128, (h + 31) / 32, 1, 32, 4, 1, 0, nullptr, a, nullptr), "mask");
        }
        int sw[5], sh[5];
        sw[0] = w;
        sh[0] = h;
        for (int s = 1; s < 5; s++) {
            sw[s] = (sw[s - 1] + 1) >> 1;
            sh[s] = (sh[s - 1] + 1) >> 1;
        }
        for (int s = 0; s < 5; s++) {
            int cw = sw[s], ch = sh[s];
            if (s > 0) {
                int pw = sw[s - 1];
                CUdeviceptr prev = (CUdeviceptr)images[s - 1], pm = (CUdeviceptr)masks[s - 1], dm = (CUdeviceptr)masks[s];
                void *a[] = {&prev, &pw, &s0, &cw, &ch};
                Kernels::launch(k.get("cambi_decimate16"), cw, ch, a, nullptr);
                void *b[] = {&pm, &pw, &dm, &cw, &ch};
                Kernels::launch(k.get("cambi_decimate8"), cw, ch, b, nullptr);
            }
            CUdeviceptr dst = (CUdeviceptr)images[s];
            void *a[] = {&s0, &cw, &ch, &dst};
            Kernels::launch(k.get("cambi_mode"), cw, ch, a, nullptr);
        }
        RefScales sc;
        int blocks = 0;
        for (int s = 0; s < 5; s++) {
            sc.img[s] = (CUdeviceptr)images[s];
            sc.mask[s] = (CUdeviceptr)masks[s];
            sc.out[s] = (CUdeviceptr)cvalues[s];
            sc.w[s] = sw[s];
            sc.h[s] = sh[s];
            sc.first[s] = blocks;
            blocks += (sw[s] + 63) / 64 * ((sh[s] + 31) / 32);
            cu_check(cuMemsetD32((CUdeviceptr)cvalues[s], 0, (size_t)sw[s] * sh[s]), "clear");
        }
        sc.first[5] = blocks;
        sc.sum = (CUdeviceptr)sums;
        sc.count = (CUdeviceptr)sums + 40;
        cu_check(cuMemsetD8((CUdeviceptr)sums, 0, 80), "clear");
        RefParams rp;
        rp.w = w;
        rp.h = h;
        rp.pad = p[0];
        rp.band_base = p[1];
        rp.band_size = p[2];
        rp.vlt = p[3];
        for (int d = 0; d < 4; d++) {
            rp.tvi[d] = p[4 + d];
            rp.weight[d] = p[8 + d];
        }
        // the dynamic shared memory src/cambi.cpp:55-56 sizes for cambi_cvalues
        const int columns = 64 + 2 * rp.pad + 1;
        const unsigned shared = (unsigned)(columns * 32 + (columns >> 4) * 8 + 8 + 32 * 33 * 2 + (rp.band_size + 8) * 2);
        CUfunction cv = k.get("cambi_cvalues");
        // only ever raise the limit above the default 48 KB: a lower one would make the reference's own Cambi class,
        // which never sets it, fail later launches that need more
        if (shared > 48 * 1024)
            cu_check(cuFuncSetAttribute(cv, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)shared), "smem");
        void *a[] = {&sc, &rp};
        cu_check(cuLaunchKernel(cv, blocks, 1, 1, 32, 1, 1, shared, nullptr, a, nullptr), "cvalues");
        cu_check(cuCtxSynchronize(), "cvalues");
    });
}

int ref_frame_planes(void *kp, const void *view, int x0, int y0, int pd, uint64_t y16, uint64_t u, uint64_t v, int w, int h)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        struct { const void *y, *u, *v; int ypitch, cpitch, semi, bytes, shift, depth; } f;
        std::memcpy(&f, view, sizeof f);
        CUdeviceptr Y = y16, U = u, V = v;
        void *a[] = {&f, &x0, &y0, &pd, &Y, &U, &V, &w, &h};
        Kernels::launch(k.get("frame_planes"), w, h, a, nullptr);
        cu_check(cuCtxSynchronize(), "frame_planes");
    });
}

int ref_window_stats(void *kp, uint64_t yr, uint64_t yd, int up, int w, int h, uint64_t mid_r, uint64_t mid_d, uint64_t out)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        CUdeviceptr a0 = yr, a1 = yd, a5 = mid_r, a6 = mid_d, a7 = out;
        const int ww = w / 16, wh = h / 16;
        void *a[] = {&a0, &a1, &up, &w, &h, &a5, &a6, &a7};
        cu_check(cuLaunchKernel(k.get("window_stats"), (ww + 7) / 8, (wh + 1) / 2, 1, 32, 4, 1, 0, nullptr, a, nullptr), "window_stats");
        cu_check(cuCtxSynchronize(), "window_stats");
    });
}

int ref_persist_stats(void *kp, uint64_t ring, uint64_t plane, int centre, uint64_t mid_d, int w, int h, uint64_t out)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        CUdeviceptr r = ring, m = mid_d, o = out;
        size_t pl = plane;
        const int ww = w / 16, wh = h / 16;
        void *a[] = {&r, &pl, &centre, &m, &w, &o};
        cu_check(cuLaunchKernel(k.get("persist_stats"), ww, wh, 1, 256, 1, 1, 0, nullptr, a, nullptr), "persist_stats");
        cu_check(cuCtxSynchronize(), "persist_stats");
    });
}

int ref_plane_sse(void *kp, uint64_t a_, uint64_t b_, uint64_t n, uint64_t sse)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        CUdeviceptr a = a_, b = b_, null = 0, s = sse;
        size_t nn = n;
        cu_check(cuMemsetD8(s, 0, 8), "clear");
        void *args[] = {&a, &b, &null, &null, &nn, &s};
        cu_check(cuLaunchKernel(k.get("plane_sse"), 256, 1, 1, 256, 1, 1, 0, nullptr, args, nullptr), "plane_sse");
        cu_check(cuCtxSynchronize(), "plane_sse");
    });
}

int ref_color_sums(void *kp, uint64_t u_, uint64_t v_, uint64_t n, int up, uint64_t sums)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        CUdeviceptr u = u_, v = v_, s = sums;
        size_t nn = n;
        cu_check(cuMemsetD8(s, 0, 24), "clear");
        void *args[] = {&u, &v, &nn, &up, &s};
        cu_check(cuLaunchKernel(k.get("color_sums"), 256, 1, 1, 256, 1, 1, 0, nullptr, args, nullptr), "color_sums");
        cu_check(cuCtxSynchronize(), "color_sums");
    });
}

// tiny_luma with the launch shape of src/main.cpp:321 (64 x 36 blocks of 32 x 8 threads): one frame's thumbnail.
int ref_tiny_luma(void *kp, const void *view, int x0, int y0, int w, int h, uint64_t out)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        struct { const void *y, *u, *v; int ypitch, cpitch, semi, bytes, shift, depth; } f;
        std::memcpy(&f, view, sizeof f);
        CUdeviceptr o = out;
        void *a[] = {&f, &x0, &y0, &w, &h, &o};
        cu_check(cuLaunchKernel(k.get("tiny_luma"), 64, 36, 1, 32, 8, 1, 0, nullptr, a, nullptr), "tiny_luma");
        cu_check(cuCtxSynchronize(), "tiny_luma");
    });
}

// to_picture with the launch shape of src/main.cpp:511 (Kernels::launch over w x h): one plane into one picture.
int ref_to_picture(void *kp, uint64_t src, int w, int h, uint64_t dst, int pitch, int bytes)
{
    return guarded([&] {
        const Kernels &k = *(Kernels *)kp;
        CUdeviceptr s = src, d = dst;
        void *a[] = {&s, &w, &h, &d, &pitch, &bytes};
        Kernels::launch(k.get("to_picture"), w, h, a, nullptr);
        cu_check(cuCtxSynchronize(), "to_picture");
    });
}

}  // extern "C"
