// es_windows: texture window energies on windows of 16 k pixels in three arithmetics (the precision study); no
// counterpart in the reference, whose window is fixed at 16 x 16 (src/kernels.cu:331) and summed in FP32.
#include <memory>

#include "es_internal.h"

namespace es {
int precision_quantities();
cudaError_t launch_precision_sat(const uint16_t *y, int w, int h, int up, long long *si, float *shi, float *slo, float *sp,
                                 cudaStream_t s);
cudaError_t launch_precision_blocks(const uint16_t *yr, const uint16_t *yd, int w, int h, int up, const long long *const si[2],
                                    const float *const shi[2], const float *const slo[2], const float *const sp[2], long long *qi,
                                    float *qc, float *qp, cudaStream_t s);
cudaError_t launch_precision_windows(const long long *qi, const float *qc, const float *qp, int bw, int bh, int k, int mode,
                                     double *out, cudaStream_t s);
}  // namespace es

using namespace es;

struct es_windows {
    int w = 0, h = 0, bw = 0, bh = 0;
    DeviceBuffer<long long> si[2];
    DeviceBuffer<float> shi[2], slo[2], sp[2];
    DeviceBuffer<long long> qi;
    DeviceBuffer<float> qc, qp;
    bool ready = false;
};

extern "C" {

int es_windows_create(int w, int h, es_windows **out)
{
    return guarded([&] {
        require(out != nullptr, "es_windows_create: NULL argument");
        require(w >= 16 && h >= 16, "es_windows_create: the picture must be at least 16 x 16");
        check_device();
        auto p = std::make_unique<es_windows>();
        p->w = w;
        p->h = h;
        p->bw = w / 16;
        p->bh = h / 16;
        const size_t n = (size_t)w * h, q = (size_t)p->bw * p->bh * precision_quantities();
        for (int i = 0; i < 2; i++) {
            p->si[i].reset(n);
            p->shi[i].reset(n);
            p->slo[i].reset(n);
            p->sp[i].reset(n);
        }
        p->qi.reset(q);
        p->qc.reset(q);
        p->qp.reset(q);
        *out = p.release();
    });
}

int es_windows_compute(es_windows *p, uint64_t src, uint64_t enc, int up, void *stream)
{
    return guarded([&] {
        require(p != nullptr && src != 0 && enc != 0, "es_windows_compute: NULL argument");
        require(up == 0 || up == 2, "es_windows_compute: up must be 0 (10-bit) or 2 (8-bit)");
        cudaStream_t s = (cudaStream_t)stream;
        const uint16_t *y[2] = {(const uint16_t *)src, (const uint16_t *)enc};
        for (int i = 0; i < 2; i++)
            cuda_check(launch_precision_sat(y[i], p->w, p->h, up, p->si[i].ptr, p->shi[i].ptr, p->slo[i].ptr, p->sp[i].ptr, s),
                       "summed-area tables");
        const long long *si[2] = {p->si[0].ptr, p->si[1].ptr};
        const float *shi[2] = {p->shi[0].ptr, p->shi[1].ptr}, *slo[2] = {p->slo[0].ptr, p->slo[1].ptr}, *sp[2] = {p->sp[0].ptr, p->sp[1].ptr};
        cuda_check(launch_precision_blocks(y[0], y[1], p->w, p->h, up, si, shi, slo, sp, p->qi.ptr, p->qc.ptr, p->qp.ptr, s),
                   "block sums");
        p->ready = true;
    });
}

int es_windows_figures(es_windows *p, int window, int mode, double *out, void *stream)
{
    return guarded([&] {
        require(p != nullptr && out != nullptr, "es_windows_figures: NULL argument");
        require(window >= 16 && window % 16 == 0, "es_windows_figures: the window must be a multiple of 16");
        require(mode >= 0 && mode <= 2, "es_windows_figures: mode 0 (integer), 1 (compensated FP32) or 2 (FP32)");
        if (!p->ready) throw Error(ES_ERR_STATE, "es_windows_figures: nothing computed");
        cuda_check(launch_precision_windows(p->qi.ptr, p->qc.ptr, p->qp.ptr, p->bw, p->bh, window / 16, mode, out, (cudaStream_t)stream),
                   "window figures");
    });
}

void es_windows_destroy(es_windows *p)
{
    if (!p) return;
    cudaDeviceSynchronize();
    delete p;
}

}  // extern "C"
