// es_thumbnails / es_offset_totals / es_find_offset: the offset search between a source and an encode that start at
// different points (src/main.cpp:301-353 with its tiny_luma kernel, src/kernels.cu:502-520).
#include <cstring>
#include <string>
#include <vector>

#include "es_internal.h"

using namespace es;

namespace {

void check_luma_view(const es_frame_view &v)
{
    require(v.y != nullptr, "es_thumbnails: missing luma plane");
    require(v.bytes == 1 || v.bytes == 2, "es_thumbnails: samples must be 1 or 2 bytes");
    require(v.depth == 8 || v.depth == 10, "es_thumbnails: depth must be 8 or 10");
    require(v.shift >= 0 && v.shift < 16, "es_thumbnails: bad shift");
    require(v.ypitch >= v.bytes, "es_thumbnails: bad pitch");
}

}  // namespace

extern "C" {

int es_thumbnails(const es_frame_view *views, int n, int x0, int y0, int w, int h, uint64_t out, void *stream)
{
    return guarded([&] {
        require(views != nullptr && out != 0, "es_thumbnails: NULL argument");
        require(n >= 0, "es_thumbnails: negative frame count");
        require(x0 >= 0 && y0 >= 0 && w > 0 && h > 0, "es_thumbnails: bad crop");
        for (int i = 0; i < n; i++) check_luma_view(views[i]);
        if (n == 0) return;
        check_device();
        const cudaStream_t s = (cudaStream_t)stream;
        for (int first = 0; first < n; first += kThumbFrames) {
            ThumbBatch b{};
            b.n = n - first < kThumbFrames ? n - first : kThumbFrames;
            for (int i = 0; i < b.n; i++) {
                const es_frame_view &v = views[first + i];
                FrameViewDev &d = b.f[i];
                d.y = v.y;
                d.u = v.u;
                d.v = v.v;
                d.ypitch = v.ypitch;
                d.cpitch = v.cpitch;
                d.semi = v.semi;
                d.bytes = v.bytes;
                d.shift = v.shift;
                d.depth = v.depth;
            }
            b.x0 = x0;
            b.y0 = y0;
            b.w = w;
            b.h = h;
            b.out = (float *)out + (size_t)first * kThumbPixels;
            cuda_check(launch_thumbnails(b, s), "thumbnails");
        }
    });
}

int es_offset_totals(uint64_t ref, int n_ref, uint64_t probe, int n_probe, uint64_t totals, void *stream)
{
    return guarded([&] {
        require(ref != 0 && probe != 0 && totals != 0, "es_offset_totals: NULL argument");
        require(n_probe > 0 && n_ref >= n_probe, "es_offset_totals: needs 1 <= n_probe <= n_ref");
        check_device();
        cuda_check(launch_offset_totals((const float *)ref, (const float *)probe, n_probe, n_ref - n_probe + 1, (double *)totals,
                                        (cudaStream_t)stream),
                   "offset totals");
    });
}

int es_find_offset(uint64_t ref, const double *ref_times, int n_ref, uint64_t probe, const double *probe_times, int n_probe,
                   void *stream, double *offset, double *best_mean)
{
    return guarded([&] {
        require(ref != 0 && probe != 0 && ref_times != nullptr && probe_times != nullptr && offset != nullptr,
                "es_find_offset: NULL argument");
        // src/main.cpp:338
        require(n_probe >= 24 && n_ref >= n_probe, "es_find_offset: too few frames to find the offset");
        check_device();
        const cudaStream_t s = (cudaStream_t)stream;
        const int lags = n_ref - n_probe + 1;
        DeviceBuffer<double> d_totals(lags);
        std::vector<double> totals(lags);
        cuda_check(launch_offset_totals((const float *)ref, (const float *)probe, n_probe, lags, d_totals.ptr, s), "offset totals");
        cuda_check(cudaMemcpyAsync(totals.data(), d_totals.ptr, lags * sizeof(double), cudaMemcpyDeviceToHost, s), "reading totals");
        cuda_check(cudaStreamSynchronize(s), "offset totals");
        // src/main.cpp:340-348: the first lag of least mean. The reference stops adding a lag's differences once its
        // partial total reaches the best lag's total; such a lag is not chosen there, nor here with its full total.
        double best = 1e30;
        int lag = 0;
        for (int l = 0; l < lags; l++) {
            const double mean = totals[l] / ((double)n_probe * 2304.0);
            if (mean < best) {
                best = mean;
                lag = l;
            }
        }
        if (best_mean) *best_mean = best;
        if (best > 16.0)  // src/main.cpp:349-351
            throw Error(ES_ERR_NO_MATCH, "es_find_offset: the probe does not match the reference at any lag (closest mean difference " +
                                             std::to_string(best) + ")");
        *offset = ref_times[lag] - probe_times[0];
    });
}

}  // extern "C"
