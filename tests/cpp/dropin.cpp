// Drop-in check: the reference's own calling pattern (src/main.cpp:360-364, 449-450, 523, 584) against include/gpu.hpp
// and include/cambi.hpp, in a context created with the driver API (as FFmpeg's CUDA device does, not the primary one).
// Usage: dropin PLANE.u16 W H DEPTH  -- prints the score of two launches of the plane, one per line.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cambi.hpp"

int main(int argc, char **argv)
try {
    if (argc != 5) {
        std::fprintf(stderr, "usage: dropin PLANE.u16 W H DEPTH\n");
        return 2;
    }
    const int w = std::atoi(argv[2]), h = std::atoi(argv[3]), depth = std::atoi(argv[4]);
    std::vector<uint16_t> plane((size_t)w * h);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f || std::fread(plane.data(), 2, plane.size(), f) != plane.size()) throw std::runtime_error("reading the plane");
    std::fclose(f);
    cu_check(cuInit(0), "cuInit");
    CUdevice dev;
    cu_check(cuDeviceGet(&dev, 0), "cuDeviceGet");
    CUcontext ctx;
    cu_check(cuCtxCreate(&ctx, 0, dev), "creating a context");
    Kernels kernels;
    kernels.load();
    CUfunction cv = kernels.get("cambi_cvalues");
    if (!cv) throw std::runtime_error("no c-value kernel");
    bool refused = false;
    try {
        kernels.get("tiny_luma");  // a reference kernel outside this path
    } catch (const std::runtime_error &) {
        refused = true;
    }
    if (!refused) throw std::runtime_error("an unknown kernel name was accepted");
    CUstream stream;
    cu_check(cuStreamCreate(&stream, CU_STREAM_NON_BLOCKING), "creating a stream");
    CUdeviceptr img;
    cu_check(cuMemAlloc(&img, plane.size() * 2), "allocating GPU memory");
    cu_check(cuMemcpyHtoD(img, plane.data(), plane.size() * 2), "uploading");
    {
        Cambi cambi(kernels, w, h, depth);
        for (int i = 0; i < 2; i++) {
            cambi.launch(img, w, stream);
            std::printf("%.17g\n", cambi.finish());
        }
    }
    cuMemFree(img);
    cuStreamDestroy(stream);
    cuCtxDestroy(ctx);
    return 0;
} catch (const std::exception &e) {
    std::fprintf(stderr, "dropin: %s\n", e.what());
    return 1;
}
