// Drop-in for the reference's src/cambi.hpp (lines 1-36): class Cambi with the same public signatures and contract,
// implemented over the C ABI of libes_b200.so (es_b200.h).
//
// CAMBI banding score of a luma plane on the GPU. launch() reads the plane on the caller's stream, after the work
// already queued there, and continues on the instance's own stream, so the caller may overwrite the plane with work it
// queues on its stream afterwards; finish() waits and returns the score, clamped to 1000. Each launch() is followed by
// its finish() before the instance's next launch().
#pragma once
#include <cstdint>

#include "gpu.hpp"

class Cambi {
public:
    // `depth` is the bit depth of the planes it will be given, 8 or 10 (src/cambi.hpp:11-12).
    Cambi(const Kernels &k, int w, int h, int depth) { es_check(es_cambi_create(k.handle(), w, h, depth, &c_), "cambi buffers"); }
    ~Cambi() { es_cambi_destroy(c_); }
    Cambi(const Cambi &) = delete;
    Cambi &operator=(const Cambi &) = delete;
    // src/cambi.hpp:15-18: the plane at `img` (values at `depth` bits, `pitch` in pixels).
    void launch(CUdeviceptr img, int pitch, CUstream stream) { es_check(es_cambi_launch(c_, (uint64_t)img, pitch, (void *)stream), "cambi"); }
    // src/cambi.hpp:19-20
    double finish()
    {
        double s = 0;
        es_check(es_cambi_finish(c_, &s), "cambi");
        return s;
    }

private:
    es_cambi *c_ = nullptr;
};
