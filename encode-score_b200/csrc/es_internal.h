// Host-side helpers of the C ABI: errors carried as exceptions inside the library and turned into status codes at
// the boundary, and owning wrappers of device and page-locked memory.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/es_b200.h"
#include "es_kernels.h"

namespace es {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string &msg);
void clear_last_error();

inline void cuda_check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return;
    const int status = e == cudaErrorMemoryAllocation ? ES_ERR_ALLOC
                       : (e == cudaErrorNoDevice || e == cudaErrorNoKernelImageForDevice || e == cudaErrorInsufficientDriver)
                           ? ES_ERR_DEVICE
                           : ES_ERR_CUDA;
    throw Error(status, std::string(what) + ": " + cudaGetErrorString(e));
}

inline void require(bool ok, const std::string &what)
{
    if (!ok) throw Error(ES_ERR_INVALID, what);
}

// Runs f, turning exceptions into a status and the thread's last error.
template <typename F>
int guarded(F &&f)
{
    try {
        clear_last_error();
        f();
        return ES_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("out of host memory");
        return ES_ERR_ALLOC;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return ES_ERR_CUDA;
    }
}

template <typename T>
struct DeviceBuffer {
    T *ptr = nullptr;
    size_t count = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) { reset(n); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    ~DeviceBuffer() { release(); }
    void reset(size_t n)
    {
        release();
        if (n) cuda_check(cudaMalloc((void **)&ptr, n * sizeof(T)), "allocating GPU memory");
        count = n;
    }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
};

template <typename T>
struct PinnedBuffer {
    T *ptr = nullptr;
    size_t count = 0;
    PinnedBuffer() = default;
    explicit PinnedBuffer(size_t n) { reset(n); }
    PinnedBuffer(const PinnedBuffer &) = delete;
    PinnedBuffer &operator=(const PinnedBuffer &) = delete;
    ~PinnedBuffer() { release(); }
    void reset(size_t n)
    {
        release();
        if (n) cuda_check(cudaMallocHost((void **)&ptr, n * sizeof(T)), "allocating host memory");
        count = n;
    }
    void release()
    {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        count = 0;
    }
};

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "creating a stream"); }
    // high: the device's greatest stream priority, else its least
    explicit Stream(bool high)
    {
        int least = 0, greatest = 0;
        cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "reading stream priorities");
        cuda_check(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, high ? greatest : least), "creating a stream");
    }
    ~Stream() { if (s) cudaStreamDestroy(s); }
    Stream(const Stream &) = delete;
};

struct Event {
    cudaEvent_t e = nullptr;
    Event() { cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "creating an event"); }
    ~Event() { if (e) cudaEventDestroy(e); }
    Event(const Event &) = delete;
};

// The current device must be an sm_100 part whose kernels load; throws ES_ERR_DEVICE otherwise.
void check_device();

// CAMBI's derived parameters (src/cambi.cpp:39-53).
es_cambi_params derive_params(int w, int h);
// lut[i] = 1/i as float for i < (2 pad + 1)^2 + 1, lut[0] = 0.
void reciprocal_table(int pad, float *lut, size_t n);
// src/cambi.cpp:29: clip((int)(topk * n), 1, n).
unsigned long long topk_count(unsigned long long n, double topk);

}  // namespace es

// Makes `stream` wait until the work of the instance's last launch is done (used by es_frame so that one event on
// the caller's stream marks the end of a whole frame step).
void cambi_join(es_cambi *c, cudaStream_t stream);

namespace es {
// The figures of one encode in a collected frame step, as the device left them in page-locked memory.
struct EncodeFigures {
    double banding, source_banding;
    const unsigned long long *sse;           // Y, Cb, Cr squared errors
    const unsigned long long *source_color;  // sum U, sum V, strength in 2^-30 units
    const unsigned long long *encode_color;
    size_t n;                                // luma samples
    int pd, windows;
    const FrameFigures *fig;
    const uint16_t *bins;                    // 6 arrays of up to `windows` bins, the counting ones from the start
    const unsigned *bin_n;                   // bins in each of the first five arrays, in the lasting array
    bool texture;                            // the lasting texture of frame f - 6 is in `fig` / `bins`
};
// The two bin counts of encode e (of nenc) follow the 6 bin arrays of every encode in one buffer.
template <typename T>
inline unsigned *bin_counts(T *bins, int windows, int nenc)
{
    return (unsigned *)(bins + (size_t)windows * 6 * nenc);
}
// src/main.cpp:584-641 for one encode: adds the figures into frame_acc and, with texture, the lasting texture into
// centre_acc (either may be null), and returns the frame's result.
es_frame_result collect_encode(const EncodeFigures &in, es_accum *frame_acc, es_accum *centre_acc);
}  // namespace es

struct es_module {
    int device = 0;
};
