// Drop-in for the reference's src/gpu.hpp (lines 1-23): cu_check and class Kernels with the same public signatures,
// implemented over the C ABI of libes_b200.so (es_b200.h). Kernels::load() binds the library's sm_100a kernels to the
// current CUDA context; get(name) returns one of them (see es_module_get for the names); launch() runs a 2-D kernel
// in 32 x 8 blocks like the reference's helper.
#pragma once
#include <cuda.h>

#include <stdexcept>
#include <string>

#include "es_b200.h"

// src/gpu.hpp:7-13: a driver API error becomes std::runtime_error("what: message").
inline void cu_check(CUresult r, const char *what)
{
    if (r == CUDA_SUCCESS) return;
    const char *msg = nullptr;
    cuGetErrorString(r, &msg);
    throw std::runtime_error(std::string(what) + ": " + (msg ? msg : "unknown CUDA error"));
}

// The library's own failures become the same exception type, with the library's message.
inline void es_check(int status, const char *what)
{
    if (status == ES_OK) return;
    throw std::runtime_error(std::string(what) + ": " + es_last_error());
}

class Kernels {
public:
    Kernels() = default;
    ~Kernels() { es_module_unload(module_); }
    Kernels(const Kernels &) = delete;
    Kernels &operator=(const Kernels &) = delete;
    // src/gpu.cpp:6
    void load() { es_check(es_module_load(&module_), "loading kernels"); }
    // src/gpu.cpp:8-13
    CUfunction get(const char *name) const
    {
        void *f = nullptr;
        es_check(es_module_get(module_, name, &f), name);
        return (CUfunction)f;
    }
    // src/gpu.hpp:19. The library's kernels live in the CUDA runtime's own module of libes_b200.so, not in a module
    // loaded with cuModuleLoadData, so there is no CUmodule to hand out: this returns a null handle (the reference's
    // program never calls it). handle() is the library's own module handle, for the es_b200.h calls.
    CUmodule module() const { return nullptr; }
    es_module *handle() const { return module_; }
    // src/gpu.cpp:15-19
    static void launch(CUfunction f, unsigned w, unsigned h, void **args, CUstream stream = nullptr)
    {
        es_check(es_module_launch((void *)f, w, h, args, (void *)stream), "kernel launch");
    }

private:
    es_module *module_ = nullptr;
};
