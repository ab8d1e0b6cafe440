// Shared host-side helpers: per-thread error state and RAII device memory.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <string>

namespace wk {

int set_error(int code, const std::string& msg);
void clear_error();

#define WK_CUDA(call)                                                                                      \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return ::wk::set_error(-2, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device allocation owned by one object. Nothing is allocated until alloc().
struct DevMem {
    void* p = nullptr;
    std::size_t bytes = 0;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // (Re)allocate when the current block is smaller than b. Returns cudaSuccess or the error.
    cudaError_t ensure(std::size_t b) {
        if (p && bytes >= b) return cudaSuccess;
        reset();
        if (b == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            (void)cudaGetLastError();
            return e;
        }
        bytes = b;
        return cudaSuccess;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

}  // namespace wk
