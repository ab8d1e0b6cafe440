// Shared host-side helpers: per-thread error state and RAII device memory.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <string>

// Register budget of the pure-gather step kernels (k_step_fast, k_step_fast_batch): blocks of
// at most WK_FAST_MAX_THREADS threads, at least WK_FAST_TRT_MIN_BLOCKS (TRT, two nodes per
// thread) or WK_FAST_OTHER_MIN_BLOCKS (BGK / MRT, one node per thread) of them resident per SM.
// 64 x 10 gives the packed TRT form 96 registers (20 warps per SM), measured 5-7% faster on the
// D3Q19 sphere channel than 128 registers (16 warps) and 20% faster than 80 (24 warps, spills).
// 64 x 8 lets the D3Q27 MRT step keep its moments in 106 registers without spills: 10% (FP32)
// and 16% (FP16 / BF16) faster on the 384^3 Taylor-Green vortex than the 64-register cap.
#ifndef WK_FAST_MAX_THREADS
#define WK_FAST_MAX_THREADS 64
#endif
#ifndef WK_FAST_TRT_MIN_BLOCKS
#define WK_FAST_TRT_MIN_BLOCKS 10
#endif
#ifndef WK_FAST_OTHER_MIN_BLOCKS
#define WK_FAST_OTHER_MIN_BLOCKS 8
#endif
// D2Q9 TRT carries nine populations per node, half of D3Q19's: at 16 blocks per SM it fits 64
// registers without spills, twice the resident warps, which its fewer loads per thread need to
// keep enough bytes in flight.
#ifndef WK_FAST_TRT9_MIN_BLOCKS
#define WK_FAST_TRT9_MIN_BLOCKS 16
#endif

namespace wk {

int set_error(int code, const std::string& msg);
void clear_error();

#define WK_CUDA(call)                                                                                      \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return ::wk::set_error(-2, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device blocks are taken from, and may be handed back to, a process-wide cache
// (alloc_cache.cpp). cudaFree synchronises the whole device, so an object whose
// work is known to be finished (its stream synchronised) returns its blocks with
// release() instead: a serving loop can then retire jobs and start new ones while
// other streams keep running, and a new lattice reuses the retired one's memory
// without a cudaMalloc. reset() keeps the synchronous cudaFree for blocks whose
// last use is not known to have finished.
cudaError_t cache_alloc(void** p, std::size_t bytes, std::size_t* block_bytes);
void cache_release(void* p, std::size_t block_bytes);
std::size_t cache_trim();         // cudaFree every cached block of the current device; bytes freed
std::size_t cache_held_bytes();   // bytes held by the cache on the current device

// Device allocation owned by one object. Nothing is allocated until ensure().
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
    // Hand the block to the cache; only when no queued work can still touch it.
    void release() {
        if (p) cache_release(p, bytes);
        p = nullptr;
        bytes = 0;
    }
    // Grow to at least b bytes when no queued work can still use the current block: the old
    // block goes back to the cache instead of a cudaFree (which would wait for the whole device).
    cudaError_t grow(std::size_t b) {
        if (p && bytes >= b) return cudaSuccess;
        release();
        return ensure(b);
    }
    // (Re)allocate when the current block is smaller than b. Returns cudaSuccess or the error.
    cudaError_t ensure(std::size_t b) {
        if (p && bytes >= b) return cudaSuccess;
        reset();
        if (b == 0) return cudaSuccess;
        cudaError_t e = cache_alloc(&p, b, &bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            bytes = 0;
            (void)cudaGetLastError();
            return e;
        }
        return cudaSuccess;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

}  // namespace wk
