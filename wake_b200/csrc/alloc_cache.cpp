// Process-wide cache of device blocks (see DevMem in common.cuh).
//
// Blocks are kept per device in a size-ordered multimap. A request takes the
// smallest cached block that is at least as large and at most twice as large,
// else a fresh cudaMalloc of the request rounded up to 2 MiB (1 KiB below
// 1 MiB), so lattices of nearby sizes share blocks. When cudaMalloc runs out of
// memory the cache is emptied and the allocation retried once.
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "common.cuh"

namespace wk {

namespace {
std::mutex g_mu;
std::multimap<std::pair<int, std::size_t>, void*> g_free;  // (device, block bytes) -> block

std::size_t round_block(std::size_t b) {
    const std::size_t g = b >= (1u << 20) ? (std::size_t(2) << 20) : std::size_t(1024);
    return (b + g - 1) / g * g;
}

std::size_t trim_locked(int dev) {
    std::size_t freed = 0;
    for (auto it = g_free.begin(); it != g_free.end();) {
        if (it->first.first == dev) {
            cudaFree(it->second);
            freed += it->first.second;
            it = g_free.erase(it);
        } else {
            ++it;
        }
    }
    return freed;
}
}  // namespace

cudaError_t cache_alloc(void** p, std::size_t bytes, std::size_t* block_bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const std::size_t want = round_block(bytes);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_free.lower_bound({dev, want});
        if (it != g_free.end() && it->first.first == dev && it->first.second <= 2 * want) {
            *p = it->second;
            *block_bytes = it->first.second;
            g_free.erase(it);
            return cudaSuccess;
        }
    }
    e = cudaMalloc(p, want);
    if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        {
            std::lock_guard<std::mutex> lk(g_mu);
            trim_locked(dev);
        }
        e = cudaMalloc(p, want);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    *block_bytes = want;
    return cudaSuccess;
}

void cache_release(void* p, std::size_t block_bytes) {
    if (!p) return;
    cudaPointerAttributes a{};
    int dev = 0;
    if (cudaPointerGetAttributes(&a, p) == cudaSuccess) dev = a.device;
    else (void)cudaGetLastError();
    std::lock_guard<std::mutex> lk(g_mu);
    g_free.emplace(std::make_pair(dev, block_bytes), p);
}

std::size_t cache_trim() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lk(g_mu);
    return trim_locked(dev);
}

std::size_t cache_held_bytes() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lk(g_mu);
    std::size_t s = 0;
    for (const auto& kv : g_free)
        if (kv.first.first == dev) s += kv.first.second;
    return s;
}

}  // namespace wk

extern "C" {

long long wake_gpu_cache_trim(void) { return static_cast<long long>(wk::cache_trim()); }
long long wake_gpu_cache_bytes(void) { return static_cast<long long>(wk::cache_held_bytes()); }

}  // extern "C"
