// common.cuh - shared host/device helpers of libumapb200.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/umapb200.h"

namespace umapb {

extern std::atomic<unsigned long long> g_kernel_launches;

// A failed call carries a umapb_status and the user-facing message.
struct Error : public std::runtime_error {
    int32_t status;
    Error(int32_t s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] inline void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e),
                  cudaGetErrorString(e), what, file, line);
    const int32_t st =
        (e == cudaErrorMemoryAllocation) ? UMAPB_ERR_OUT_OF_MEMORY : UMAPB_ERR_CUDA;
    throw Error(st, buf);
}

#define UMAPB_CUDA(call)                                                          \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) ::umapb::throw_cuda(e_, #call, __FILE__, __LINE__); \
    } while (0)

// Kernel launches issued by this library (cub primitives excluded); every
// launch site is followed by UMAPB_LAUNCH_CHECK(), which counts it.

#define UMAPB_LAUNCH_CHECK()                                                     \
    do {                                                                         \
        ::umapb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);      \
        UMAPB_CUDA(cudaGetLastError());                                          \
    } while (0)

[[noreturn]] inline void invalid(const std::string& msg) {
    throw Error(UMAPB_ERR_INVALID_PARAMETER, "invalid parameter: " + msg);
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Blocks released by DevBuf are kept per (device, stream, exact size) and
// handed to the next request of that size on that stream, in stream order.
// A fit asks for the same sizes in the same order every time, so repeated
// fits of one size make no allocator call: a pool allocation, even one served
// from memory the pool already holds, occasionally took most of a second on
// a shared machine.  At most kBlockCacheBytes are kept (a 1M-query transform
// beside a 1M-row fit cycles several GB); a block that would go beyond
// returns to the device's stream-ordered pool (cudaFreeAsync on its own
// stream).  Blocks of a stream that is gone stay until the process ends,
// within the same limit.  An allocation the pool cannot serve returns every
// block kept for the device and is tried once more.
constexpr size_t kBlockCacheBytes = static_cast<size_t>(32) << 30;

struct BlockCache {
    std::mutex mu;
    std::map<std::tuple<int, cudaStream_t, size_t>, std::vector<void*>> free_blocks;
    size_t held = 0;
    static BlockCache& get() {
        static BlockCache c;
        return c;
    }
};

inline void* dev_alloc(size_t bytes, cudaStream_t s, int* dev_out) {
    int dev = 0;
    cudaGetDevice(&dev);
    *dev_out = dev;
    BlockCache& c = BlockCache::get();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.free_blocks.find(std::make_tuple(dev, s, bytes));
        if (it != c.free_blocks.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            c.held -= bytes;
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, s);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // clear the failed request's error
        std::vector<void*> blocks;
        {
            std::lock_guard<std::mutex> lk(c.mu);
            for (auto it = c.free_blocks.begin(); it != c.free_blocks.end();) {
                if (std::get<0>(it->first) == dev) {
                    c.held -= std::get<2>(it->first) * it->second.size();
                    blocks.insert(blocks.end(), it->second.begin(), it->second.end());
                    it = c.free_blocks.erase(it);
                } else {
                    ++it;
                }
            }
        }
        if (!blocks.empty()) {
            // their streams may be gone: wait for the device, then free directly
            cudaDeviceSynchronize();
            for (void* b : blocks) cudaFree(b);
            e = cudaMallocAsync(&p, bytes, s);
        }
    }
    if (e != cudaSuccess) throw_cuda(e, "cudaMallocAsync", __FILE__, __LINE__);
    return p;
}

inline void dev_free(void* p, size_t bytes, cudaStream_t s, int dev) {
    BlockCache& c = BlockCache::get();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.held + bytes <= kBlockCacheBytes) {
            c.free_blocks[std::make_tuple(dev, s, bytes)].push_back(p);
            c.held += bytes;
            return;
        }
    }
    cudaFreeAsync(p, s);
}

// Returns the blocks kept for stream `s` to the pool; called before the
// stream is destroyed (its work has finished).
inline void dev_release_stream(cudaStream_t s) {
    std::vector<void*> blocks;
    BlockCache& c = BlockCache::get();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        for (auto it = c.free_blocks.begin(); it != c.free_blocks.end();) {
            if (std::get<1>(it->first) == s) {
                c.held -= std::get<2>(it->first) * it->second.size();
                blocks.insert(blocks.end(), it->second.begin(), it->second.end());
                it = c.free_blocks.erase(it);
            } else {
                ++it;
            }
        }
    }
    for (void* p : blocks) cudaFreeAsync(p, s);
}

// Stream-ordered device buffer on the block cache above (backed by the
// device's default memory pool, cudaMallocAsync).
template <typename T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;
    cudaStream_t stream = nullptr;
    int device = 0;

    DevBuf() = default;
    DevBuf(size_t n, cudaStream_t s) { alloc(n, s); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), count(o.count), stream(o.stream), device(o.device) {
        o.ptr = nullptr;
        o.count = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            count = o.count;
            stream = o.stream;
            device = o.device;
            o.ptr = nullptr;
            o.count = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }

    void alloc(size_t n, cudaStream_t s) {
        release();
        stream = s;
        count = n;
        if (n > 0) ptr = static_cast<T*>(dev_alloc(n * sizeof(T), s, &device));
    }
    void release() {
        if (ptr) dev_free(ptr, count * sizeof(T), stream, device);
        ptr = nullptr;
        count = 0;
    }
    T* get() const { return ptr; }
    size_t bytes() const { return count * sizeof(T); }
};

// ------------------------------------------------------------- device ---

// Order key of a kNN candidate: (distance, index) compared lexicographically,
// valid for non-negative finite or +inf distances (all distances produced on
// this path).  Equals the reference's neighbor_cmp order
// (rust_umap/src/lib.rs:2768-2772) as a single unsigned comparison.
__host__ __device__ inline uint64_t knn_key(float d, uint32_t idx) {
#ifdef __CUDA_ARCH__
    const uint32_t b = __float_as_uint(d);
#else
    uint32_t b;
    std::memcpy(&b, &d, 4);
#endif
    return (static_cast<uint64_t>(b) << 32) | idx;
}

__host__ __device__ inline float key_dist(uint64_t key) {
    const uint32_t b = static_cast<uint32_t>(key >> 32);
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    std::memcpy(&f, &b, 4);
    return f;
#endif
}

__host__ __device__ inline uint32_t key_index(uint64_t key) {
    return static_cast<uint32_t>(key & 0xffffffffu);
}

// Counter-based random numbers: SplitMix64 finaliser over a combined
// (seed, stream, counter) word.  Every consumer derives its stream id from
// what it processes (edge, epoch, sample), so results do not depend on the
// launch shape.
__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__host__ __device__ inline uint64_t rng_word(uint64_t seed, uint64_t a, uint64_t b) {
    return mix64(mix64(seed ^ mix64(a)) ^ b);
}

// Uniform integer in [0, n) from a 64-bit word (multiply-high reduction).
__host__ __device__ inline uint32_t rng_below(uint64_t word, uint32_t n) {
    return static_cast<uint32_t>(((word >> 32) * static_cast<uint64_t>(n)) >> 32);
}

// Uniform integer in [0, n) from 32 random bits (multiply-high reduction).
__host__ __device__ inline uint32_t rng_below32(uint32_t word, uint32_t n) {
    return static_cast<uint32_t>((static_cast<uint64_t>(word) * n) >> 32);
}

// Uniform float in [0, 1) from 24 random bits.
__host__ __device__ inline float rng_unit_f32(uint64_t word) {
    return static_cast<float>(word >> 40) * (1.0f / 16777216.0f);
}

__host__ __device__ inline double rng_unit_f64(uint64_t word) {
    return static_cast<double>(word >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace umapb
