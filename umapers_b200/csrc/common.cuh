// common.cuh - shared host/device helpers of libumapb200.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

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

// Stream-ordered device buffer.  Memory comes from the device's default
// memory pool (cudaMallocAsync), which keeps freed blocks cached so repeated
// fits of the same size do not go back to the driver.
template <typename T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;
    cudaStream_t stream = nullptr;

    DevBuf() = default;
    DevBuf(size_t n, cudaStream_t s) { alloc(n, s); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), count(o.count), stream(o.stream) {
        o.ptr = nullptr;
        o.count = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            count = o.count;
            stream = o.stream;
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
        if (n > 0) UMAPB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ptr), n * sizeof(T), s));
    }
    void release() {
        if (ptr) cudaFreeAsync(ptr, stream);
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

// Uniform float in [0, 1) from 24 random bits.
__host__ __device__ inline float rng_unit_f32(uint64_t word) {
    return static_cast<float>(word >> 40) * (1.0f / 16777216.0f);
}

__host__ __device__ inline double rng_unit_f64(uint64_t word) {
    return static_cast<double>(word >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace umapb
