// tcgen05.cuh - sm_100a building blocks shared by the tensor-core kernels:
// mbarrier waits bounded by %globaltimer, TMA 2-D tile loads (no multicast),
// SWIZZLE_128B K-major UMMA descriptors, tcgen05.mma kind::f16 issue and
// commit, TMEM loads, and the host-side tensor-map encoder.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <mutex>

#include "common.cuh"

namespace umapb {
namespace tc {

constexpr int kBK = 64;                        // bf16 columns per k-block (one 128-byte row)
constexpr int kUK = 16;                        // K of one tcgen05.mma kind::f16
constexpr uint64_t kWaitNs = 2000000000ull;    // 2 s bound on every wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c,
                                             uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c),
                 "r"(d)
                 : "memory");
}

__device__ __forceinline__ float ld_shared_f32(uint32_t addr) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred P1;\n mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n"
        " selp.b32 %0, 1, 0, P1;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait with a suspend-time hint: the thread sleeps in hardware until the
// phase completes or the hint elapses, instead of spinning on issue slots.
__device__ __forceinline__ bool mbar_try_suspend(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred P1;\n mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n"
        " selp.b32 %0, 1, 0, P1;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after kWaitNs or when another role aborted.  Each try
// suspends for at most 1 ms, so the deadline and the abort flag are checked
// at least that often.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true) {
        if (mbar_try_suspend(bar, parity, 1000000u)) return true;
        if (*abort_flag) return false;
        if (global_ns() - t0 > kWaitNs) return false;
    }
}

// 2-D tile load of this GPU's memory into this CTA's shared memory.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// K-major SWIZZLE_128B operand descriptor: LBO = 16 B, SBO = 1024 B (8 rows of
// 128 B), descriptor version 1, layout type 2.  Advancing K by 16 bf16 inside
// the 128-byte swizzle row adds 2 (32 B in 16-byte units) to the address.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    uint64_t d = static_cast<uint64_t>((saddr & 0x3FFFF) >> 4);
    d |= static_cast<uint64_t>(1) << 16;
    d |= static_cast<uint64_t>(1024 >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(2) << 61;
    return d;
}

// K-major operand descriptor of a narrow k-block whose rows are `row_bytes`
// = 32 or 64 bytes (16 or 32 FP16 columns) with the matching TMA swizzle:
// SBO = 8 rows, layout type 6 (SWIZZLE_32B) or 4 (SWIZZLE_64B).  The tile's
// base must be aligned to the swizzle's 256- or 512-byte period.
__device__ __forceinline__ uint64_t desc_narrow(uint32_t saddr, int row_bytes) {
    uint64_t d = static_cast<uint64_t>((saddr & 0x3FFFF) >> 4);
    d |= static_cast<uint64_t>(1) << 16;
    d |= static_cast<uint64_t>((8 * row_bytes) >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(row_bytes == 32 ? 6 : 4) << 61;
    return d;
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both
// K-major, shape M x N.
constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

// kind::f16 instruction descriptor: F32 accumulate, FP16 A and B (format
// code 0 in both operand fields), both K-major, shape M x N.
constexpr uint32_t idesc_f16(int m, int n) {
    return (1u << 4) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                          uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

// Arrives on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Whole-warp TMEM allocation of `cols` columns; the base address is written
// to shared memory at `holder`.
__device__ __forceinline__ void tmem_alloc(uint32_t holder, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(holder),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols)
                 : "memory");
}

#define UMAPB_R8(i) "=r"(r[i]), "=r"(r[i + 1]), "=r"(r[i + 2]), "=r"(r[i + 3]), \
                    "=r"(r[i + 4]), "=r"(r[i + 5]), "=r"(r[i + 6]), "=r"(r[i + 7])

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];"
        : UMAPB_R8(0), UMAPB_R8(8), UMAPB_R8(16), UMAPB_R8(24)
        : "r"(taddr));
}

#undef UMAPB_R8

__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ----------------------------------------------------------------- host --
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeFn encoder() {
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    if (!fn) throw Error(UMAPB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    return fn;
}

// Tensor map over a row-major bf16 matrix of `rows` x `cols` (cols a multiple
// of 64, base 16-byte aligned) with box {64 columns, box_rows rows} and the
// 128-byte swizzle; rows past the end read as zero.
inline CUtensorMap make_bf16_map(const void* base, int64_t rows, int64_t cols, int box_rows) {
    if (cols % kBK != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0)
        throw Error(UMAPB_ERR_CUDA, "tensor map operand is not 64-column / 16-byte aligned");
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base),
                                 dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(UMAPB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

// Tensor map over a row-major FP16 matrix of `rows` x `cols` (cols a
// multiple of 16 and at least 64, base 16-byte aligned) with box {64 columns,
// box_rows rows} and the 128-byte swizzle.  Columns and rows past the end
// read as zero, so the last 64-column block of a row may be partial.
inline CUtensorMap make_f16_map(const void* base, int64_t rows, int64_t cols, int box_rows) {
    if (cols % 16 != 0 || cols < kBK || (reinterpret_cast<uintptr_t>(base) & 15) != 0 ||
        box_rows < 1 || box_rows > 256)
        throw Error(UMAPB_ERR_CUDA, "tensor map operand is not 16-column / 16-byte aligned");
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base),
                                 dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(UMAPB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

// Tensor map over the same FP16 matrix for its last, narrow k-block: box
// {tail_cols, box_rows} at the matching swizzle (16 columns = 32 bytes:
// SWIZZLE_32B; 32 columns: SWIZZLE_64B), rows past the end read as zero.
// The box starts at column cols - tail_cols, which the caller keeps a
// multiple of 64.
inline CUtensorMap make_f16_tail_map(const void* base, int64_t rows, int64_t cols, int tail_cols,
                                     int box_rows) {
    if ((tail_cols != 16 && tail_cols != 32) || cols % 16 != 0 || cols < tail_cols ||
        (reinterpret_cast<uintptr_t>(base) & 15) != 0 || box_rows < 1 || box_rows > 256)
        throw Error(UMAPB_ERR_CUDA, "narrow tensor map: unsupported tail width or alignment");
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(tail_cols),
                               static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encoder()(
        &m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
        CU_TENSOR_MAP_INTERLEAVE_NONE,
        tail_cols == 16 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B,
        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(UMAPB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

// True on sm_100 devices (the tcgen05 kernels are built for sm_100a only).
inline bool device_is_sm100() {
    int dev = 0, major = 0, minor = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    return major == 10 && minor == 0;
}

}  // namespace tc
}  // namespace umapb
