// knn_tc.cu - exact kNN through tcgen05 tensor-core distance tiles.
//
// Replaces exact_nearest_neighbors{,_to_reference} (rust_umap/src/lib.rs:
// 2863-2928, 3346-3399) for euclidean rows with the same result as the
// reference, bit for bit, in three steps:
//
// 1. prep: every row x becomes two BF16 operand rows of K' (a multiple of 64)
//    columns.  With h = bf16(x), l = bf16(x - h), n = |x|^2 (FP32):
//        A = [-2h | -2h | -2l | split3((1-c2) n) | 1 1 1 | bf16(-c1 sqrt n) | 0...]
//        B = [  h |   l |   h | 1 1 1 | split3((1-c2) n) | bf16(sqrt n)     | 0...]
//    so one GEMM gives L_ij = n_i + n_j - 2 x_i.x_j - e_ij, a certified lower
//    bound of the reference's FP32 squared distance d_ij, where
//    e_ij = c1 sqrt(n_i n_j) + c2 (n_i + n_j) bounds the BF16 split error
//    (3.02 * 2^-16 per product, doubled), the FP32 accumulation of K' terms,
//    and the reference's own FP32 rounding (see kBoundC1/kBoundC2 below).
// 2. tc_knn_kernel: a persistent, warp-specialised tcgen05 kernel.  A CTA
//    keeps MT query tiles of 128 rows of A resident in shared memory, streams
//    128-row candidate tiles of B through a TMA ring (SWIZZLE_128B, no
//    multicast), and one thread issues tcgen05.mma (kind::f16, BF16 in, FP32
//    accumulate) into double-buffered TMEM accumulators.  Eight epilogue
//    warps per query tile each own 32 rows x 64 columns of the accumulator:
//    they read it with tcgen05.ld and keep, per (row, column half), the
//    S = 32 smallest (L, index) keys in a global list.  A per-list threshold
//    skips a row's 64 columns with one vote in the common case; otherwise the
//    row's values are transposed across the warp through a shared-memory
//    scratch and its qualifying keys are inserted cooperatively (one list
//    entry per lane), while the next pending row's list is already being
//    loaded.  When the query tiles are fewer than the SMs, the candidate
//    tiles are split too (one wave of units), with lists per split.  A self
//    kNN over at least one wave of query groups first regroups its rows by
//    nearest pivot ("cell order" below), and each group starts its candidate
//    walk at its own cell, so the lists fill with near candidates first.
// 3. rerank: one warp per row recomputes exact FP32 distances in the
//    reference's summation order and keeps the k smallest (distance, index)
//    keys.  With U_j = L_j + 2 e_j and B the smallest largest-L of the full
//    lists, every candidate missing from the lists has d >= B, so the row is
//    certified when at least k candidates have U < B.  Only listed candidates
//    with L <= T, T the k-th smallest U, can rank in the top k, so only they
//    are recomputed.  Rows that fail (near-ties wider than the bound) are
//    recomputed by knn_plain.
//
// Every wait on an mbarrier is bounded by a %globaltimer deadline; a timeout
// sets an error word, stops all roles, drains in-flight copies and frees TMEM.
#include <cub/cub.cuh>
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "kernels.cuh"
#include "tcgen05.cuh"

namespace umapb {
namespace {

using namespace tc;

constexpr int BM = 128;     // query rows per tile (UMMA M)
constexpr int BN = 128;     // candidate rows per tile (UMMA N)
constexpr int BK = kBK;     // bf16 columns per k-block (one 128-byte swizzle row)
constexpr int UK = kUK;     // K of one tcgen05.mma kind::f16
constexpr int S = 32;       // shortlist length per row
constexpr int kTileBytes = BM * BK * 2;  // 16 KiB
constexpr int kBarBytes = 256;           // mbarriers, TMEM address, abort flag
constexpr int kScratchBytes = 256;       // per epilogue warp: one row's 64 values
constexpr uint32_t kIdesc = idesc_bf16(BM, BN);

// Bound constants (see header comment).  c1 covers the split products
// (2 * 3.02 * 2^-16) with 2% slack for the BF16 rounding of the bound term;
// c2 = (K' + D + 8) * 2^-22 covers the FP32 accumulation of the GEMM and the
// FP32 rounding of the norms and of the reference distance.
constexpr double kBoundC1 = 1.02 * 2.0 * 3.02 / 65536.0;

inline int padded_k(int d) { return ((3 * d + 7 + BK - 1) / BK) * BK; }
inline double bound_c2(int d) { return (padded_k(d) + d + 8) * std::ldexp(1.0, -22); }

// order-preserving map of a float to uint32 (negative values included)
__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return (o & 0x80000000u) ? __uint_as_float(o & 0x7FFFFFFFu) : __uint_as_float(~o);
}

__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Minimum of 32 FP32 values held as bit patterns (16 three-input mins).
__device__ __forceinline__ float min32(const uint32_t* r) {
    float m = min3f(__uint_as_float(r[0]), __uint_as_float(r[1]), __uint_as_float(r[2]));
#pragma unroll
    for (int j = 3; j < 31; j += 2) m = min3f(m, __uint_as_float(r[j]), __uint_as_float(r[j + 1]));
    return fminf(m, __uint_as_float(r[31]));
}

// Bitonic sort of one value per lane, ascending with the lane index.
template <typename T>
__device__ __forceinline__ T warp_sort_asc(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const T o = __shfl_xor_sync(0xffffffffu, v, stride);
            const bool up = (lane & size) == 0;
            const bool lower = (lane & stride) == 0;
            v = (lower == up) ? (v < o ? v : o) : (v < o ? o : v);
        }
    }
    return v;
}

// Merges 32 keys (one per lane, any order) into a list sorted ascending
// across the lanes and keeps the 32 smallest: sort the keys, reverse them,
// take the lane-wise minimum (a bitonic sequence holding the 32 smallest of
// both) and sort that with five compare-exchange stages.
__device__ __forceinline__ uint64_t warp_merge_keys(uint64_t list, uint64_t keys) {
    const int lane = threadIdx.x & 31;
    const uint64_t srt = warp_sort_asc<uint64_t>(keys);
    const uint64_t rev = __shfl_sync(0xffffffffu, srt, 31 - lane);
    uint64_t m = list < rev ? list : rev;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
        const uint64_t o = __shfl_xor_sync(0xffffffffu, m, st);
        m = (lane & st) ? (m > o ? m : o) : (m < o ? m : o);
    }
    return m;
}

// A chunk with at least this many qualifying keys is merged in one bitonic
// pass instead of key by key (about 6 sequential insertions cost as much).
constexpr int kBulkMergeMin = 6;

// CTAs begin their candidate range at staggered tiles (16 groups, 4 tiles
// apart: a window of 4 MiB of B at K' = 256, L2-resident) so they do not all
// request the same tile at once.  The shortlist certificate does not depend
// on the visiting order.
constexpr int32_t kStaggerGroups = 16, kStaggerStep = 4;

struct TcArgs {
    int64_t n_q;
    int64_t n_r;
    int kb;          // k-blocks of 64 columns
    int64_t n_units;      // work units: (group of MT query tiles, candidate split)
    int n_split;          // candidate splits per group (1 unless query tiles are few)
    int64_t split_tiles;  // candidate tiles per split (the last split may hold fewer)
    int64_t n_ctiles;     // candidate tiles
    uint64_t* lists;      // n_q x n_split x 2 x S keys (L order-mapped << 32 | index), one
                          // list per (row, candidate split, half of each tile's columns)
    const int32_t* start_tile;  // per query group, the first candidate tile to visit (rows in
                                // cell order, one split), or null for the staggered start
    int* err;
};

// Work unit u covers query group u / n_split and the candidate tiles of
// split u % n_split, visited from tile begin + rot onwards (cyclically).
// With rows in cell order a group starts at its own cell's first tile.
struct Unit {
    int32_t group, split, begin, len, rot;  // tile counts stay far below 2^31
};
__device__ __forceinline__ Unit unit_of(const TcArgs& p, int64_t u) {
    Unit r;
    r.group = static_cast<int32_t>(u / p.n_split);
    r.split = static_cast<int32_t>(u - static_cast<int64_t>(r.group) * p.n_split);
    r.begin = r.split * static_cast<int32_t>(p.split_tiles);
    r.len = static_cast<int32_t>(min(p.split_tiles, p.n_ctiles - r.begin));
    r.rot = p.start_tile != nullptr ? p.start_tile[r.group]
                                    : static_cast<int32_t>(blockIdx.x % kStaggerGroups) * kStaggerStep;
    if (r.rot >= r.len || r.rot < 0) r.rot = 0;
    return r;
}

// Candidate tile visited at step t of unit w.
__device__ __forceinline__ int32_t tile_at(int32_t t, const Unit& w) {
    const int32_t c = t + w.rot;
    return w.begin + (c >= w.len ? c - w.len : c);
}

constexpr uint32_t kTileDesc = kTileBytes >> 4;  // one 16 KiB tile in descriptor units

// Threads: warp 0 TMA, warp 1 MMA, then 8 epilogue warps per query tile.
template <int MT>
constexpr int tc_threads() { return 64 + 256 * MT; }

template <int MT, int ST>
__global__ void __launch_bounds__(tc_threads<MT>(), 1)
    tc_knn_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                  TcArgs p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int KB = p.kb;
    const uint32_t sA = smem_u32(smem);
    const uint32_t sB = sA + MT * KB * kTileBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + MT * KB * kTileBytes + ST * kTileBytes);
    const uint32_t b_full = smem_u32(bars);
    const uint32_t b_empty = b_full + 8 * ST;
    const uint32_t b_tfull = b_empty + 8 * ST;
    const uint32_t b_tempty = b_tfull + 16;
    const uint32_t b_afull = b_tempty + 16;
    const uint32_t b_aempty = b_afull + 8;
    const uint32_t b_final = b_aempty + 8;
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(bars + 2 * ST + 7);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr uint32_t kTmemCols = MT == 2 ? 512 : 256;

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(b_full + 8 * s, 1);
            mbar_init(b_empty + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(b_tfull + 8 * b, 1);
            mbar_init(b_tempty + 8 * b, 8 * MT);
        }
        mbar_init(b_afull, 1);
        mbar_init(b_aempty, 1);
        mbar_init(b_final, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmem_holder), kTmemCols);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_holder;

    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicCAS(p.err, 0, code);
    };

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            uint64_t it = 0;
            int64_t u_iter = 0;
            for (int64_t unit = blockIdx.x; unit < p.n_units && !*abort_flag;
                 unit += gridDim.x, ++u_iter) {
                if (u_iter > 0 && !mbar_wait(b_aempty, static_cast<uint32_t>((u_iter - 1) & 1),
                                             abort_flag)) {
                    fail(1);
                    break;
                }
                const Unit w = unit_of(p, unit);
                mbar_expect_tx(b_afull, MT * KB * kTileBytes);
                for (int mt = 0; mt < MT; ++mt)
                    for (int kb = 0; kb < KB; ++kb)
                        tma_load_2d(sA + (mt * KB + kb) * kTileBytes, &tmA, b_afull, kb * BK,
                                    static_cast<int>((w.group * MT + mt) * BM));
                bool ok = true;
                for (int32_t c = 0; c < w.len && ok; ++c) {
                    for (int kb = 0; kb < KB; ++kb, ++it) {
                        const int stage = static_cast<int>(it % ST);
                        const uint32_t round = static_cast<uint32_t>(it / ST);
                        if (!mbar_wait(b_empty + 8 * stage, (round & 1) ^ 1, abort_flag)) {
                            fail(2);
                            ok = false;
                            break;
                        }
                        mbar_expect_tx(b_full + 8 * stage, kTileBytes);
                        tma_load_2d(sB + stage * kTileBytes, &tmB, b_full + 8 * stage, kb * BK,
                                    static_cast<int>(tile_at(c, w) * BN));
                    }
                }
                if (!ok) break;
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------- MMA issuer
        if (lane == 0) {
            uint64_t it = 0, cg = 0;
            int64_t u_iter = 0;
            bool ok = true;
            // ring-stage descriptors advance by address / 16
            const uint64_t dB0 = desc_sw128(sB);
            for (int64_t unit = blockIdx.x; unit < p.n_units && ok; unit += gridDim.x, ++u_iter) {
                if (!mbar_wait(b_afull, static_cast<uint32_t>(u_iter & 1), abort_flag)) {
                    fail(3);
                    break;
                }
                fence_after();
                const int32_t len = unit_of(p, unit).len;
                for (int32_t c = 0; c < len && ok; ++c, ++cg) {
                    const uint32_t buf = static_cast<uint32_t>(cg & 1);
                    if (!mbar_wait(b_tempty + 8 * buf, static_cast<uint32_t>(((cg >> 1) & 1) ^ 1),
                                   abort_flag)) {
                        fail(4);
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t dcol = tmem_base + buf * (MT * BN);
                    for (int kb = 0; kb < KB; ++kb, ++it) {
                        const int stage = static_cast<int>(it % ST);
                        if (!mbar_wait(b_full + 8 * stage, static_cast<uint32_t>((it / ST) & 1),
                                       abort_flag)) {
                            fail(5);
                            ok = false;
                            break;
                        }
                        fence_after();
                        // All four k-steps of every k-block, the zero columns past
                        // 3d + 7 included (they add exact zeros): a loop of constant
                        // trip count keeps the tensor pipe fed, skipping them does not.
                        const uint64_t db0 = dB0 + static_cast<uint64_t>(stage) * kTileDesc;
#pragma unroll
                        for (int ks = 0; ks < BK / UK; ++ks) {
#pragma unroll
                            for (int mt = 0; mt < MT; ++mt) {
                                const uint64_t da =
                                    desc_sw128(sA + (mt * KB + kb) * kTileBytes) + 2 * ks;
                                umma_bf16(dcol + mt * BN, da, db0 + 2 * ks, kIdesc,
                                          (kb | ks) != 0 ? 1u : 0u);
                            }
                        }
                        umma_commit(b_empty + 8 * stage);
                    }
                    if (ok) umma_commit(b_tfull + 8 * buf);
                }
                if (ok) umma_commit(b_aempty);
            }
            // every MMA issued by this thread has completed before TMEM is freed
            umma_commit(b_final);
            mbar_wait(b_final, 0, abort_flag);
        }
    } else {
        // --------------------------------------------------- epilogue
        // Warp w reads TMEM lanes 32 * (w % 4) (hardware rule); the four warps
        // of each quarter split (query tile, column half).
        const int quarter = warp & 3;
        const int slot = (warp - 2) >> 2;
        const int mt = slot >> 1;
        const int half = slot & 1;
        const uint32_t scratch = b_full + kBarBytes + (warp - 2) * kScratchBytes;
        uint64_t cg = 0;
        bool ok = true;
        for (int64_t unit = blockIdx.x; unit < p.n_units && ok; unit += gridDim.x) {
            const Unit w = unit_of(p, unit);
            const int32_t row = (w.group * MT + mt) * BM + quarter * 32 + lane;
            const bool row_ok = row < p.n_q;
            const int32_t list_base = w.split * 2 + half;  // list of (row, split, half)
            auto list_of = [&](int32_t srow) {
                return p.lists + (static_cast<int64_t>(srow) * 2 * p.n_split + list_base) * S;
            };
            float tau = INFINITY;  // this list's current S-th smallest bound
            for (int32_t c = 0; c < w.len; ++c, ++cg) {
                const uint32_t buf = static_cast<uint32_t>(cg & 1);
                if (!mbar_wait(b_tfull + 8 * buf, static_cast<uint32_t>((cg >> 1) & 1), abort_flag)) {
                    fail(6);
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                       buf * (MT * BN) + mt * BN + half * (BN / 2);
                uint32_t r[2][32];
                tmem_ld32(taddr, r[0]);
                tmem_ld32(taddr + 32, r[1]);
                tmem_wait_ld();
                // the accumulator buffer can be overwritten as soon as it is in registers
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(b_tempty + 8 * buf);
                const float m0 = min32(r[0]), m1 = min32(r[1]);
                unsigned pend = __ballot_sync(0xffffffffu, row_ok && fminf(m0, m1) < tau);
                if (pend == 0) continue;
                const int32_t colh = tile_at(c, w) * BN + half * (BN / 2);
                const int32_t valid_cols = static_cast<int32_t>(p.n_r - colh);
                // Rows are served one at a time; the next pending row's list is
                // loaded while the current one is merged, hiding its L2 latency.
                int src = __ffs(pend) - 1;
                uint64_t* lst = list_of(__shfl_sync(0xffffffffu, row, src));
                uint64_t lk_next = lst[lane];
                while (pend) {
                    pend &= pend - 1;
                    const int cur = src;
                    uint64_t* cur_lst = lst;
                    uint64_t lk = lk_next;
                    if (pend) {
                        src = __ffs(pend) - 1;
                        lst = list_of(__shfl_sync(0xffffffffu, row, src));
                        lk_next = lst[lane];
                    }
                    // transpose through the warp's scratch: lane j takes
                    // columns j and 32 + j of the source row
                    if (lane == cur) {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            st_shared_v4(scratch + 16 * j, r[j >> 3][(j & 7) * 4],
                                         r[j >> 3][(j & 7) * 4 + 1], r[j >> 3][(j & 7) * 4 + 2],
                                         r[j >> 3][(j & 7) * 4 + 3]);
                    }
                    __syncwarp();
                    const float v0 = ld_shared_f32(scratch + 4 * lane);
                    const float v1 = ld_shared_f32(scratch + 4 * (32 + lane));
                    __syncwarp();
                    float stau = __shfl_sync(0xffffffffu, tau, cur);
#pragma unroll
                    for (int ch = 0; ch < 2; ++ch) {
                        const float mine = ch == 0 ? v0 : v1;
                        const bool qual = mine < stau && lane + ch * 32 < valid_cols;
                        unsigned q = __ballot_sync(0xffffffffu, qual);
                        if (__popc(q) >= kBulkMergeMin) {
                            const uint64_t key =
                                qual ? (static_cast<uint64_t>(f2o(mine)) << 32) |
                                           static_cast<uint32_t>(colh + ch * 32 + lane)
                                     : ~0ull;
                            lk = warp_merge_keys(lk, key);
                            const uint64_t last = __shfl_sync(0xffffffffu, lk, S - 1);
                            stau = last == ~0ull ? INFINITY : o2f(static_cast<uint32_t>(last >> 32));
                            q = 0;
                        }
                        while (q) {
                            const int b = __ffs(q) - 1;
                            q &= q - 1;
                            const float val = __shfl_sync(0xffffffffu, mine, b);
                            if (!(val < stau)) continue;
                            const uint64_t key = (static_cast<uint64_t>(f2o(val)) << 32) |
                                                 static_cast<uint32_t>(colh + ch * 32 + b);
                            const int pos = __popc(__ballot_sync(0xffffffffu, lk < key));
                            const uint64_t up = __shfl_up_sync(0xffffffffu, lk, 1);
                            if (lane > pos)
                                lk = up;
                            else if (lane == pos)
                                lk = key;
                            const uint64_t last = __shfl_sync(0xffffffffu, lk, S - 1);
                            stau = last == ~0ull ? INFINITY : o2f(static_cast<uint32_t>(last >> 32));
                        }
                    }
                    cur_lst[lane] = lk;
                    if (lane == cur) tau = stau;
                }
            }
        }
    }

    __syncthreads();
    if (*abort_flag) {
        // let copies already in flight land before the CTA's shared memory goes away
        const uint64_t t0 = global_ns();
        while (global_ns() - t0 < 2000000ull) {
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        tmem_dealloc(tmem_base, kTmemCols);
    }
}

// ------------------------------------------------------------ operands --
__global__ void prep_kernel(const float* __restrict__ X, const float* __restrict__ sq, int64_t n,
                            int d, int kp, float c1, float c2, bool is_query,
                            __nv_bfloat16* __restrict__ out) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* x = X + row * d;
    __nv_bfloat16* o = out + row * kp;
    for (int c = lane; c < d; c += 32) {
        const float v = x[c];
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
        if (is_query) {
            const __nv_bfloat16 h2 = __float2bfloat16_rn(-2.0f * __bfloat162float(h));
            o[c] = h2;
            o[d + c] = h2;
            o[2 * d + c] = __float2bfloat16_rn(-2.0f * __bfloat162float(l));
        } else {
            o[c] = h;
            o[d + c] = l;
            o[2 * d + c] = h;
        }
    }
    for (int c = 3 * d + 7 + lane; c < kp; c += 32) o[c] = __float2bfloat16_rn(0.0f);
    if (lane == 0) {
        const float n2 = sq[row];
        const float v = (1.0f - c2) * n2;
        const __nv_bfloat16 s1 = __float2bfloat16_rn(v);
        const float r1 = v - __bfloat162float(s1);
        const __nv_bfloat16 s2 = __float2bfloat16_rn(r1);
        const __nv_bfloat16 s3 = __float2bfloat16_rn(r1 - __bfloat162float(s2));
        const __nv_bfloat16 one = __float2bfloat16_rn(1.0f);
        const float rn = sqrtf(n2);
        __nv_bfloat16* a = o + 3 * d;
        if (is_query) {
            a[0] = s1; a[1] = s2; a[2] = s3;
            a[3] = one; a[4] = one; a[5] = one;
            a[6] = __float2bfloat16_rn(-c1 * rn);
        } else {
            a[0] = one; a[1] = one; a[2] = one;
            a[3] = s1; a[4] = s2; a[5] = s3;
            a[6] = __float2bfloat16_rn(rn);
        }
    }
}

// ------------------------------------------------------------ re-rank ---
__device__ __forceinline__ float sqdist_ref(const float* __restrict__ x, const float* __restrict__ y,
                                            int d) {
    if (d >= 64) {
        float lane[8];
#pragma unroll
        for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
        int i = 0;
        if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0) {
            // the same operations in the same order, from 16-byte loads
            for (; i + 8 <= d; i += 8) {
                const float4 xa = *reinterpret_cast<const float4*>(x + i);
                const float4 xb = *reinterpret_cast<const float4*>(x + i + 4);
                const float4 ya = __ldg(reinterpret_cast<const float4*>(y + i));
                const float4 yb = __ldg(reinterpret_cast<const float4*>(y + i + 4));
                const float xs[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
                const float ys[8] = {ya.x, ya.y, ya.z, ya.w, yb.x, yb.y, yb.z, yb.w};
#pragma unroll
                for (int l = 0; l < 8; ++l) {
                    const float df = __fsub_rn(xs[l], ys[l]);
                    lane[l] = __fadd_rn(lane[l], __fmul_rn(df, df));
                }
            }
        }
        for (; i + 8 <= d; i += 8)
#pragma unroll
            for (int l = 0; l < 8; ++l) {
                const float df = __fsub_rn(x[i + l], y[i + l]);
                lane[l] = __fadd_rn(lane[l], __fmul_rn(df, df));
            }
        float s = lane[0];
#pragma unroll
        for (int l = 1; l < 8; ++l) s = __fadd_rn(s, lane[l]);
        for (; i < d; ++i) {
            const float df = __fsub_rn(x[i], y[i]);
            s = __fadd_rn(s, __fmul_rn(df, df));
        }
        return s;
    }
    float s = 0.0f;
    for (int i = 0; i < d; ++i) {
        const float df = __fsub_rn(x[i], y[i]);
        s = __fadd_rn(s, __fmul_rn(df, df));
    }
    return s;
}

__global__ void rerank_kernel(const float* __restrict__ Q, const float* __restrict__ R,
                              const float* __restrict__ qsq, const float* __restrict__ rsq,
                              const uint64_t* __restrict__ lists, int n_lists, int64_t n_q,
                              int d, int k, double c1, double c2,
                              const int32_t* __restrict__ perm, int32_t* __restrict__ out_idx,
                              float* __restrict__ out_dist, int* __restrict__ fb_count,
                              int32_t* __restrict__ fb_rows) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n_q) return;
    // rows in cell order (perm non-null): position -> original row; keys, outputs
    // and fallback rows use original indices, so ties break as in the reference
    const int64_t orow = perm != nullptr ? perm[row] : row;
    const uint64_t* rl = lists + row * n_lists * S;
    // The smallest bound a candidate missing from every list can have: a full
    // list left out only candidates with L >= its largest entry, a list that
    // is not full kept every candidate of its range.
    double bound = INFINITY;
    for (int h = 0; h < n_lists; ++h) {
        const uint64_t lk = rl[h * S + lane];
        const bool valid = lk != ~0ull;
        float lmax = valid ? o2f(static_cast<uint32_t>(lk >> 32)) : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
        if (__popc(__ballot_sync(0xffffffffu, valid)) == S)
            bound = fmin(bound, static_cast<double>(lmax));
    }
    // Upper bounds U = L + 2e (rounded up to FP32): `below` counts the
    // candidates with U < bound (k of them certify the row), and T is the k-th
    // smallest U.  A candidate with L > T has k others with d <= U <= T < L <= d
    // ahead of it, so only candidates with L <= T can rank in the top k: each
    // list (sorted by L) contributes a prefix, usually empty.
    const double nq = qsq[row];
    int below = 0;
    float topu = INFINITY;  // the 32 smallest U, sorted across the warp
    for (int h = 0; h < n_lists; ++h) {
        const uint64_t lk = rl[h * S + lane];
        const float l0 = o2f(static_cast<uint32_t>(__shfl_sync(0xffffffffu, lk, 0) >> 32));
        double U = INFINITY;
        if (lk != ~0ull) {
            const double nc = rsq[static_cast<uint32_t>(lk)];
            U = static_cast<double>(o2f(static_cast<uint32_t>(lk >> 32))) +
                2.0 * (c1 * sqrt(nq * nc) + c2 * (nq + nc));
        }
        below += __popc(__ballot_sync(0xffffffffu, U < bound));
        // a list whose smallest L already exceeds the k-th smallest U so far
        // cannot lower it
        if (!(l0 <= __shfl_sync(0xffffffffu, topu, k - 1))) continue;
        const float u = warp_sort_asc<float>(__double2float_ru(U));
        const float ur = __shfl_sync(0xffffffffu, u, 31 - lane);
        float m = fminf(topu, ur);
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
            const float o = __shfl_xor_sync(0xffffffffu, m, st);
            m = (lane & st) ? fmaxf(m, o) : fminf(m, o);
        }
        topu = m;
    }
    const float T = __shfl_sync(0xffffffffu, topu, k - 1);
    // Exact keys in the reference's order for the candidates with L <= T; the
    // 32 smallest are kept sorted across the warp (bitonic merge of each
    // list's keys into them).
    uint64_t top = ~0ull;
    for (int h = 0; h < n_lists; ++h) {
        const uint64_t lk = rl[h * S + lane];
        const bool take = lk != ~0ull && o2f(static_cast<uint32_t>(lk >> 32)) <= T;
        if (__ballot_sync(0xffffffffu, take) == 0) continue;
        uint64_t key = ~0ull;
        if (take) {
            const uint32_t j = static_cast<uint32_t>(lk);
            key = knn_key(sqdist_ref(Q + row * d, R + static_cast<int64_t>(j) * d, d),
                          perm != nullptr ? static_cast<uint32_t>(perm[j]) : j);
        }
        top = warp_merge_keys(top, key);
    }
    if (lane < k) {
        out_idx[orow * k + lane] = static_cast<int32_t>(key_index(top));
        out_dist[orow * k + lane] = __fsqrt_rn(key_dist(top));
    }
    if (below < k && lane == 0) fb_rows[atomicAdd(fb_count, 1)] = static_cast<int32_t>(orow);
}

// --------------------------------------------------------------- host ----
CUtensorMap make_map(const void* base, int64_t rows, int kp) {
    return make_bf16_map(base, rows, kp, BM);
}

int query_tiles_for(int kb) { return kb <= 4 ? 2 : (kb <= 10 ? 1 : 0); }

template <int MT, int ST>
void launch_tc(const CUtensorMap& ma, const CUtensorMap& mb, const TcArgs& a, cudaStream_t s) {
    // tiles + 1 KiB alignment slack + barriers/flags + epilogue scratch
    const size_t smem = static_cast<size_t>(MT * a.kb + ST) * kTileBytes + 1024 + kBarBytes +
                        static_cast<size_t>(8 * MT) * kScratchBytes;
    auto kern = tc_knn_kernel<MT, ST>;
    UMAPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    int dev = 0, sms = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t grid = std::min<int64_t>(a.n_units, sms);
    kern<<<static_cast<unsigned>(grid), tc_threads<MT>(), smem, s>>>(ma, mb, a);
    UMAPB_LAUNCH_CHECK();
}

// Work decomposition: groups of MT query tiles; when the groups are fewer
// than the SMs the candidate tiles are split too (at least 8 per split, and
// no more units than SMs, so every unit starts at once), so small query sets
// still occupy the GPU.
TcArgs plan(int64_t n_q, int64_t n_r, int d, bool allow_split) {
    const int kp = padded_k(d);
    TcArgs a{};
    a.n_q = n_q;
    a.n_r = n_r;
    a.kb = kp / BK;
    a.n_ctiles = ceil_div(n_r, BN);
    const int mt = query_tiles_for(a.kb);
    const int64_t groups = ceil_div(n_q, static_cast<int64_t>(BM) * mt);
    int64_t split = 1;
    if (allow_split) {
        int dev = 0, sms = 0;
        UMAPB_CUDA(cudaGetDevice(&dev));
        UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (groups < sms)
            split = std::min<int64_t>(std::max<int64_t>(sms / groups, 1),
                                      std::max<int64_t>(1, a.n_ctiles / 8));
    }
    a.split_tiles = ceil_div(a.n_ctiles, split);
    a.n_split = static_cast<int>(ceil_div(a.n_ctiles, a.split_tiles));
    a.n_units = groups * a.n_split;
    return a;
}

// ------------------------------------------------------------ cell order --
// A self kNN over at least one wave of query groups runs on its rows
// regrouped by cell.
// - Every row joins the nearest of C pivot rows (rows p * (n / C)).
// - The rows are stably sorted by cell.
// - Each query group starts its candidate walk at its own cell's first tile.
// The shortlists then fill with near candidates in the first tiles. Their
// thresholds drop early, and later tiles rarely hold a qualifying key.
// The groups of one wave start within a few hundred tiles of each other, so
// they still stream the candidate operand in step through L2.
// The result does not change: the certificate does not depend on the
// visiting order, and the re-rank maps positions back to original rows.
constexpr int kMaxCells = 256;
constexpr int64_t kCellPivotFloats = 16384;  // 64 KiB of pivots in shared memory

// Cells: 32, 64, 128 or 256, as many as keep at least 2,048 rows per cell
// (512 at 32 cells) and the pivots within 64 KiB; 0 = rows stay in order.
int cell_count(int64_t n, int d) {
    int c = kMaxCells;
    while (c > 32 && (c * static_cast<int64_t>(d) > kCellPivotFloats || c * int64_t{2048} > n))
        c >>= 1;
    if (c * static_cast<int64_t>(d) > kCellPivotFloats || c * int64_t{512} > n) return 0;
    return c;
}

// One warp per row: lane l scores pivots l + 32 q (q < PPL) from shared
// memory ([d][C], conflict-free), the row's values broadcast by shuffle, and
// the warp keeps the pivot with the smallest |p|^2 - 2 x.p (lower on ties).
template <int PPL>
__global__ void __launch_bounds__(256) cell_assign_kernel(const float* __restrict__ X, int64_t n,
                                                          int d, int64_t stride,
                                                          uint8_t* __restrict__ cell,
                                                          int32_t* __restrict__ iota) {
    constexpr int C = 32 * PPL;
    extern __shared__ float piv[];
    float* pn = piv + static_cast<int64_t>(d) * C;
    for (int i = threadIdx.x; i < C * d; i += blockDim.x) {
        const int pc = i / d, t = i - pc * d;
        piv[t * C + pc] = X[static_cast<int64_t>(pc) * stride * d + t];
    }
    __syncthreads();
    for (int pc = threadIdx.x; pc < C; pc += blockDim.x) {
        float sq = 0.0f;
        for (int t = 0; t < d; ++t) sq = fmaf(piv[t * C + pc], piv[t * C + pc], sq);
        pn[pc] = sq;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; row < n;
         row += warps) {
        const float* x = X + row * d;
        float acc[PPL];
#pragma unroll
        for (int q = 0; q < PPL; ++q) acc[q] = 0.0f;
        for (int t0 = 0; t0 < d; t0 += 32) {
            const float xv = t0 + lane < d ? x[t0 + lane] : 0.0f;
            const int tn = min(32, d - t0);
            for (int j = 0; j < tn; ++j) {
                const float xj = __shfl_sync(0xffffffffu, xv, j);
                const float* pr = piv + (t0 + j) * C + lane;
#pragma unroll
                for (int q = 0; q < PPL; ++q) acc[q] = fmaf(xj, pr[32 * q], acc[q]);
            }
        }
        float best = INFINITY;
        int bi = C;
#pragma unroll
        for (int q = 0; q < PPL; ++q) {
            const float sc = pn[lane + 32 * q] - 2.0f * acc[q];
            if (sc < best) {
                best = sc;
                bi = lane + 32 * q;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob < best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        if (lane == 0) {
            cell[row] = static_cast<uint8_t>(bi < C ? bi : 0);
            iota[row] = static_cast<int32_t>(row);
        }
    }
}

// First candidate tile of each query group: the tile holding the first row
// of the cell that the group's first row belongs to (binary search in the
// sorted cell keys).
__global__ void group_start_kernel(const uint8_t* __restrict__ skey, int64_t groups,
                                   int rows_per_group, int32_t* __restrict__ start_tile) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= groups) return;
    const int64_t r0 = g * rows_per_group;
    const uint8_t c = skey[r0];
    int64_t lo = 0, hi = r0;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (skey[mid] < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    start_tile[g] = static_cast<int32_t>(lo / BN);
}

__global__ void gather_rows_kernel(const float* __restrict__ X, const int32_t* __restrict__ perm,
                                   int64_t n, int d, float* __restrict__ out) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* src = X + static_cast<int64_t>(perm[row]) * d;
    float* dst = out + row * d;
    for (int t = lane; t < d; t += 32) dst[t] = src[t];
}

struct CellOrder {
    DevBuf<float> rows;          // the rows in cell order
    DevBuf<int32_t> perm;        // position -> original row
    DevBuf<int32_t> start_tile;  // per query group
};

template <int PPL>
void launch_assign(const float* X, int64_t n, int d, uint8_t* cell, int32_t* iota,
                   cudaStream_t s) {
    constexpr int C = 32 * PPL;
    const size_t smem = (static_cast<size_t>(C) * d + C) * sizeof(float);
    auto kern = cell_assign_kernel<PPL>;
    UMAPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    int dev = 0, sms = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 8), static_cast<int64_t>(sms) * 3);
    kern<<<static_cast<unsigned>(blocks), 256, smem, s>>>(X, n, d, n / C, cell, iota);
    UMAPB_LAUNCH_CHECK();
}

void cell_order(const float* X, int64_t n, int d, int cells, int rows_per_group, int64_t groups,
                CellOrder& co, cudaStream_t s) {
    DevBuf<uint8_t> key(n, s), skey(n, s);
    DevBuf<int32_t> iota(n, s);
    co.perm.alloc(n, s);
    switch (cells) {
        case 32: launch_assign<1>(X, n, d, key.get(), iota.get(), s); break;
        case 64: launch_assign<2>(X, n, d, key.get(), iota.get(), s); break;
        case 128: launch_assign<4>(X, n, d, key.get(), iota.get(), s); break;
        default: launch_assign<8>(X, n, d, key.get(), iota.get(), s); break;
    }
    size_t tmp_bytes = 0;
    UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.get(), skey.get(),
                                               iota.get(), co.perm.get(), static_cast<int>(n), 0,
                                               8, s));
    DevBuf<uint8_t> tmp(tmp_bytes, s);
    UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, key.get(), skey.get(),
                                               iota.get(), co.perm.get(), static_cast<int>(n), 0,
                                               8, s));
    co.start_tile.alloc(groups, s);
    group_start_kernel<<<static_cast<unsigned>(ceil_div(groups, 256)), 256, 0, s>>>(
        skey.get(), groups, rows_per_group, co.start_tile.get());
    UMAPB_LAUNCH_CHECK();
    co.rows.alloc(static_cast<size_t>(n) * d, s);
    gather_rows_kernel<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, s>>>(
        X, co.perm.get(), n, d, co.rows.get());
    UMAPB_LAUNCH_CHECK();
}

}  // namespace

bool knn_tc_supported(int d, int k, int metric) {
    if (metric != UMAPB_METRIC_EUCLIDEAN) return false;
    if (k < 1 || k > S - 2 || d < 1) return false;
    if (query_tiles_for(padded_k(d) / BK) == 0) return false;
    return device_is_sm100();
}

void knn_tc(const float* Q, int64_t n_q, const float* R, int64_t n_r, int d, int k, int metric,
            int32_t* out_idx, float* out_dist, TcKnnStats* stats, cudaStream_t s) {
    if (!knn_tc_supported(d, k, metric))
        invalid("the tensor-core kNN path does not support this metric/shape on this device");
    if (n_q == 0) return;
    if (k > n_r) invalid("kNN needs k <= number of reference rows");
    const bool self = Q == R && n_q == n_r;
    const float* const Q0 = Q;  // original rows: the fallback recomputes rows of these
    const float* const R0 = R;
    const int kp = padded_k(d);
    const int kb = kp / BK;
    const double c1 = kBoundC1;
    const double c2 = bound_c2(d);
    TcArgs a = plan(n_q, n_r, d, true);
    const int mt = query_tiles_for(kb);
    CellOrder co;
    const int cells = self && a.n_split == 1 ? cell_count(n_q, d) : 0;
    if (cells > 0) {
        cell_order(Q, n_q, d, cells, mt * BM, ceil_div(n_q, static_cast<int64_t>(BM) * mt), co, s);
        Q = R = co.rows.get();
        a.start_tile = co.start_tile.get();
    }
    DevBuf<float> qsq(n_q, s), rsq;
    row_norms(Q, n_q, d, nullptr, qsq.get(), s);
    if (!self) {
        rsq.alloc(n_r, s);
        row_norms(R, n_r, d, nullptr, rsq.get(), s);
    }
    const float* rsq_p = self ? qsq.get() : rsq.get();
    DevBuf<__nv_bfloat16> A(n_q * kp, s), B(n_r * kp, s);
    prep_kernel<<<static_cast<unsigned>(ceil_div(n_q * 32, 256)), 256, 0, s>>>(
        Q, qsq.get(), n_q, d, kp, static_cast<float>(c1), static_cast<float>(c2), true, A.get());
    UMAPB_LAUNCH_CHECK();
    prep_kernel<<<static_cast<unsigned>(ceil_div(n_r * 32, 256)), 256, 0, s>>>(
        R, rsq_p, n_r, d, kp, static_cast<float>(c1), static_cast<float>(c2), false, B.get());
    UMAPB_LAUNCH_CHECK();
    const int n_lists = 2 * a.n_split;
    DevBuf<uint64_t> lists(n_q * n_lists * S, s);
    UMAPB_CUDA(cudaMemsetAsync(lists.get(), 0xFF, n_q * n_lists * S * 8, s));
    DevBuf<int> err(1, s), fb_count(1, s);
    UMAPB_CUDA(cudaMemsetAsync(err.get(), 0, 4, s));
    UMAPB_CUDA(cudaMemsetAsync(fb_count.get(), 0, 4, s));
    const CUtensorMap ma = make_map(A.get(), n_q, kp);
    const CUtensorMap mb = make_map(B.get(), n_r, kp);
    a.lists = lists.get();
    a.err = err.get();
    cudaEvent_t e0, e1;
    UMAPB_CUDA(cudaEventCreate(&e0));
    UMAPB_CUDA(cudaEventCreate(&e1));
    UMAPB_CUDA(cudaEventRecord(e0, s));
    if (mt == 2)
        launch_tc<2, 4>(ma, mb, a, s);
    else
        launch_tc<1, 3>(ma, mb, a, s);
    UMAPB_CUDA(cudaEventRecord(e1, s));
    int err_h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&err_h, err.get(), 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    UMAPB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err_h != 0)
        throw Error(UMAPB_ERR_CUDA,
                    "tensor-core kNN kernel stopped on a wait timeout (code " +
                        std::to_string(err_h) + ")");
    DevBuf<int32_t> fb_rows(n_q, s);
    rerank_kernel<<<static_cast<unsigned>(ceil_div(n_q * 32, 256)), 256, 0, s>>>(
        Q, R, qsq.get(), rsq_p, lists.get(), n_lists, n_q, d, k, c1, c2,
        cells > 0 ? co.perm.get() : nullptr, out_idx, out_dist, fb_count.get(), fb_rows.get());
    UMAPB_LAUNCH_CHECK();
    int fb = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&fb, fb_count.get(), 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    if (fb > 0) knn_plain(Q0, fb_rows.get(), fb, R0, n_r, d, k, metric, nullptr, nullptr, out_idx,
                          out_dist, s);
    if (stats) {
        stats->fallback_rows = fb;
        stats->kernel_ms = ms;
        stats->shortlist = S;
    }
}

}  // namespace umapb

// ===================================================== allocation-free entry
// umapb_knn_exact_noalloc: the tensor-core exact kNN for callers that cannot
// allocate device memory.  Its scratch (operands, shortlists, flags) lives in
// one file-scope device array of kNoAllocScratchBytes that every GPU loading
// this library holds until the process exits.  In host code the array's name
// is only a host-side stand-in, so the device address is fetched once per
// device with cudaGetSymbolAddress (on the first call made with that device
// current) and reused afterwards.
namespace umapb {
namespace {
constexpr size_t kNoAllocScratchBytes = static_cast<size_t>(64) << 20;
}  // namespace
}  // namespace umapb

static __device__ __align__(256) unsigned char umapb_noalloc_scratch[umapb::kNoAllocScratchBytes];

namespace umapb {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};

unsigned char* noalloc_scratch() {
    int dev = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) invalid("device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        UMAPB_CUDA(cudaGetSymbolAddress(&p, umapb_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_noalloc_ptr[dev];
}

inline size_t round256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// bytes of scratch one call needs for n rows of d features
size_t noalloc_need(int64_t n, int d) {
    const size_t rows = static_cast<size_t>(n);
    const size_t kp = static_cast<size_t>(padded_k(d));
    return round256(rows * 4) + 2 * round256(rows * kp * 2) + round256(rows * 2 * S * 8) +
           round256(8) + round256(rows * 4);
}

void knn_noalloc(const float* X, int64_t n, int d, int k, int32_t* out_idx, float* out_dist,
                 cudaStream_t s) {
    if (n < 1 || d < 1) invalid("empty input");
    if (k < 1 || k > n) invalid("k must be in [1, n_rows]");
    if (!knn_tc_supported(d, k, UMAPB_METRIC_EUCLIDEAN))
        invalid("the allocation-free kNN runs the tensor-core path only (sm_100, euclidean, "
                "k <= 30, n_cols <= 210)");
    const size_t need = noalloc_need(n, d);
    if (need > kNoAllocScratchBytes) {
        int64_t max_rows = 0;
        while (noalloc_need(max_rows + 1024, d) <= kNoAllocScratchBytes) max_rows += 1024;
        invalid("the allocation-free kNN needs " + std::to_string(need) +
                " bytes of scratch, above its static limit of " +
                std::to_string(kNoAllocScratchBytes) + " bytes (about " +
                std::to_string(max_rows) + " rows at " + std::to_string(d) + " columns)");
    }
    const int kp = padded_k(d);
    const int kb = kp / BK;
    const double c1 = kBoundC1;
    const double c2 = bound_c2(d);
    unsigned char* base = noalloc_scratch();
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += round256(bytes);
        return p;
    };
    float* sq = reinterpret_cast<float*>(carve(static_cast<size_t>(n) * 4));
    __nv_bfloat16* A = reinterpret_cast<__nv_bfloat16*>(carve(static_cast<size_t>(n) * kp * 2));
    __nv_bfloat16* B = reinterpret_cast<__nv_bfloat16*>(carve(static_cast<size_t>(n) * kp * 2));
    uint64_t* lists = reinterpret_cast<uint64_t*>(carve(static_cast<size_t>(n) * 2 * S * 8));
    int* flags = reinterpret_cast<int*>(carve(8));  // [0] = kernel error, [1] = fallback count
    int32_t* fb_rows = reinterpret_cast<int32_t*>(carve(static_cast<size_t>(n) * 4));

    // every call starts from cleared shortlists and flags (the array keeps
    // the previous call's contents)
    UMAPB_CUDA(cudaMemsetAsync(lists, 0xFF, static_cast<size_t>(n) * 2 * S * 8, s));
    UMAPB_CUDA(cudaMemsetAsync(flags, 0, 8, s));
    row_norms(X, n, d, nullptr, sq, s);
    prep_kernel<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, s>>>(
        X, sq, n, d, kp, static_cast<float>(c1), static_cast<float>(c2), true, A);
    UMAPB_LAUNCH_CHECK();
    prep_kernel<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, s>>>(
        X, sq, n, d, kp, static_cast<float>(c1), static_cast<float>(c2), false, B);
    UMAPB_LAUNCH_CHECK();
    const CUtensorMap ma = make_map(A, n, kp);
    const CUtensorMap mb = make_map(B, n, kp);
    const int mt = query_tiles_for(kb);
    TcArgs a = plan(n, n, d, false);  // one split: the scratch holds 2 lists per row
    a.lists = lists;
    a.err = flags;
    if (mt == 2)
        launch_tc<2, 4>(ma, mb, a, s);
    else
        launch_tc<1, 3>(ma, mb, a, s);
    int flags_h[2] = {0, 0};
    UMAPB_CUDA(cudaMemcpyAsync(flags_h, flags, 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    if (flags_h[0] != 0)
        throw Error(UMAPB_ERR_CUDA, "tensor-core kNN kernel stopped on a wait timeout (code " +
                                        std::to_string(flags_h[0]) + ")");
    rerank_kernel<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, s>>>(
        X, X, sq, sq, lists, 2, n, d, k, c1, c2, nullptr, out_idx, out_dist, flags + 1, fb_rows);
    UMAPB_LAUNCH_CHECK();
    UMAPB_CUDA(cudaMemcpyAsync(flags_h, flags, 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    if (flags_h[1] > 0)
        knn_plain(X, fb_rows, flags_h[1], X, n, d, k, UMAPB_METRIC_EUCLIDEAN, nullptr, nullptr,
                  out_idx, out_dist, s);
    UMAPB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace umapb

extern "C" int32_t umapb_knn_exact_noalloc(const float* data, int64_t n_rows, int64_t n_cols,
                                           int64_t k, int32_t* indices, float* dists,
                                           void* stream) {
    try {
        umapb::knn_noalloc(data, n_rows, static_cast<int>(n_cols), static_cast<int>(k), indices,
                           dists, static_cast<cudaStream_t>(stream));
        umapb::set_last_error("");
        return UMAPB_OK;
    } catch (const umapb::Error& e) {
        umapb::set_last_error(e.what());
        return e.status;
    } catch (const std::exception& e) {
        umapb::set_last_error(e.what());
        return UMAPB_ERR_CUDA;
    }
}
