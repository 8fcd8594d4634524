// gemm_tc.cu - BF16 tensor-core GEMM with fused epilogues, the building
// block of the transform surrogate's forward and backward passes.
//
// C[M x N] = A[M x K] B[N x K]^T.  One CTA computes one 128 x 128 tile of C:
//   warp 0      TMA producer: k-blocks of A and B (64 bf16 columns each,
//               SWIZZLE_128B) through a kStages-deep shared-memory ring;
//   warp 1      allocates 128 TMEM columns; one thread issues
//               tcgen05.mma kind::f16 (M = N = 128, K = 16) into them;
//   warps 2..5  epilogue: each reads its 32 TMEM lanes (rows) with
//               tcgen05.ld, 32 columns at a time, and applies the fused
//               operation (bias + GELU, GELU backward, output head, row min).
// Tiles are numbered along N first, so the CTAs that share an A tile run
// together and A is read from HBM once.  TMA loads read only this GPU's
// memory and never multicast.  Every wait is bounded; a timeout sets a
// device error word that gemm_take_error() reports.
#include "kernels.cuh"
#include "tcgen05.cuh"

__device__ int umapb_gemm_error_word;

namespace umapb {
namespace {

using namespace tc;

constexpr int GM = 128, GN = 128;
constexpr int kStages = 3;
constexpr int kTileBytes = GM * kBK * 2;         // 16 KiB per operand k-block
constexpr int kStageBytes = 2 * kTileBytes;      // A + B
constexpr uint32_t kGemmIdesc = idesc_bf16(GM, GN);
constexpr uint32_t kTmemCols = GN;

struct GemmParams {
    int64_t M, N;
    int kb;           // K / 64
    int64_t n_tiles;  // column tiles
    GemmOut o;
};

__device__ __forceinline__ float gelu_f(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
// d/dz [z Phi(z)] = Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_grad_f(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// 32 bf16 values of one row (64 contiguous bytes) from fp32 values.
__device__ __forceinline__ void store_bf16x32(__nv_bfloat16* dst, const float* v) {
    uint4* d4 = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int q = 0; q < 4; ++q)
        d4[q] = make_uint4(pack_bf16(v[8 * q + 0], v[8 * q + 1]), pack_bf16(v[8 * q + 2], v[8 * q + 3]),
                           pack_bf16(v[8 * q + 4], v[8 * q + 5]), pack_bf16(v[8 * q + 6], v[8 * q + 7]));
}

__device__ __forceinline__ void store_f32x32(float* dst, const float* v) {
    float4* d4 = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int q = 0; q < 8; ++q) d4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

template <int EPI>
__device__ __forceinline__ void epilogue(const GemmParams& p, uint32_t taddr, int64_t row,
                                         int64_t n0, int64_t tile_n) {
    const bool rv = row < p.M;
    const GemmOut& o = p.o;
    float head[kGemmMaxHead];
#pragma unroll
    for (int h = 0; h < kGemmMaxHead; ++h) head[h] = 0.0f;
    float best = INFINITY;
    int32_t best_n = -1;
#pragma unroll 1
    for (int c = 0; c < GN / 32; ++c) {
        uint32_t r[32];
        tmem_ld32(taddr + 32 * c, r);
        tmem_wait_ld();
        const int64_t nb = n0 + 32 * c;
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
        if (EPI == kEpiF32) {
            if (rv) store_f32x32(o.c + row * p.N + nb, v);
        } else if (EPI == kEpiBiasGelu || EPI == kEpiBiasGeluHead) {
            const float4* b4 = reinterpret_cast<const float4*>(o.bias + nb);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 b = __ldg(b4 + q);
                v[4 * q] += b.x;
                v[4 * q + 1] += b.y;
                v[4 * q + 2] += b.z;
                v[4 * q + 3] += b.w;
            }
            if (rv && o.z) store_f32x32(o.z + row * p.N + nb, v);
#pragma unroll
            for (int j = 0; j < 32; ++j)
                v[j] = __bfloat162float(__float2bfloat16_rn(gelu_f(v[j])));
            if (rv && o.act) store_bf16x32(o.act + row * p.N + nb, v);
            if (rv && o.act_t) {
#pragma unroll
                for (int j = 0; j < 32; ++j) o.act_t[(nb + j) * o.ld_t + row] = __float2bfloat16_rn(v[j]);
            }
            if (EPI == kEpiBiasGeluHead) {
#pragma unroll
                for (int h = 0; h < kGemmMaxHead; ++h) {
                    if (h < o.head_dim) {
                        const float* w = o.head_w + h * p.N + nb;
                        float acc = 0.0f;
#pragma unroll
                        for (int j = 0; j < 32; ++j) acc = fmaf(v[j], __ldg(w + j), acc);
                        head[h] += acc;
                    }
                }
            }
        } else if (EPI == kEpiGeluBwd) {
            if (rv) {
                const float4* z4 = reinterpret_cast<const float4*>(o.z_in + row * p.N + nb);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float4 z = z4[q];
                    v[4 * q] *= gelu_grad_f(z.x);
                    v[4 * q + 1] *= gelu_grad_f(z.y);
                    v[4 * q + 2] *= gelu_grad_f(z.z);
                    v[4 * q + 3] *= gelu_grad_f(z.w);
                }
                if (o.act) store_bf16x32(o.act + row * p.N + nb, v);
                if (o.act_t) {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        o.act_t[(nb + j) * o.ld_t + row] = __float2bfloat16_rn(v[j]);
                }
            }
        } else if (EPI == kEpiRowMin) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int64_t n = nb + j;
                if (n < o.n_valid) {
                    const float d = fmaf(-2.0f, v[j], __ldg(o.col_sq + n));
                    if (d < best) {
                        best = d;
                        best_n = static_cast<int32_t>(n);
                    }
                }
            }
        }
    }
    if (EPI == kEpiBiasGeluHead && rv) {
        float* dst = o.head_part + (tile_n * p.M + row) * o.head_dim;
        for (int h = 0; h < o.head_dim; ++h) dst[h] = head[h];
    }
    if (EPI == kEpiRowMin && rv) {
        o.min_val[tile_n * p.M + row] = best;
        o.min_idx[tile_n * p.M + row] = best_n;
    }
}

template <int EPI>
__global__ void __launch_bounds__(192, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                GemmParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const uint32_t s0 = smem_u32(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    const uint32_t b_full = smem_u32(bars);
    const uint32_t b_empty = b_full + 8 * kStages;
    const uint32_t b_tfull = b_empty + 8 * kStages;
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t tile = blockIdx.x;
    const int64_t tile_n = tile % p.n_tiles;
    const int64_t m0 = (tile / p.n_tiles) * GM;
    const int64_t n0 = tile_n * GN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(b_full + 8 * s, 1);
            mbar_init(b_empty + 8 * s, 1);
        }
        mbar_init(b_tfull, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(smem_u32(tmem_holder), kTmemCols);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_holder;

    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicCAS(&umapb_gemm_error_word, 0, code);
    };

    if (warp == 0) {
        if (lane == 0) {
            for (int kb = 0; kb < p.kb; ++kb) {
                const int st = kb % kStages;
                const uint32_t round = static_cast<uint32_t>(kb / kStages);
                if (!mbar_wait(b_empty + 8 * st, (round & 1) ^ 1, abort_flag)) {
                    fail(1);
                    break;
                }
                const uint32_t sa = s0 + st * kStageBytes;
                mbar_expect_tx(b_full + 8 * st, kStageBytes);
                tma_load_2d(sa, &tmA, b_full + 8 * st, kb * kBK, static_cast<int>(m0));
                tma_load_2d(sa + kTileBytes, &tmB, b_full + 8 * st, kb * kBK, static_cast<int>(n0));
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            bool ok = true;
            for (int kb = 0; kb < p.kb; ++kb) {
                const int st = kb % kStages;
                if (!mbar_wait(b_full + 8 * st, static_cast<uint32_t>((kb / kStages) & 1),
                               abort_flag)) {
                    fail(2);
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t sa = s0 + st * kStageBytes;
                const uint64_t da = desc_sw128(sa), db = desc_sw128(sa + kTileBytes);
#pragma unroll
                for (int ks = 0; ks < kBK / kUK; ++ks)
                    umma_bf16(tmem_base, da + 2 * ks, db + 2 * ks, kGemmIdesc,
                              (kb | ks) != 0 ? 1u : 0u);
                umma_commit(b_empty + 8 * st);
            }
            if (ok) umma_commit(b_tfull);
        }
    } else {
        const int quarter = warp & 3;
        if (mbar_wait(b_tfull, 0, abort_flag)) {
            fence_after();
            epilogue<EPI>(p, tmem_base + (static_cast<uint32_t>(quarter * 32) << 16),
                          m0 + quarter * 32 + lane, n0, tile_n);
        } else if (lane == 0) {
            fail(3);
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

template <int EPI>
void launch(const CUtensorMap& ma, const CUtensorMap& mb, const GemmParams& p, int64_t m_tiles,
            cudaStream_t s) {
    const size_t smem = static_cast<size_t>(kStages) * kStageBytes + 1024 + 128;
    auto kern = gemm_kernel<EPI>;
    UMAPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    const int64_t grid = m_tiles * p.n_tiles;
    kern<<<static_cast<unsigned>(grid), 192, smem, s>>>(ma, mb, p);
    UMAPB_LAUNCH_CHECK();
}

}  // namespace

void gemm_bf16_tn(const __nv_bfloat16* A, const __nv_bfloat16* B, int64_t M, int64_t N, int64_t K,
                  int epilogue, const GemmOut& out, cudaStream_t s) {
    if (M < 1 || N < 1 || K < kBK || K % kBK != 0)
        invalid("gemm_bf16_tn: M, N must be positive and K a positive multiple of 64");
    if (epilogue != kEpiRowMin && N % GN != 0)
        invalid("gemm_bf16_tn: N must be a multiple of 128");
    if (epilogue == kEpiBiasGeluHead && (out.head_dim < 1 || out.head_dim > kGemmMaxHead))
        invalid("gemm_bf16_tn: head_dim must be in [1, 4]");
    if (!device_is_sm100()) invalid("the tensor-core GEMM needs an sm_100 device");
    GemmParams p{};
    p.M = M;
    p.N = N;
    p.kb = static_cast<int>(K / kBK);
    p.n_tiles = ceil_div(N, static_cast<int64_t>(GN));
    p.o = out;
    if (epilogue == kEpiRowMin && p.o.n_valid == 0) p.o.n_valid = N;
    const int64_t m_tiles = ceil_div(M, static_cast<int64_t>(GM));
    if (m_tiles * p.n_tiles > 0x7FFFFFFFll) invalid("gemm_bf16_tn: too many tiles");
    const CUtensorMap ma = make_bf16_map(A, M, K, GM);
    const CUtensorMap mb = make_bf16_map(B, N, K, GN);
    switch (epilogue) {
        case kEpiF32: launch<kEpiF32>(ma, mb, p, m_tiles, s); break;
        case kEpiBiasGelu: launch<kEpiBiasGelu>(ma, mb, p, m_tiles, s); break;
        case kEpiGeluBwd: launch<kEpiGeluBwd>(ma, mb, p, m_tiles, s); break;
        case kEpiBiasGeluHead: launch<kEpiBiasGeluHead>(ma, mb, p, m_tiles, s); break;
        case kEpiRowMin: launch<kEpiRowMin>(ma, mb, p, m_tiles, s); break;
        default: invalid("gemm_bf16_tn: unknown epilogue");
    }
}

int gemm_take_error(cudaStream_t s) {
    int h = 0;
    UMAPB_CUDA(cudaMemcpyFromSymbolAsync(&h, umapb_gemm_error_word, sizeof(int), 0,
                                         cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    if (h != 0) {
        const int zero = 0;
        UMAPB_CUDA(cudaMemcpyToSymbolAsync(umapb_gemm_error_word, &zero, sizeof(int), 0,
                                           cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
    }
    return h;
}

}  // namespace umapb
