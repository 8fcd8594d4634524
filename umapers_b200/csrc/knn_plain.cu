// knn_plain.cu - exact kNN on FP32 CUDA cores (the plain path).
//
// Replaces exact_nearest_neighbors{,_to_reference} (rust_umap/src/lib.rs:
// 2863-2928, 3283-3399).  Each distance is accumulated with the same
// operations in the same order as the reference's AVX2 kernel
// (lib.rs:2468-2492, dim >= 64: eight strided lanes of acc + d*d, lanes summed
// in order, then the scalar tail) or its scalar kernel (lib.rs:2457-2466),
// using __fadd_rn/__fmul_rn so no FMA contraction changes a bit; the fused
// top-k keeps (distance, index) keys, which is the reference's neighbor_cmp
// order.  A CTA owns QT query rows and sweeps all candidate rows in CT-row
// tiles staged in shared memory with the dims permuted into lane order.
#include <cfloat>
#include <climits>

#include "kernels.cuh"

namespace umapb {
namespace {

constexpr int kThreads = 256;

struct LaneLayout {
    int nl;    // lanes: 8 for d >= 64, else 1
    int ll;    // dims per lane
    int tail;  // first dim of the scalar tail
};

__host__ __device__ inline LaneLayout lane_layout(int d) {
    LaneLayout L;
    if (d >= 64) {
        L.nl = 8;
        L.ll = d / 8;
    } else {
        L.nl = 1;
        L.ll = d;
    }
    L.tail = L.nl * L.ll;
    return L;
}

// position in the lane-ordered sequence of feature `dim`
__device__ inline int lane_pos(int dim, const LaneLayout& L) {
    if (dim >= L.tail) return dim;
    return (dim % L.nl) * L.ll + dim / L.nl;
}

// Candidate rows [blockIdx.y * span, min(n_r, (blockIdx.y + 1) * span)) are
// scanned by this CTA.  With `part` non-null the CTA writes its k smallest
// keys to part[(blockIdx.y * n_q + row) * k ...] for knn_merge_kernel instead
// of the final outputs.
template <int QT, int CT, bool COSINE>
__global__ void __launch_bounds__(kThreads)
    knn_plain_kernel(const float* __restrict__ Q, const int32_t* __restrict__ q_rows, int64_t n_q,
                     const float* __restrict__ R, int64_t n_r, int d, int k,
                     const float* __restrict__ qnorm, const float* __restrict__ rnorm,
                     int32_t* __restrict__ out_idx, float* __restrict__ out_dist, int64_t span,
                     uint64_t* __restrict__ part) {
    constexpr int TQ = QT / 16;
    constexpr int TC = CT / 16;
    extern __shared__ __align__(16) unsigned char smem[];
    float* Qs = reinterpret_cast<float*>(smem);                    // [d][QT]
    float* Cs = Qs + static_cast<size_t>(d) * QT;                  // [d][CT]
    float* dt = Cs + static_cast<size_t>(d) * CT;                  // [QT][CT+1]
    uint64_t* lists = reinterpret_cast<uint64_t*>(dt + QT * (CT + 1));  // [QT][k] (8B aligned)
    __shared__ float qn_s[QT];

    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * QT;
    const LaneLayout L = lane_layout(d);

    // stage the query tile
    for (int e = tid; e < QT * d; e += kThreads) {
        const int r = e / d, dim = e % d;
        const int64_t rr = r0 + r;
        float v = 0.0f;
        if (rr < n_q) {
            const int64_t src = q_rows ? q_rows[rr] : rr;
            v = Q[src * d + dim];
        }
        Qs[lane_pos(dim, L) * QT + r] = v;
    }
    if (tid < QT) {
        const int64_t rr = r0 + tid;
        float qv = 0.0f;
        if (COSINE && rr < n_q) qv = qnorm[q_rows ? q_rows[rr] : rr];
        qn_s[tid] = qv;
    }
    for (int e = tid; e < QT * k; e += kThreads) lists[e] = ~0ULL;

    const int64_t c_begin = static_cast<int64_t>(blockIdx.y) * span;
    const int64_t c_end = min(n_r, c_begin + span);
    for (int64_t c0 = c_begin; c0 < c_end; c0 += CT) {
        __syncthreads();  // previous tile's list updates are done
        for (int e = tid; e < CT * d; e += kThreads) {
            const int r = e / d, dim = e % d;
            const int64_t cc = c0 + r;
            Cs[lane_pos(dim, L) * CT + r] = cc < c_end ? R[cc * d + dim] : 0.0f;
        }
        __syncthreads();

        float cur[TQ][TC], sum[TQ][TC];
#pragma unroll
        for (int i = 0; i < TQ; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) sum[i][j] = 0.0f;
        int p = 0;
        for (int l = 0; l < L.nl; ++l) {
#pragma unroll
            for (int i = 0; i < TQ; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) cur[i][j] = 0.0f;
            for (int t = 0; t < L.ll; ++t, ++p) {
                float qv[TQ], cv[TC];
#pragma unroll
                for (int i = 0; i < TQ; ++i) qv[i] = Qs[p * QT + ty * TQ + i];
#pragma unroll
                for (int j = 0; j < TC; ++j) cv[j] = Cs[p * CT + tx * TC + j];
#pragma unroll
                for (int i = 0; i < TQ; ++i)
#pragma unroll
                    for (int j = 0; j < TC; ++j) {
                        if (COSINE) {
                            cur[i][j] = __fadd_rn(cur[i][j], __fmul_rn(qv[i], cv[j]));
                        } else {
                            const float df = __fsub_rn(qv[i], cv[j]);
                            cur[i][j] = __fadd_rn(cur[i][j], __fmul_rn(df, df));
                        }
                    }
            }
#pragma unroll
            for (int i = 0; i < TQ; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j)
                    sum[i][j] = (l == 0) ? cur[i][j] : __fadd_rn(sum[i][j], cur[i][j]);
        }
        for (; p < d; ++p) {
            float qv[TQ], cv[TC];
#pragma unroll
            for (int i = 0; i < TQ; ++i) qv[i] = Qs[p * QT + ty * TQ + i];
#pragma unroll
            for (int j = 0; j < TC; ++j) cv[j] = Cs[p * CT + tx * TC + j];
#pragma unroll
            for (int i = 0; i < TQ; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) {
                    if (COSINE) {
                        sum[i][j] = __fadd_rn(sum[i][j], __fmul_rn(qv[i], cv[j]));
                    } else {
                        const float df = __fsub_rn(qv[i], cv[j]);
                        sum[i][j] = __fadd_rn(sum[i][j], __fmul_rn(df, df));
                    }
                }
        }
#pragma unroll
        for (int i = 0; i < TQ; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) {
                float v = sum[i][j];
                if (COSINE) {
                    // cosine_distance_with_norms (rust_umap/src/lib.rs:2740-2765)
                    const int64_t cc = c0 + tx * TC + j;
                    const float xn = qn_s[ty * TQ + i];
                    const float yn = cc < c_end ? rnorm[cc] : 0.0f;
                    if (xn == 0.0f && yn == 0.0f) {
                        v = 0.0f;
                    } else if (xn == 0.0f || yn == 0.0f) {
                        v = 1.0f;
                    } else {
                        float c = __fdiv_rn(v, __fmul_rn(xn, yn));
                        c = fminf(fmaxf(c, -1.0f), 1.0f);
                        v = __fsub_rn(1.0f, c);
                    }
                }
                dt[(ty * TQ + i) * (CT + 1) + tx * TC + j] = v;
            }
        __syncthreads();

        if (tid < QT && r0 + tid < n_q) {
            uint64_t* list = lists + tid * k;
            uint64_t thr = list[k - 1];
            const int64_t rem = c_end - c0;
            const int cmax = rem < CT ? static_cast<int>(rem) : CT;
            for (int c = 0; c < cmax; ++c) {
                const uint64_t key = knn_key(dt[tid * (CT + 1) + c], static_cast<uint32_t>(c0 + c));
                if (key < thr) {
                    int at = k - 1;
                    while (at > 0 && list[at - 1] > key) {
                        list[at] = list[at - 1];
                        --at;
                    }
                    list[at] = key;
                    thr = list[k - 1];
                }
            }
        }
    }
    __syncthreads();
    if (part != nullptr) {
        if (tid < QT && r0 + tid < n_q) {
            uint64_t* o = part + (static_cast<int64_t>(blockIdx.y) * n_q + r0 + tid) * k;
            for (int c = 0; c < k; ++c) o[c] = lists[tid * k + c];
        }
        return;
    }
    if (tid < QT && r0 + tid < n_q) {
        const int64_t rr = r0 + tid;
        const int64_t dst = q_rows ? q_rows[rr] : rr;
        const uint64_t* list = lists + tid * k;
        for (int c = 0; c < k; ++c) {
            const uint64_t key = list[c];
            float dist = key_dist(key);
            if (!COSINE) dist = __fsqrt_rn(dist);  // sqrt_row_dists (lib.rs:2830-2834)
            out_idx[dst * k + c] = static_cast<int32_t>(key_index(key));
            out_dist[dst * k + c] = dist;
        }
    }
}

// One warp per query row: the k smallest of its `splits` sorted partial
// lists (repeated warp minimum over the list heads), written as the final
// outputs (sqrt of the squared distance for euclidean).
__global__ void knn_merge_kernel(const uint64_t* __restrict__ part, int splits, int64_t n_q,
                                 int k, const int32_t* __restrict__ q_rows, bool cosine,
                                 int32_t* __restrict__ out_idx, float* __restrict__ out_dist) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n_q) return;
    const int64_t dst = q_rows ? q_rows[row] : row;
    // lane l follows the heads of lists l, l + 32, ... (at most 8 per lane)
    int pos[8];
    for (int j = 0; j < 8; ++j) pos[j] = 0;
    for (int c = 0; c < k; ++c) {
        uint64_t best = ~0ull;
        int bj = -1;
        for (int j = 0; j < 8; ++j) {
            const int sp = lane + 32 * j;
            if (sp >= splits || pos[j] >= k) continue;
            const uint64_t v = part[(static_cast<int64_t>(sp) * n_q + row) * k + pos[j]];
            if (v < best) {
                best = v;
                bj = j;
            }
        }
        uint64_t m = best;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const uint64_t t = __shfl_xor_sync(0xffffffffu, m, o);
            m = t < m ? t : m;
        }
        // keys are unique (indices differ), so exactly one lane holds the minimum
        if (best == m && bj >= 0 && m != ~0ull) ++pos[bj];
        if (lane == 0) {
            out_idx[dst * k + c] = static_cast<int32_t>(key_index(m));
            const float dd = key_dist(m);
            out_dist[dst * k + c] = cosine ? dd : __fsqrt_rn(dd);
        }
    }
}

template <int QT, int CT>
size_t plain_smem(int d, int k) {
    return static_cast<size_t>(d) * (QT + CT) * 4 + static_cast<size_t>(QT) * (CT + 1) * 4 +
           static_cast<size_t>(QT) * k * 8 + 16;
}

// When the query tiles fill fewer than two waves and scratch may be
// allocated, the candidate rows are split across CTAs (at least 64 tiles of
// candidates each) and the partial lists merged per row.
template <int QT, int CT, bool COS>
void launch_plain(const float* Q, const int32_t* q_rows, int64_t n_q, const float* R, int64_t n_r,
                  int d, int k, const float* qn, const float* rn, int32_t* oi, float* od,
                  cudaStream_t s, bool allow_scratch) {
    const size_t smem = plain_smem<QT, CT>(d, k);
    auto kern = knn_plain_kernel<QT, CT, COS>;
    UMAPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    const int64_t blocks = ceil_div(n_q, QT);
    int dev = 0, sms = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int64_t splits = 1;
    if (allow_scratch && blocks < 2 * sms)
        splits = std::min<int64_t>(std::min<int64_t>(ceil_div(2 * sms, blocks), 256),
                                   std::max<int64_t>(1, n_r / (64 * CT)));
    if (splits <= 1) {
        kern<<<static_cast<unsigned>(blocks), kThreads, smem, s>>>(Q, q_rows, n_q, R, n_r, d, k,
                                                                  qn, rn, oi, od, n_r, nullptr);
        UMAPB_LAUNCH_CHECK();
        return;
    }
    const int64_t span = ceil_div(ceil_div(n_r, splits), CT) * CT;
    splits = ceil_div(n_r, span);
    DevBuf<uint64_t> part(static_cast<size_t>(splits) * n_q * k, s);
    kern<<<dim3(static_cast<unsigned>(blocks), static_cast<unsigned>(splits)), kThreads, smem, s>>>(
        Q, q_rows, n_q, R, n_r, d, k, qn, rn, oi, od, span, part.get());
    UMAPB_LAUNCH_CHECK();
    knn_merge_kernel<<<static_cast<unsigned>(ceil_div(n_q * 32, 256)), 256, 0, s>>>(
        part.get(), static_cast<int>(splits), n_q, k, q_rows, COS, oi, od);
    UMAPB_LAUNCH_CHECK();
}

__global__ void row_norms_kernel(const float* __restrict__ X, int64_t n, int d,
                                 float* __restrict__ norms, float* __restrict__ sq) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* x = X + i * d;
    float s;
    if (d >= 64) {
        float lane[8];
#pragma unroll
        for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
        int idx = 0;
        for (; idx + 8 <= d; idx += 8)
#pragma unroll
            for (int l = 0; l < 8; ++l) lane[l] = __fadd_rn(lane[l], __fmul_rn(x[idx + l], x[idx + l]));
        s = lane[0];
#pragma unroll
        for (int l = 1; l < 8; ++l) s = __fadd_rn(s, lane[l]);
        for (; idx < d; ++idx) s = __fadd_rn(s, __fmul_rn(x[idx], x[idx]));
    } else {
        s = 0.0f;
        for (int idx = 0; idx < d; ++idx) s = __fadd_rn(s, __fmul_rn(x[idx], x[idx]));
    }
    if (sq) sq[i] = s;
    if (norms) norms[i] = __fsqrt_rn(s);
}

__global__ void nonfinite_kernel(const float* __restrict__ X, int64_t total, int d,
                                 int64_t row_offset, unsigned long long* first_row) {
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (!isfinite(X[e]))
            atomicMin(first_row, static_cast<unsigned long long>(e / d + row_offset));
    }
}

// The same scan over a 16-byte aligned array: four 16-byte loads in flight
// per thread; elements past the last whole float4 are checked one by one.
__global__ void nonfinite_v4_kernel(const float* __restrict__ X, int64_t total, int d,
                                    int64_t row_offset, unsigned long long* first_row) {
    const float4* X4 = reinterpret_cast<const float4*>(X);
    const int64_t total4 = total >> 2;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t e = t; e < total4; e += 4 * stride) {
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t f = e + u * stride;
            v[u] = f < total4 ? __ldg(X4 + f) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float c[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (!isfinite(c[i])) {
                    atomicMin(first_row, static_cast<unsigned long long>(
                                             (4 * (e + u * stride) + i) / d + row_offset));
                    break;
                }
        }
    }
    const int64_t tail = (total4 << 2) + t;
    if (tail < total && !isfinite(X[tail]))
        atomicMin(first_row, static_cast<unsigned long long>(tail / d + row_offset));
}

}  // namespace

void row_norms(const float* X, int64_t n, int d, float* norms, float* sq, cudaStream_t s) {
    if (n == 0) return;
    row_norms_kernel<<<static_cast<unsigned>(ceil_div(n, 256)), 256, 0, s>>>(X, n, d, norms, sq);
    UMAPB_LAUNCH_CHECK();
}

void nonfinite_rows_async(const float* X, int64_t n, int d, int64_t row_offset,
                          unsigned long long* first_row, cudaStream_t s) {
    const int64_t total = n * d;
    if (total <= 0) return;
    const int blocks = static_cast<int>(std::min<int64_t>(ceil_div(total, 256), 148 * 16));
    if ((reinterpret_cast<uintptr_t>(X) & 15) == 0)
        nonfinite_v4_kernel<<<blocks, 256, 0, s>>>(X, total, d, row_offset, first_row);
    else
        nonfinite_kernel<<<blocks, 256, 0, s>>>(X, total, d, row_offset, first_row);
    UMAPB_LAUNCH_CHECK();
}

int64_t first_nonfinite_row(const float* X, int64_t n, int d, cudaStream_t s) {
    DevBuf<unsigned long long> flag(1, s);
    UMAPB_CUDA(cudaMemsetAsync(flag.get(), 0xFF, 8, s));
    nonfinite_rows_async(X, n, d, 0, flag.get(), s);
    unsigned long long h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, flag.get(), 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return h == ~0ULL ? INT64_MAX : static_cast<int64_t>(h);
}

bool knn_plain_supported(int d, int k) {
    return plain_smem<16, 16>(d, k) <= 200 * 1024;
}

void knn_plain(const float* Q, const int32_t* q_rows, int64_t n_q, const float* R, int64_t n_r,
               int d, int k, int metric, const float* qnorm, const float* rnorm,
               int32_t* out_idx, float* out_dist, cudaStream_t s, bool allow_scratch) {
    if (n_q == 0) return;
    if (k < 1 || k > n_r) invalid("kNN needs 1 <= k <= number of reference rows");
    const bool cos = metric == UMAPB_METRIC_COSINE;
    if (!cos && metric != UMAPB_METRIC_EUCLIDEAN)
        invalid("the B200 kNN kernels support metric euclidean and cosine");
    const size_t limit = 200 * 1024;
    if (plain_smem<64, 64>(d, k) <= limit) {
        if (cos)
            launch_plain<64, 64, true>(Q, q_rows, n_q, R, n_r, d, k, qnorm, rnorm, out_idx,
                                       out_dist, s, allow_scratch);
        else
            launch_plain<64, 64, false>(Q, q_rows, n_q, R, n_r, d, k, qnorm, rnorm, out_idx,
                                        out_dist, s, allow_scratch);
    } else if (plain_smem<32, 32>(d, k) <= limit) {
        if (cos)
            launch_plain<32, 32, true>(Q, q_rows, n_q, R, n_r, d, k, qnorm, rnorm, out_idx,
                                       out_dist, s, allow_scratch);
        else
            launch_plain<32, 32, false>(Q, q_rows, n_q, R, n_r, d, k, qnorm, rnorm, out_idx,
                                        out_dist, s, allow_scratch);
    } else if (plain_smem<16, 16>(d, k) <= limit) {
        if (cos)
            launch_plain<16, 16, true>(Q, q_rows, n_q, R, n_r, d, k, qnorm, rnorm, out_idx,
                                       out_dist, s, allow_scratch);
        else
            launch_plain<16, 16, false>(Q, q_rows, n_q, R, n_r, d, k, qnorm, rnorm, out_idx,
                                        out_dist, s, allow_scratch);
    } else {
        invalid("n_features/n_neighbors too large for the exact kNN tile (need d*128 + k*128 < 200 KiB)");
    }
}

}  // namespace umapb
