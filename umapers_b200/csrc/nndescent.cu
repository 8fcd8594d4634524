// nndescent.cu - the reference's NN-descent variant on the device.
//
// approximate_nearest_neighbors_with_distance (rust_umap/src/lib.rs:3086-3151)
// with its candidate rule (collect_approx_candidate_indices, lib.rs:3051-3084):
// pool = min(max(cand, k), n-1); max_candidates = 4*max(cand, k) + 1; the
// initial lists are self + `pool` unique random rows; every iteration a row's
// candidates are its neighbours, their neighbours, itself and
// max(4, min(k/2, max_candidates)) random rows, de-duplicated and sorted by
// index, cut to max_candidates by a random partial Fisher-Yates shuffle, all
// evaluated, best k kept by (distance, index).  Iterations read the previous
// lists and write new ones (as the reference's collect-then-replace does) and
// stop when no row changed.  One warp owns one row; candidates live in shared
// memory and are ordered with warp bitonic sorts.  Distances use the
// reference's summation order (euclidean = sqrt of the squared distance,
// lib.rs:3167).  Random streams are counter-based per (row, iteration).
//
// Candidate evaluation is a gather of whole rows.  For d >= 64 the warp
// splits into four groups of eight lanes; a group evaluates one candidate,
// lane r of the group accumulating the reference's AVX2 lane r (dims r,
// r + 8, ...) from the row's consecutive 32-byte sectors, so each step of a
// group reads one sector and a warp four candidates at once.  The group's
// eight partial sums are added in lane order, then the scalar tail, exactly
// as the reference does.  The query row sits in shared memory.
#include <climits>
#include <vector>

#include "kernels.cuh"

namespace umapb {
namespace {

constexpr int kWarps = 4;

// Bitonic sort of `cnt` (<= cap, cap a power of two) 64-bit keys in shared
// memory by one warp; slots past `cnt` must hold ~0.
__device__ inline void warp_sort_u64(uint64_t* a, int cap) {
    const int lane = threadIdx.x & 31;
    for (int size = 2; size <= cap; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < cap / 2; t += 32) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool up = ((lo & size) == 0);
                const uint64_t x = a[lo], y = a[hi];
                if ((x > y) == up) {
                    a[lo] = y;
                    a[hi] = x;
                }
            }
            __syncwarp();
        }
    }
}

// Distance of query row i (in shared memory `qs`) to the candidates in
// keys[0, m) (row indices), written back in place as (distance, index) keys.
// Every lane of the warp calls it with the same m.
__device__ inline void eval_candidates(const float* __restrict__ X, const float* __restrict__ norms,
                                       int64_t i, int d, bool cosine, const float* qs,
                                       uint64_t* keys, int m) {
    const int lane = threadIdx.x & 31;
    if (d < 64) {
        // the reference's scalar loop: one lane per candidate
        for (int c = lane; c < m; c += 32) {
            const int64_t j = static_cast<int64_t>(keys[c]);
            const float* y = X + j * d;
            float sum = 0.0f;
            for (int t = 0; t < d; ++t) {
                if (cosine) {
                    sum = __fadd_rn(sum, __fmul_rn(qs[t], y[t]));
                } else {
                    const float df = __fsub_rn(qs[t], y[t]);
                    sum = __fadd_rn(sum, __fmul_rn(df, df));
                }
            }
            float dist;
            if (!cosine) {
                dist = __fsqrt_rn(sum);
            } else {
                const float xn = norms[i], yn = norms[j];
                if (xn == 0.0f && yn == 0.0f) {
                    dist = 0.0f;
                } else if (xn == 0.0f || yn == 0.0f) {
                    dist = 1.0f;
                } else {
                    float cs = __fdiv_rn(sum, __fmul_rn(xn, yn));
                    cs = fminf(fmaxf(cs, -1.0f), 1.0f);
                    dist = __fsub_rn(1.0f, cs);
                }
            }
            keys[c] = knn_key(dist, static_cast<uint32_t>(j));
        }
        return;
    }
    const int g = lane >> 3, r = lane & 7, leader = lane & ~7;
    const int body = (d / 8) * 8;
    for (int base = 0; base < m; base += 4) {
        const int c = base + g;
        const bool act = c < m;
        const int64_t j = act ? static_cast<int64_t>(keys[c]) : i;
        const float* y = X + j * d;
        float acc = 0.0f;
        if (cosine) {
            for (int t = r; t < body; t += 8) acc = __fadd_rn(acc, __fmul_rn(qs[t], __ldg(y + t)));
        } else {
            for (int t = r; t < body; t += 8) {
                const float df = __fsub_rn(qs[t], __ldg(y + t));
                acc = __fadd_rn(acc, __fmul_rn(df, df));
            }
        }
        // lanes summed in order, then the tail (lib.rs:2468-2492, 2717-2738)
        float sum = __shfl_sync(0xffffffffu, acc, leader);
#pragma unroll
        for (int l = 1; l < 8; ++l) sum = __fadd_rn(sum, __shfl_sync(0xffffffffu, acc, leader + l));
        if (r == 0 && act) {
            for (int t = body; t < d; ++t) {
                if (cosine) {
                    sum = __fadd_rn(sum, __fmul_rn(qs[t], y[t]));
                } else {
                    const float df = __fsub_rn(qs[t], y[t]);
                    sum = __fadd_rn(sum, __fmul_rn(df, df));
                }
            }
            float dist;
            if (!cosine) {
                dist = __fsqrt_rn(sum);
            } else {
                const float xn = norms[i], yn = norms[j];
                if (xn == 0.0f && yn == 0.0f) {
                    dist = 0.0f;
                } else if (xn == 0.0f || yn == 0.0f) {
                    dist = 1.0f;
                } else {
                    float cs = __fdiv_rn(sum, __fmul_rn(xn, yn));
                    cs = fminf(fmaxf(cs, -1.0f), 1.0f);
                    dist = __fsub_rn(1.0f, cs);
                }
            }
            keys[c] = knn_key(dist, static_cast<uint32_t>(j));
        }
    }
}

// CSR rows for the sparse variant: the reference's SparseCsrMatrix fields
// (sparse.rs:9-147) with its norms (sum of v * v in stored order, sqrt).
struct NdCsr {
    const int64_t* ptr;
    const int32_t* idx;
    const float* val;
    const float* sq;
    const float* l2;
    int max_nnz;
};

// Distance of CSR row i (its columns and values in shared memory) to the
// candidates in keys[0, m), one lane per candidate: the sparse dot is a
// merge of the two sorted column lists, products of shared columns added in
// ascending column order from +0.0 (sparse_dot, sparse.rs:220-239), and the
// distance comes from it and the norms as in the exact sparse kNN
// (sparse.rs:605-626); a row's distance to itself is 0 (sparse.rs:614-617).
__device__ inline void eval_candidates_csr(const NdCsr& x, int64_t i, int metric, const int32_t* qc,
                                           const float* qv, int qn, uint64_t* keys, int m) {
    const int lane = threadIdx.x & 31;
    const float q_sq = x.sq[i], q_l2 = x.l2[i];
    for (int c = lane; c < m; c += 32) {
        const int64_t j = static_cast<int64_t>(keys[c]);
        float dist = 0.0f;
        if (j != i) {
            float dot = 0.0f;
            int a = 0;
            int64_t b = x.ptr[j];
            const int64_t be = x.ptr[j + 1];
            while (a < qn && b < be) {
                const int32_t ca = qc[a], cb = x.idx[b];
                if (ca == cb) {
                    dot = __fadd_rn(dot, __fmul_rn(qv[a], x.val[b]));
                    ++a;
                    ++b;
                } else if (ca < cb) {
                    ++a;
                } else {
                    ++b;
                }
            }
            if (metric == UMAPB_METRIC_COSINE) {
                const float r_l2 = x.l2[j];
                if (q_l2 == 0.0f && r_l2 == 0.0f) {
                    dist = 0.0f;
                } else if (q_l2 == 0.0f || r_l2 == 0.0f) {
                    dist = 1.0f;
                } else {
                    float cs = __fdiv_rn(dot, __fmul_rn(q_l2, r_l2));
                    cs = fminf(fmaxf(cs, -1.0f), 1.0f);
                    dist = __fsub_rn(1.0f, cs);
                }
            } else {
                float t = __fsub_rn(__fadd_rn(q_sq, x.sq[j]), __fmul_rn(2.0f, dot));
                if (!(t > 0.0f)) t = 0.0f;
                dist = __fsqrt_rn(t);
            }
        }
        keys[c] = knn_key(dist, static_cast<uint32_t>(j));
    }
}

struct NdArgs {
    const float* X;
    const float* norms;
    int64_t n;
    int d;
    int k;
    int pool;
    int maxc;
    int expl;
    int cap;  // power of two >= k + k*k + 1 + expl
    bool cosine;
    uint64_t seed;
    const int32_t* old_idx;
    const float* old_dist;
    int32_t* new_idx;
    float* new_dist;
    int* changed;
    unsigned long long* evaluated;  // kEvalSlots counters of candidates evaluated
    NdCsr csr;                       // sparse rows (the SP kernels)
    int metric;
};

constexpr int kEvalSlots = 64;  // spread the per-warp counts over 64 addresses

// Shared memory of one warp: cap keys, cap candidate indices, the query row
// (d floats dense; columns and values of at most `d` stored entries sparse).
__host__ __device__ inline size_t nd_warp_smem(int cap, int d, bool sparse = false) {
    return static_cast<size_t>(cap) * 12 + static_cast<size_t>((d + 3) / 4) * 16 * (sparse ? 2 : 1);
}

// The query row into the warp's shared memory; returns its stored entries
// (sparse) or d (dense).
template <bool SP>
__device__ inline int load_query(const NdArgs& p, int64_t i, float* qs) {
    const int lane = threadIdx.x & 31;
    if (!SP) {
        for (int t = lane; t < p.d; t += 32) qs[t] = p.X[i * p.d + t];
        return p.d;
    }
    const int64_t b = p.csr.ptr[i];
    const int qn = static_cast<int>(p.csr.ptr[i + 1] - b);
    int32_t* qc = reinterpret_cast<int32_t*>(qs);
    float* qv = qs + p.csr.max_nnz;
    for (int t = lane; t < qn; t += 32) {
        qc[t] = p.csr.idx[b + t];
        qv[t] = p.csr.val[b + t];
    }
    return qn;
}

template <bool SP>
__device__ inline void eval_any(const NdArgs& p, int64_t i, const float* qs, int qn,
                                uint64_t* keys, int m) {
    if (SP)
        eval_candidates_csr(p.csr, i, p.metric, reinterpret_cast<const int32_t*>(qs),
                            qs + p.csr.max_nnz, qn, keys, m);
    else
        eval_candidates(p.X, p.norms, i, p.d, p.cosine, qs, keys, m);
}

// initial lists: self + `pool` unique random rows, best k kept (lib.rs:3100-3115)
template <bool SP>
__global__ void __launch_bounds__(kWarps * 32) nd_init_kernel(NdArgs p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ws = smem + warp * nd_warp_smem(p.cap, SP ? p.csr.max_nnz : p.d, SP);
    uint64_t* keys = reinterpret_cast<uint64_t*>(ws);
    int32_t* cand = reinterpret_cast<int32_t*>(keys + p.cap);
    float* qs = reinterpret_cast<float*>(cand + p.cap);
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kWarps + warp;
    if (i >= p.n) return;
    const int qn = load_query<SP>(p, i, qs);
    int cnt = 0;
    if (lane == 0) {
        cand[cnt++] = static_cast<int32_t>(i);
        uint64_t ctr = 0;
        while (cnt < p.pool + 1) {
            const int32_t j = static_cast<int32_t>(
                rng_below(rng_word(p.seed, static_cast<uint64_t>(i), ctr++), static_cast<uint32_t>(p.n)));
            bool dup = false;
            for (int c = 0; c < cnt; ++c) dup |= cand[c] == j;
            if (!dup) cand[cnt++] = j;
        }
    }
    cnt = __shfl_sync(0xffffffffu, cnt, 0);
    __syncwarp();
    for (int c = lane; c < p.cap; c += 32)
        keys[c] = c < cnt ? static_cast<uint64_t>(cand[c]) : ~0ULL;
    __syncwarp();
    eval_any<SP>(p, i, qs, qn, keys, cnt);
    __syncwarp();
    if (lane == 0)
        atomicAdd(p.evaluated + blockIdx.x % kEvalSlots, static_cast<unsigned long long>(cnt));
    warp_sort_u64(keys, p.cap);
    for (int c = lane; c < p.k; c += 32) {
        p.new_idx[i * p.k + c] = static_cast<int32_t>(key_index(keys[c]));
        p.new_dist[i * p.k + c] = key_dist(keys[c]);
    }
}

template <bool SP>
__global__ void __launch_bounds__(kWarps * 32) nd_iter_kernel(NdArgs p, uint64_t iteration) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ws = smem + warp * nd_warp_smem(p.cap, SP ? p.csr.max_nnz : p.d, SP);
    uint64_t* keys = reinterpret_cast<uint64_t*>(ws);
    float* qs = reinterpret_cast<float*>(reinterpret_cast<int32_t*>(keys + p.cap) + p.cap);
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kWarps + warp;
    if (i >= p.n) return;
    const int qn = load_query<SP>(p, i, qs);
    const int k = p.k;
    // neighbours and neighbours of neighbours, as index keys (duplicates removed after sorting)
    int cnt = 0;
    for (int c = lane; c < k; c += 32) keys[c] = static_cast<uint64_t>(p.old_idx[i * k + c]);
    for (int t = lane; t < k * k; t += 32) {
        const int32_t nb = p.old_idx[i * k + t / k];
        keys[k + t] = static_cast<uint64_t>(p.old_idx[static_cast<int64_t>(nb) * k + t % k]);
    }
    cnt = k + k * k;
    if (lane == 0) keys[cnt] = static_cast<uint64_t>(i);
    ++cnt;
    const uint64_t rbase = iteration << 40;
    for (int e = lane; e < p.expl; e += 32)
        keys[cnt + e] = rng_below(rng_word(p.seed, static_cast<uint64_t>(i), rbase + e),
                                  static_cast<uint32_t>(p.n));
    cnt += p.expl;
    for (int c = cnt + lane; c < p.cap; c += 32) keys[c] = ~0ULL;
    __syncwarp();
    warp_sort_u64(keys, p.cap);
    // unique (sorted by index, as out.sort_unstable() leaves it)
    int uniq = 0;
    for (int base = 0; base < cnt; base += 32) {
        const int c = base + lane;
        const uint64_t v = c < cnt ? keys[c] : ~0ULL;
        const uint64_t prev = (c > 0 && c < cnt) ? keys[c - 1] : ~0ULL - 1;
        const bool keep = c < cnt && v != prev;
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) keys[uniq + __popc(mask & ((1u << lane) - 1))] = v;
        __syncwarp();
        uniq += __popc(mask);
    }
    // random partial Fisher-Yates down to max_candidates (lib.rs:3076-3083)
    if (uniq > p.maxc && lane == 0) {
        uint64_t ctr = 1u << 20;
        for (int s = 0; s < p.maxc; ++s) {
            const uint32_t span = static_cast<uint32_t>(uniq - s);
            const int r = s + static_cast<int>(rng_below(
                                  rng_word(p.seed, static_cast<uint64_t>(i), rbase + ctr++), span));
            const uint64_t t = keys[s];
            keys[s] = keys[r];
            keys[r] = t;
        }
    }
    __syncwarp();
    const int m = min(uniq, p.maxc);
    // evaluate every candidate
    for (int c = m + lane; c < p.cap; c += 32) keys[c] = ~0ULL;
    __syncwarp();
    eval_any<SP>(p, i, qs, qn, keys, m);
    __syncwarp();
    if (lane == 0)
        atomicAdd(p.evaluated + blockIdx.x % kEvalSlots, static_cast<unsigned long long>(m));
    warp_sort_u64(keys, p.cap);
    bool diff = false;
    for (int c = lane; c < k; c += 32) {
        const int32_t ni = static_cast<int32_t>(key_index(keys[c]));
        const float nd = key_dist(keys[c]);
        diff |= (ni != p.old_idx[i * k + c]) || (nd != p.old_dist[i * k + c]);
        p.new_idx[i * k + c] = ni;
        p.new_dist[i * k + c] = nd;
    }
    if (__any_sync(0xffffffffu, diff) && lane == 0) *p.changed = 1;
}

}  // namespace

namespace {

// The iteration loop shared by the dense and CSR rows: initial lists, then
// iterations until no row changes (lists alternate between the output arrays
// and a scratch pair).
template <bool SP>
int64_t nndescent_run(NdArgs p, int64_t n, int k, int64_t n_iters, size_t smem, int32_t* out_idx,
                      float* out_dist, cudaStream_t s, NdStats* stats) {
    DevBuf<int32_t> idx_b(n * k, s);
    DevBuf<float> dist_b(n * k, s);
    DevBuf<int> changed(1, s);
    DevBuf<unsigned long long> evaluated(kEvalSlots, s);
    UMAPB_CUDA(cudaMemsetAsync(evaluated.get(), 0, kEvalSlots * 8, s));
    p.evaluated = evaluated.get();
    p.changed = changed.get();
    UMAPB_CUDA(cudaFuncSetAttribute(nd_init_kernel<SP>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    UMAPB_CUDA(cudaFuncSetAttribute(nd_iter_kernel<SP>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    const unsigned grid = static_cast<unsigned>(ceil_div(n, kWarps));
    int32_t* cur_i = out_idx;
    float* cur_d = out_dist;
    int32_t* nxt_i = idx_b.get();
    float* nxt_d = dist_b.get();
    p.new_idx = cur_i;
    p.new_dist = cur_d;
    cudaEvent_t e0, e1;
    UMAPB_CUDA(cudaEventCreate(&e0));
    UMAPB_CUDA(cudaEventCreate(&e1));
    float kernel_ms = 0.0f;
    UMAPB_CUDA(cudaEventRecord(e0, s));
    nd_init_kernel<SP><<<grid, kWarps * 32, smem, s>>>(p);
    UMAPB_LAUNCH_CHECK();
    UMAPB_CUDA(cudaEventRecord(e1, s));
    UMAPB_CUDA(cudaEventSynchronize(e1));
    {
        float ms = 0.0f;
        UMAPB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        kernel_ms += ms;
    }
    int64_t ran = 0;
    for (int64_t it = 0; it < n_iters; ++it) {
        UMAPB_CUDA(cudaMemsetAsync(changed.get(), 0, 4, s));
        p.old_idx = cur_i;
        p.old_dist = cur_d;
        p.new_idx = nxt_i;
        p.new_dist = nxt_d;
        UMAPB_CUDA(cudaEventRecord(e0, s));
        nd_iter_kernel<SP><<<grid, kWarps * 32, smem, s>>>(p, static_cast<uint64_t>(it + 1));
        UMAPB_LAUNCH_CHECK();
        UMAPB_CUDA(cudaEventRecord(e1, s));
        std::swap(cur_i, nxt_i);
        std::swap(cur_d, nxt_d);
        ran = it + 1;
        int h = 0;
        UMAPB_CUDA(cudaMemcpyAsync(&h, changed.get(), 4, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
        float ms = 0.0f;
        UMAPB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        kernel_ms += ms;
        if (!h) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        unsigned long long ev[kEvalSlots] = {};
        UMAPB_CUDA(cudaMemcpyAsync(ev, evaluated.get(), sizeof(ev), cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
        int64_t total = 0;
        for (int e = 0; e < kEvalSlots; ++e) total += static_cast<int64_t>(ev[e]);
        stats->candidates = total;
        stats->kernel_sec = kernel_ms * 1e-3;
    }
    if (cur_i != out_idx) {
        UMAPB_CUDA(cudaMemcpyAsync(out_idx, cur_i, n * k * 4, cudaMemcpyDeviceToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(out_dist, cur_d, n * k * 4, cudaMemcpyDeviceToDevice, s));
    }
    return ran;
}

// Candidate-rule sizes of approximate_nearest_neighbors_with_distance
// (lib.rs:3097-3098) and the shared-memory key capacity they need.
void nd_sizes(NdArgs& p, int64_t n, int k, int64_t candidate_pool) {
    const int64_t ck = std::max<int64_t>(candidate_pool, k);
    p.pool = static_cast<int>(std::min<int64_t>(ck, n - 1));
    p.maxc = static_cast<int>(ck * 4 + 1);
    p.expl = static_cast<int>(std::min<int64_t>(std::max<int64_t>(k / 2, 4), p.maxc));
    int cap = 32;
    const int need = std::max(k + k * k + 1 + p.expl, p.pool + 1);
    while (cap < need) cap <<= 1;
    p.cap = cap;
}

}  // namespace

int64_t nndescent(const float* X, int64_t n, int d, int k, int metric, int64_t candidate_pool,
                  int64_t n_iters, uint64_t seed, int32_t* out_idx, float* out_dist,
                  cudaStream_t s, NdStats* stats) {
    if (metric != UMAPB_METRIC_EUCLIDEAN && metric != UMAPB_METRIC_COSINE)
        invalid("the B200 NN-descent kernel supports metric euclidean and cosine");
    if (n < 2 || k < 1 || k >= n) invalid("NN-descent needs 1 <= k < n_rows");
    NdArgs p{};
    nd_sizes(p, n, k, candidate_pool);
    const size_t smem = static_cast<size_t>(kWarps) * nd_warp_smem(p.cap, d);
    if (smem > 200 * 1024)
        invalid("n_neighbors / n_features too large for the NN-descent kernel");
    DevBuf<float> norms;
    if (metric == UMAPB_METRIC_COSINE) {
        norms.alloc(n, s);
        row_norms(X, n, d, norms.get(), nullptr, s);
    }
    p.X = X;
    p.norms = norms.get();
    p.n = n;
    p.d = d;
    p.k = k;
    p.cosine = metric == UMAPB_METRIC_COSINE;
    p.metric = metric;
    p.seed = seed;
    return nndescent_run<false>(p, n, k, n_iters, smem, out_idx, out_dist, s, stats);
}

int64_t nndescent_csr(const CsrDevice& x, int k, int metric, int64_t candidate_pool,
                      int64_t n_iters, uint64_t seed, int32_t* out_idx, float* out_dist,
                      cudaStream_t s, NdStats* stats) {
    if (metric != UMAPB_METRIC_EUCLIDEAN && metric != UMAPB_METRIC_COSINE)
        invalid("the B200 sparse NN-descent supports metric euclidean and cosine");
    const int64_t n = x.n_rows;
    if (n < 2 || k < 1 || k >= n) invalid("NN-descent needs 1 <= k < n_rows");
    // the widest row bounds the query row kept in shared memory
    std::vector<int64_t> ptr(n + 1);
    UMAPB_CUDA(cudaMemcpyAsync(ptr.data(), x.indptr.get(), (n + 1) * 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    int64_t max_nnz = 1;
    for (int64_t i = 0; i < n; ++i) max_nnz = std::max(max_nnz, ptr[i + 1] - ptr[i]);
    NdArgs p{};
    nd_sizes(p, n, k, candidate_pool);
    const size_t smem =
        static_cast<size_t>(kWarps) * nd_warp_smem(p.cap, static_cast<int>(max_nnz), true);
    if (max_nnz > (1 << 20) || smem > 200 * 1024)
        invalid("rows with this many stored values are too wide for the sparse NN-descent kernel");
    p.csr.ptr = x.indptr.get();
    p.csr.idx = x.indices.get();
    p.csr.val = x.values.get();
    p.csr.sq = x.sq.get();
    p.csr.l2 = x.l2.get();
    p.csr.max_nnz = static_cast<int>(max_nnz);
    p.n = n;
    p.d = static_cast<int>(std::min<int64_t>(x.n_cols, 1 << 30));
    p.k = k;
    p.cosine = metric == UMAPB_METRIC_COSINE;
    p.metric = metric;
    p.seed = seed;
    return nndescent_run<true>(p, n, k, n_iters, smem, out_idx, out_dist, s, stats);
}

}  // namespace umapb
