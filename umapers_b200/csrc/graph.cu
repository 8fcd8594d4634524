// graph.cu - fuzzy simplicial set of the kNN graph on the device.
//
//  * smooth_knn: rust_umap/src/lib.rs:3424-3523 (one thread per row, FP32,
//    the reference's sequential summation order and expf).
//  * fuzzy_union: compute_membership_strengths (lib.rs:3525-3560) and
//    symmetrize_fuzzy_graph (lib.rs:3597-3649) as a sort-based merge: every
//    directed edge becomes a key (min, max, direction) packed in 64 bits, one
//    radix sort groups the two directions of a pair next to each other, a
//    merge pass forms w_ij + w_ji - w_ij*w_ji (set_op_mix_ratio blend), and a
//    second radix sort on (head, tail) emits both directions in CSR order.
//  * prune_edges (lib.rs:3804-3822) as a stable compaction.
#include <cub/cub.cuh>

#include <cfloat>
#include <climits>

#include <chrono>

#include "kernels.cuh"

namespace umapb {
namespace {

constexpr float SMOOTH_K_TOLERANCE = 1e-5f;  // lib.rs:19
constexpr float MIN_K_DIST_SCALE = 1e-3f;    // lib.rs:20

int bits_for(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) ++b;
    return b;
}

__global__ void include_self_kernel(const int32_t* __restrict__ idx,
                                    const float* __restrict__ dist, int64_t n, int k,
                                    int* __restrict__ flag) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (idx[i * k] != i || fabsf(dist[i * k]) > SMOOTH_K_TOLERANCE) atomicAnd(flag, 0);
}

// Sum and count of the distances smooth_knn_dist averages into
// `mean_distances` (lib.rs:3434-3446), accumulated in FP64.
__global__ void mean_dist_kernel(const float* __restrict__ dist, int64_t n, int k, int start,
                                 double* __restrict__ sum) {
    double acc = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        for (int c = start; c < k; ++c) acc += static_cast<double>(dist[i * k + c]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, acc);
}

__global__ void smooth_knn_kernel(const float* __restrict__ dist, int64_t n, int k, int start,
                                  float target, float local_conn, const double* __restrict__ gsum,
                                  double gcount, float* __restrict__ sigmas,
                                  float* __restrict__ rhos) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* row = dist + i * k;
    const int m = k - start;
    // non-zero distances in row order
    int nnz = 0;
    float mean_ith = 0.0f;
    if (m > 0) {
        float s = 0.0f;
        for (int c = start; c < k; ++c) s = __fadd_rn(s, row[c]);
        mean_ith = __fdiv_rn(s, static_cast<float>(m));
    }
    for (int c = start; c < k; ++c) nnz += row[c] > 0.0f;
    float rho = 0.0f;
    if (static_cast<float>(nnz) >= local_conn) {
        const int index = static_cast<int>(floorf(local_conn));
        const float interp = __fsub_rn(local_conn, static_cast<float>(index));
        // the index-th and (index+1)-th non-zero entries
        float nz_a = 0.0f, nz_b = 0.0f, nz_first = 0.0f;
        int seen = 0;
        for (int c = start; c < k; ++c) {
            const float v = row[c];
            if (v > 0.0f) {
                if (seen == 0) nz_first = v;
                if (seen == index - 1) nz_a = v;
                if (seen == index) nz_b = v;
                ++seen;
            }
        }
        if (index > 0) {
            rho = nz_a;
            if (interp > SMOOTH_K_TOLERANCE && index < nnz)
                rho = __fadd_rn(rho, __fmul_rn(interp, __fsub_rn(nz_b, nz_a)));
        } else if (nnz > 0) {
            rho = __fmul_rn(interp, nz_first);
        }
    } else if (nnz > 0) {
        float mx = -FLT_MAX;
        for (int c = start; c < k; ++c)
            if (row[c] > 0.0f) mx = fmaxf(mx, row[c]);
        rho = mx;
    }
    float lo = 0.0f, hi = INFINITY, mid = 1.0f;
    for (int it = 0; it < 64; ++it) {
        float psum = 0.0f;
        for (int c = start; c < k; ++c) {
            const float dd = __fsub_rn(row[c], rho);
            if (dd > 0.0f)
                psum = __fadd_rn(psum, expf(-__fdiv_rn(dd, mid)));
            else
                psum = __fadd_rn(psum, 1.0f);
        }
        if (fabsf(__fsub_rn(psum, target)) < SMOOTH_K_TOLERANCE) break;
        if (psum > target) {
            hi = mid;
            mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        } else {
            lo = mid;
            if (isinf(hi))
                mid = __fmul_rn(mid, 2.0f);
            else
                mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        }
    }
    float min_scale;
    if (rho > 0.0f) {
        min_scale = __fmul_rn(MIN_K_DIST_SCALE, mean_ith);
    } else if (gsum != nullptr) {
        const float mean_all = gcount > 0 ? static_cast<float>(*gsum / gcount) : 0.0f;
        min_scale = __fmul_rn(MIN_K_DIST_SCALE, mean_all);
    } else {
        // a request of this row alone: the FP64 sum of its own distances
        double acc = 0.0;
        for (int c = start; c < k; ++c) acc += static_cast<double>(row[c]);
        const float mean_row = m > 0 ? static_cast<float>(acc / static_cast<double>(m)) : 0.0f;
        min_scale = __fmul_rn(MIN_K_DIST_SCALE, mean_row);
    }
    sigmas[i] = fmaxf(mid, min_scale);
    rhos[i] = rho;
}

// membership weight of one (row, neighbour) entry (lib.rs:3541-3549)
__device__ inline float membership_weight(float d, float rho, float sigma) {
    const float t = __fsub_rn(d, rho);
    if (t <= 0.0f || sigma == 0.0f) return 1.0f;
    return expf(__fdiv_rn(-t, sigma));
}

// One key per directed edge: (min << (b+1)) | (max << 1) | (head > tail).
// Self edges and zero weights get the all-ones key and sort to the end.
__global__ void membership_keys_kernel(const int32_t* __restrict__ idx,
                                       const float* __restrict__ dist,
                                       const float* __restrict__ sig, const float* __restrict__ rho,
                                       int64_t n, int k, int b, uint64_t invalid_key,
                                       uint64_t* __restrict__ keys, float* __restrict__ vals,
                                       unsigned long long* __restrict__ n_valid) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool in_range = e < n * k;
    bool valid = false;
    if (in_range) {
    const int64_t i = e / k;
    const int64_t j = idx[e];
    float w = 0.0f;
    if (j != i) w = membership_weight(dist[e], rho[i], sig[i]);
    if (w > 0.0f && j != i) {
        const uint64_t lo = static_cast<uint64_t>(i < j ? i : j);
        const uint64_t hi = static_cast<uint64_t>(i < j ? j : i);
        keys[e] = (lo << (b + 1)) | (hi << 1) | static_cast<uint64_t>(i > j);
        valid = true;
    } else {
        keys[e] = invalid_key;
    }
    vals[e] = w;
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, valid);
    if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(n_valid, static_cast<unsigned long long>(__popc(ballot)));
}

// First entry of each (min,max) group merges w_ij / w_ji and, when the
// symmetric weight is positive, writes both directions as (head, tail) keys.
__global__ void merge_pairs_kernel(const uint64_t* __restrict__ keys,
                                   const float* __restrict__ vals, int64_t m, int b, float mix,
                                   int* __restrict__ count, uint64_t* __restrict__ out_keys,
                                   float* __restrict__ out_w) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= m) return;
    const uint64_t pair = keys[p] >> 1;
    if (p > 0 && (keys[p - 1] >> 1) == pair) return;
    float wij = 0.0f, wji = 0.0f;
    for (int64_t q = p; q < m && (keys[q] >> 1) == pair; ++q) {
        if ((keys[q] & 1) == 0) {
            if (vals[q] > 0.0f) wij = vals[q];
        } else {
            if (vals[q] > 0.0f) wji = vals[q];
        }
    }
    const float prod = __fmul_rn(wij, wji);
    const float sym = __fadd_rn(__fmul_rn(mix, __fsub_rn(__fadd_rn(wij, wji), prod)),
                                __fmul_rn(__fsub_rn(1.0f, mix), prod));
    if (sym > 0.0f) {
        const uint64_t mask = (uint64_t(1) << b) - 1;
        const uint64_t i = (pair >> b) & mask;
        const uint64_t j = pair & mask;
        const int at = atomicAdd(count, 2);
        out_keys[at] = (i << 32) | j;
        out_w[at] = sym;
        out_keys[at + 1] = (j << 32) | i;
        out_w[at + 1] = sym;
    }
}

__global__ void split_keys_kernel(const uint64_t* __restrict__ keys, int64_t m,
                                  int32_t* __restrict__ heads, int32_t* __restrict__ tails) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    heads[e] = static_cast<int32_t>(keys[e] >> 32);
    tails[e] = static_cast<int32_t>(keys[e] & 0xffffffffu);
}

__global__ void row_ptr_kernel(const int32_t* __restrict__ heads, int64_t m, int64_t n,
                               int32_t* __restrict__ row_ptr) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e > m) return;
    // row_ptr[h] = first edge with head >= h
    const int64_t hprev = e == 0 ? -1 : heads[e - 1];
    const int64_t hcur = e == m ? n : heads[e];
    for (int64_t h = hprev + 1; h <= hcur; ++h) row_ptr[h] = static_cast<int32_t>(e);
}

struct KeepFlag {
    const float* w;
    float thr;
    __device__ bool operator()(const int64_t& e) const { return w[e] >= thr && w[e] > 0.0f; }
};

// The same rule against each query's own threshold (row-local graphs).
struct RowKeepFlag {
    const float* w;
    const float* thr;  // per query
    int k;
    __device__ bool operator()(const int64_t& e) const {
        return w[e] >= thr[e / k] && w[e] > 0.0f;
    }
};

// Each query's largest weight and its prune threshold max / denom.
__global__ void row_max_kernel(const float* __restrict__ w, int64_t nq, int k, float denom,
                               float* __restrict__ row_max, float* __restrict__ thr) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    float mx = -INFINITY;
    for (int c = 0; c < k; ++c) mx = fmaxf(mx, w[i * k + c]);
    row_max[i] = mx;
    thr[i] = __fdiv_rn(mx, denom);
}

__global__ void bipartite_kernel(const int32_t* __restrict__ idx, const float* __restrict__ dist,
                                 const float* __restrict__ sig, const float* __restrict__ rho,
                                 int64_t nq, int k, float* __restrict__ w) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= nq * k) return;
    const int64_t i = e / k;
    w[e] = membership_weight(dist[e], rho[i], sig[i]);
}

__global__ void gather_edges_kernel(const int64_t* __restrict__ sel, int64_t m, int k,
                                    const int32_t* __restrict__ idx, const float* __restrict__ w,
                                    int32_t* __restrict__ heads, int32_t* __restrict__ tails,
                                    float* __restrict__ wout) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= m) return;
    const int64_t e = sel[p];
    heads[p] = static_cast<int32_t>(e / k);
    tails[p] = idx[e];
    wout[p] = w[e];
}

__global__ void gather_sel_kernel(const int64_t* __restrict__ sel, int64_t m,
                                  const int32_t* __restrict__ hin, const int32_t* __restrict__ tin,
                                  const float* __restrict__ win, int32_t* __restrict__ hout,
                                  int32_t* __restrict__ tout, float* __restrict__ wout) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= m) return;
    const int64_t e = sel[p];
    hout[p] = hin[e];
    tout[p] = tin[e];
    wout[p] = win[e];
}

// apply_categorical_target_intersection (lib.rs:3694-3731): each edge's
// weight times 1 (same label), exp(-1) (either label -1) or exp(-far_dist)
// (different labels), both scales computed on the host in FP32; a product
// that is not positive and finite drops the edge (0).  Every head's largest
// kept weight is kept as its bit pattern (positive floats order as uints).
__global__ void target_scale_kernel(const int32_t* __restrict__ heads,
                                    const int32_t* __restrict__ tails,
                                    const float* __restrict__ w, int64_t m,
                                    const int64_t* __restrict__ labels, float unknown_scale,
                                    float far_scale, float* __restrict__ scaled,
                                    unsigned* __restrict__ row_max) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int64_t lhs = labels[heads[e]], rhs = labels[tails[e]];
    const float scale = (lhs == -1 || rhs == -1) ? unknown_scale : (lhs != rhs ? far_scale : 1.0f);
    const float v = __fmul_rn(w[e], scale);
    const bool keep = v > 0.0f && isfinite(v);
    scaled[e] = keep ? v : 0.0f;
    if (keep) atomicMax(row_max + heads[e], __float_as_uint(v));
}

// reset_local_connectivity_edges (lib.rs:3733-3760): every kept edge divided
// by its head's largest kept weight, as a directed edge keyed for the fuzzy
// union (min << (b+1) | max << 1 | head > tail); dropped edges get the
// invalid key.
__global__ void target_keys_kernel(const int32_t* __restrict__ heads,
                                   const int32_t* __restrict__ tails,
                                   const float* __restrict__ scaled, int64_t m,
                                   const unsigned* __restrict__ row_max, int b,
                                   uint64_t invalid_key, uint64_t* __restrict__ keys,
                                   float* __restrict__ vals,
                                   unsigned long long* __restrict__ n_valid) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool valid = false;
    if (e < m) {
        const int64_t i = heads[e], j = tails[e];
        const float v = scaled[e];
        const float mx = __uint_as_float(row_max[i]);
        if (v > 0.0f && i != j && mx > 0.0f && isfinite(mx)) {
            const uint64_t lo = static_cast<uint64_t>(i < j ? i : j);
            const uint64_t hi = static_cast<uint64_t>(i < j ? j : i);
            keys[e] = (lo << (b + 1)) | (hi << 1) | static_cast<uint64_t>(i > j);
            vals[e] = __fdiv_rn(v, mx);
            valid = true;
        } else {
            keys[e] = invalid_key;
            vals[e] = 0.0f;
        }
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, valid);
    if ((threadIdx.x & 31) == 0 && ballot)
        atomicAdd(n_valid, static_cast<unsigned long long>(__popc(ballot)));
}

inline unsigned grid_for(int64_t n, int threads = 256) {
    return static_cast<unsigned>(ceil_div(std::max<int64_t>(n, 1), threads));
}

// Stable selection of the edges with w >= threshold && w > 0; returns the
// indices and the count.
template <typename Flag>
int64_t select_kept_if(int64_t m, Flag flag, DevBuf<int64_t>& sel, cudaStream_t s) {
    sel.alloc(std::max<int64_t>(m, 1), s);
    DevBuf<int64_t> nsel(1, s);
    cub::CountingInputIterator<int64_t> it(0);
    size_t tmp_bytes = 0;
    UMAPB_CUDA(cub::DeviceSelect::If(nullptr, tmp_bytes, it, sel.get(), nsel.get(), m, flag, s));
    DevBuf<unsigned char> tmp(tmp_bytes, s);
    UMAPB_CUDA(
        cub::DeviceSelect::If(tmp.get(), tmp_bytes, it, sel.get(), nsel.get(), m, flag, s));
    int64_t h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, nsel.get(), 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return h;
}

int64_t select_kept(const float* w, int64_t m, float thr, DevBuf<int64_t>& sel, cudaStream_t s) {
    return select_kept_if(m, KeepFlag{w, thr}, sel, s);
}

}  // namespace

bool knn_includes_self(const int32_t* idx, const float* dist, int64_t n, int k, cudaStream_t s) {
    DevBuf<int> flag(1, s);
    const int one = 1;
    UMAPB_CUDA(cudaMemcpyAsync(flag.get(), &one, 4, cudaMemcpyHostToDevice, s));
    if (n > 0 && k > 0) {
        include_self_kernel<<<grid_for(n), 256, 0, s>>>(idx, dist, n, k, flag.get());
        UMAPB_LAUNCH_CHECK();
    }
    int h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, flag.get(), 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return n > 0 && k > 0 && h != 0;
}

void smooth_knn(const float* dist, int64_t n, int k, float k_f, float local_conn, float bandwidth,
                bool include_self, float* sigmas, float* rhos, cudaStream_t s, bool row_local) {
    if (n == 0) return;
    const int start = (include_self && k > 0) ? 1 : 0;
    DevBuf<double> gsum;
    if (!row_local) {
        gsum.alloc(1, s);
        UMAPB_CUDA(cudaMemsetAsync(gsum.get(), 0, 8, s));
        const unsigned mb = static_cast<unsigned>(std::min<int64_t>(ceil_div(n, 256), 148 * 8));
        mean_dist_kernel<<<mb, 256, 0, s>>>(dist, n, k, start, gsum.get());
        UMAPB_LAUNCH_CHECK();
    }
    const float target = __builtin_log2f(k_f) * bandwidth;
    const double count = static_cast<double>(n) * (k - start);
    smooth_knn_kernel<<<grid_for(n, 128), 128, 0, s>>>(dist, n, k, start, target, local_conn,
                                                       gsum.get(), count, sigmas, rhos);
    UMAPB_LAUNCH_CHECK();
}

float max_weight(const float* w, int64_t n, cudaStream_t s) {
    if (n == 0) return -INFINITY;
    DevBuf<float> out(1, s);
    size_t tmp_bytes = 0;
    UMAPB_CUDA(cub::DeviceReduce::Max(nullptr, tmp_bytes, w, out.get(), n, s));
    DevBuf<unsigned char> tmp(tmp_bytes, s);
    UMAPB_CUDA(cub::DeviceReduce::Max(tmp.get(), tmp_bytes, w, out.get(), n, s));
    float h = 0.0f;
    UMAPB_CUDA(cudaMemcpyAsync(&h, out.get(), 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return h;
}

void build_row_ptr(const int32_t* heads, int64_t m, int64_t n, int32_t* row_ptr, cudaStream_t s) {
    row_ptr_kernel<<<grid_for(m + 1), 256, 0, s>>>(heads, m, n, row_ptr);
    UMAPB_LAUNCH_CHECK();
}

void fuzzy_union(const int32_t* idx, const float* dist, const float* sigmas, const float* rhos,
                 int64_t n, int k, float mix, int64_t n_epochs, Graph& g, cudaStream_t s,
                 double* phase_sec, const CategoricalTarget* target) {
    // phase clock of FitTimingBreakdown's membership / symmetrize / prune
    // fields (lib.rs:51-68); it synchronises only when asked for
    auto t_last = std::chrono::steady_clock::now();
    auto phase = [&](int i) {
        if (!phase_sec) return;
        UMAPB_CUDA(cudaStreamSynchronize(s));
        const auto t = std::chrono::steady_clock::now();
        phase_sec[i] = std::chrono::duration<double>(t - t_last).count();
        t_last = t;
    };
    const int64_t m = n * k;
    const int b = bits_for(n);
    const int key_bits = 2 * b + 1;
    const uint64_t invalid_key = (key_bits >= 64) ? ~0ULL : ((uint64_t(1) << key_bits) - 1);
    // The symmetric graph: (head << 32 | tail) keys sorted, weights, heads, tails.
    DevBuf<uint64_t> sym_keys2;
    DevBuf<float> sym_w2;
    DevBuf<int32_t> heads, tails;
    int n_sym = 0;
    // symmetrize_fuzzy_graph (lib.rs:3597-3649) of `mm` directed edges given
    // as (min, max, head > tail) keys (invalid ones sort last, `nv` counts the
    // rest): sort, merge each pair, sort by (head, tail), split.
    auto union_keys = [&](DevBuf<uint64_t>& kin, DevBuf<float>& vin, int64_t mm,
                          DevBuf<unsigned long long>& nv, float mixv, bool timed) {
        DevBuf<uint64_t> ksorted(mm, s);
        DevBuf<float> vsorted(mm, s);
        {
            size_t tmp_bytes = 0;
            UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kin.get(),
                                                       ksorted.get(), vin.get(), vsorted.get(),
                                                       mm, 0, key_bits, s));
            DevBuf<unsigned char> tmp(tmp_bytes, s);
            UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, kin.get(),
                                                       ksorted.get(), vin.get(), vsorted.get(),
                                                       mm, 0, key_bits, s));
        }
        if (timed) phase(0);
        DevBuf<int> cnt(1, s);
        UMAPB_CUDA(cudaMemsetAsync(cnt.get(), 0, 4, s));
        DevBuf<uint64_t> sym_keys(2 * mm + 2, s);
        DevBuf<float> sym_w(2 * mm + 2, s);
        sym_keys2.alloc(2 * mm + 2, s);
        sym_w2.alloc(2 * mm + 2, s);
        // valid keys form the sorted prefix
        unsigned long long valid_h = 0;
        UMAPB_CUDA(cudaMemcpyAsync(&valid_h, nv.get(), 8, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
        const int64_t valid = static_cast<int64_t>(valid_h);
        if (valid > 0) {
            merge_pairs_kernel<<<grid_for(valid), 256, 0, s>>>(ksorted.get(), vsorted.get(), valid,
                                                               b, mixv, cnt.get(), sym_keys.get(),
                                                               sym_w.get());
            UMAPB_LAUNCH_CHECK();
        }
        UMAPB_CUDA(cudaMemcpyAsync(&n_sym, cnt.get(), 4, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
        if (n_sym > 0) {
            size_t tmp_bytes = 0;
            const int end_bit = 32 + b;
            UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, sym_keys.get(),
                                                       sym_keys2.get(), sym_w.get(), sym_w2.get(),
                                                       n_sym, 0, end_bit, s));
            DevBuf<unsigned char> tmp(tmp_bytes, s);
            UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, sym_keys.get(),
                                                       sym_keys2.get(), sym_w.get(), sym_w2.get(),
                                                       n_sym, 0, end_bit, s));
        }
        heads.alloc(std::max(n_sym, 1), s);
        tails.alloc(std::max(n_sym, 1), s);
        if (n_sym > 0) {
            split_keys_kernel<<<grid_for(n_sym), 256, 0, s>>>(sym_keys2.get(), n_sym, heads.get(),
                                                              tails.get());
            UMAPB_LAUNCH_CHECK();
        }
    };
    {
        DevBuf<uint64_t> keys(m, s);
        DevBuf<float> vals(m, s);
        DevBuf<unsigned long long> nvalid(1, s);
        UMAPB_CUDA(cudaMemsetAsync(nvalid.get(), 0, 8, s));
        membership_keys_kernel<<<grid_for(m), 256, 0, s>>>(idx, dist, sigmas, rhos, n, k, b,
                                                           invalid_key, keys.get(), vals.get(),
                                                           nvalid.get());
        UMAPB_LAUNCH_CHECK();
        union_keys(keys, vals, m, nvalid, mix, true);
    }
    if (target != nullptr && target->weight > 0.0f && n_sym > 0) {
        // apply_categorical_target_intersection (lib.rs:1426-1431, 3694-3760):
        // label-scaled weights, each head's row divided by its largest kept
        // weight, and the fuzzy union of those directed edges with mix 1
        DevBuf<float> scaled(n_sym, s);
        DevBuf<unsigned> row_max(n, s);
        UMAPB_CUDA(cudaMemsetAsync(row_max.get(), 0, n * 4, s));
        target_scale_kernel<<<grid_for(n_sym), 256, 0, s>>>(
            heads.get(), tails.get(), sym_w2.get(), n_sym, target->labels, target->unknown_scale,
            target->far_scale, scaled.get(), row_max.get());
        UMAPB_LAUNCH_CHECK();
        DevBuf<uint64_t> keys(n_sym, s);
        DevBuf<float> vals(n_sym, s);
        DevBuf<unsigned long long> nvalid(1, s);
        UMAPB_CUDA(cudaMemsetAsync(nvalid.get(), 0, 8, s));
        target_keys_kernel<<<grid_for(n_sym), 256, 0, s>>>(heads.get(), tails.get(), scaled.get(),
                                                           n_sym, row_max.get(), b, invalid_key,
                                                           keys.get(), vals.get(), nvalid.get());
        UMAPB_LAUNCH_CHECK();
        union_keys(keys, vals, n_sym, nvalid, 1.0f, false);
    }
    g.n = n;
    phase(1);
    if (n_epochs > 0 && n_sym > 0) {
        // prune_edges (lib.rs:3804-3822)
        const float mx = max_weight(sym_w2.get(), n_sym, s);
        const float denom = n_epochs > 10 ? static_cast<float>(n_epochs) : 500.0f;
        const float thr = mx / denom;
        DevBuf<int64_t> sel;
        const int64_t kept = select_kept(sym_w2.get(), n_sym, thr, sel, s);
        g.heads.alloc(std::max<int64_t>(kept, 1), s);
        g.tails.alloc(std::max<int64_t>(kept, 1), s);
        g.weights.alloc(std::max<int64_t>(kept, 1), s);
        if (kept > 0) {
            gather_sel_kernel<<<grid_for(kept), 256, 0, s>>>(sel.get(), kept, heads.get(),
                                                             tails.get(), sym_w2.get(),
                                                             g.heads.get(), g.tails.get(),
                                                             g.weights.get());
            UMAPB_LAUNCH_CHECK();
        }
        g.n_edges = kept;
    } else {
        g.heads = std::move(heads);
        g.tails = std::move(tails);
        g.weights = std::move(sym_w2);
        g.n_edges = n_sym;
    }
    g.row_ptr.alloc(n + 1, s);
    build_row_ptr(g.heads.get(), g.n_edges, n, g.row_ptr.get(), s);
    phase(2);
}

void bipartite_graph(const int32_t* idx, const float* dist, const float* sigmas,
                     const float* rhos, int64_t nq, int k, int64_t n_epochs, Graph& g,
                     cudaStream_t s, bool row_local) {
    const int64_t m = nq * k;
    DevBuf<float> w(std::max<int64_t>(m, 1), s);
    g.n = nq;
    if (m == 0) {
        g.n_edges = 0;
        g.row_ptr.alloc(nq + 1, s);
        UMAPB_CUDA(cudaMemsetAsync(g.row_ptr.get(), 0, (nq + 1) * 4, s));
        return;
    }
    bipartite_kernel<<<grid_for(m), 256, 0, s>>>(idx, dist, sigmas, rhos, nq, k, w.get());
    UMAPB_LAUNCH_CHECK();
    const float denom = n_epochs > 10 ? static_cast<float>(n_epochs) : 500.0f;
    DevBuf<int64_t> sel;
    int64_t kept = 0;
    if (row_local) {
        DevBuf<float> thr(nq, s);
        g.row_max.alloc(nq, s);
        row_max_kernel<<<grid_for(nq), 256, 0, s>>>(w.get(), nq, k, denom, g.row_max.get(),
                                                    thr.get());
        UMAPB_LAUNCH_CHECK();
        kept = select_kept_if(m, RowKeepFlag{w.get(), thr.get(), k}, sel, s);
    } else {
        const float mx = max_weight(w.get(), m, s);
        kept = select_kept(w.get(), m, mx / denom, sel, s);
    }
    g.heads.alloc(std::max<int64_t>(kept, 1), s);
    g.tails.alloc(std::max<int64_t>(kept, 1), s);
    g.weights.alloc(std::max<int64_t>(kept, 1), s);
    if (kept > 0) {
        gather_edges_kernel<<<grid_for(kept), 256, 0, s>>>(sel.get(), kept, k, idx, w.get(),
                                                           g.heads.get(), g.tails.get(),
                                                           g.weights.get());
        UMAPB_LAUNCH_CHECK();
    }
    g.n_edges = kept;
    g.row_ptr.alloc(nq + 1, s);
    build_row_ptr(g.heads.get(), kept, nq, g.row_ptr.get(), s);
}

}  // namespace umapb
