// knn_sparse.cu - exact kNN of CSR rows (rust_umap/src/sparse.rs:605-657,
// 753-910) for the euclidean and cosine metrics, with the reference's result
// bit for bit.
//
// The reference scores every pair (i, j) from its sparse dot product
// (sparse_dot, sparse.rs:220-239: products of the shared columns summed in
// ascending column order, FP32) and the rows' norms (SparseCsrMatrix::new,
// sparse.rs:90-97: sum of v * v in stored order, and its square root):
//     euclidean  sqrt(max((|x|^2 + |y|^2) - 2 dot, 0))
//     cosine     1 - clamp(dot / (|x| |y|), -1, 1)   (0 if both norms are 0,
//                1 if one is)
// and keeps the k smallest (distance, index) keys.  A row that shares no
// stored column with the query has dot = +0.0 exactly.
//
// Here one warp serves one query row:
// 1. Touched rows.  The reference rows are regrouped once into tiles of 2048
//    rows, and within a tile by column (CSC order, rows ascending).  For each
//    tile the warp walks the query's columns in ascending order and adds
//    q_c * v_jc into a per-warp shared-memory accumulator of the tile's rows.
//    Every row's products therefore arrive in ascending column order, the
//    reference's summation order.  The first entries of four columns are
//    loaded together, and rows touched for the first time are appended to a
//    per-warp list.  The list is then walked once: each touched row's dot
//    becomes a distance, its key is offered to the warp's sorted list of the
//    32 smallest keys, and its accumulator entry is reset.
// 2. Untouched rows (dot = 0).  Their distances depend only on the other
//    row's norm: cosine gives 1 for all of them (or 0 / 1 for an empty
//    query), euclidean sqrt(|x|^2 + |y|^2), non-decreasing in |y|^2.  The
//    warp walks the rows in index order (cosine) or in (squared norm, index)
//    order (euclidean), skips rows that share a column with the query, and
//    stops once no later row can enter the full list.
// In the self join a row's distance to itself is 0, as in the reference.
#include <cub/cub.cuh>

#include <algorithm>

#include "kernels.cuh"

namespace umapb {
namespace {

constexpr int kTileRows = 2048;             // reference rows per accumulator tile
constexpr int kTileShift = 11;
constexpr int kWarps = 16;                  // warps (queries in flight) per block
constexpr int kList = 32;                   // list length: k <= 32
constexpr uint32_t kUnset = 0x7fc00001u;    // accumulator entry not touched yet

__device__ __forceinline__ float csr_distance_from_dot(float dot, float q_sq, float q_l2,
                                                       float r_sq, float r_l2, int metric) {
    if (metric == UMAPB_METRIC_COSINE) {
        if (q_l2 == 0.0f && r_l2 == 0.0f) return 0.0f;
        if (q_l2 == 0.0f || r_l2 == 0.0f) return 1.0f;
        float c = __fdiv_rn(dot, __fmul_rn(q_l2, r_l2));
        if (c < -1.0f) c = -1.0f;
        else if (c > 1.0f) c = 1.0f;
        return __fsub_rn(1.0f, c);
    }
    float t = __fsub_rn(__fadd_rn(q_sq, r_sq), __fmul_rn(2.0f, dot));
    if (!(t > 0.0f)) t = 0.0f;
    return __fsqrt_rn(t);
}

__device__ __forceinline__ uint64_t warp_sort_keys(uint64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const uint64_t o = __shfl_xor_sync(0xffffffffu, v, stride);
            const bool up = (lane & size) == 0;
            const bool lower = (lane & stride) == 0;
            v = (lower == up) ? (v < o ? v : o) : (v < o ? o : v);
        }
    }
    return v;
}

// The 32 smallest of a sorted list (one key per lane, ascending) and 32 new
// keys (any order): sort the new keys, reverse them, take lane-wise minima
// (a bitonic sequence) and sort that in five stages.
__device__ __forceinline__ uint64_t warp_merge(uint64_t list, uint64_t keys) {
    const int lane = threadIdx.x & 31;
    const uint64_t srt = warp_sort_keys(keys);
    const uint64_t rev = __shfl_sync(0xffffffffu, srt, 31 - lane);
    uint64_t m = list < rev ? list : rev;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
        const uint64_t o = __shfl_xor_sync(0xffffffffu, m, st);
        m = (lane & st) ? (m > o ? m : o) : (m < o ? m : o);
    }
    return m;
}

// Offers one key per lane (~0 for none) to the warp's list.
__device__ __forceinline__ void offer(uint64_t& list, uint64_t key) {
    const uint64_t tau = __shfl_sync(0xffffffffu, list, kList - 1);
    unsigned q = __ballot_sync(0xffffffffu, key < tau);
    if (!q) return;
    if (__popc(q) >= 6) {
        list = warp_merge(list, key < tau ? key : ~0ull);
        return;
    }
    const int lane = threadIdx.x & 31;
    while (q) {
        const int b = __ffs(q) - 1;
        q &= q - 1;
        const uint64_t k = __shfl_sync(0xffffffffu, key, b);
        if (!(k < __shfl_sync(0xffffffffu, list, kList - 1))) continue;
        const int pos = __popc(__ballot_sync(0xffffffffu, list < k));
        const uint64_t up = __shfl_up_sync(0xffffffffu, list, 1);
        if (lane > pos)
            list = up;
        else if (lane == pos)
            list = k;
    }
}

// True when row j of r stores a column that query row i of q stores too.
__device__ __forceinline__ bool shares_column(const int64_t* __restrict__ qptr,
                                              const int32_t* __restrict__ qidx, int64_t i,
                                              const int64_t* __restrict__ rptr,
                                              const int32_t* __restrict__ ridx, int64_t j) {
    int64_t a = qptr[i], ae = qptr[i + 1], b = rptr[j], be = rptr[j + 1];
    while (a < ae && b < be) {
        const int32_t ca = qidx[a], cb = ridx[b];
        if (ca == cb) return true;
        if (ca < cb)
            ++a;
        else
            ++b;
    }
    return false;
}

struct SparseArgs {
    // queries
    const int64_t* qptr;
    const int32_t* qidx;
    const float* qval;
    const float* qsq;
    const float* ql2;
    int64_t nq;
    // reference rows
    const int64_t* rptr;
    const int32_t* ridx;
    const float* rsq;
    const float* rl2;
    int64_t nr;
    int64_t n_cols;
    // reference regrouped by (row tile, column)
    const int64_t* tile_colptr;  // n_tiles * n_cols + 1
    const int32_t* tile_rows;    // row within its tile
    const float* tile_vals;
    int64_t n_tiles;
    const int32_t* norm_order;   // rows by (squared norm, index)
    int k, metric, self;
    int32_t* out_idx;
    float* out_dist;
};

// Adds q * v of one stored entry (valid lanes) into the warp's accumulator and
// appends rows touched for the first time to the warp's list of touched rows.
__device__ __forceinline__ void accumulate(float* acc, uint16_t* touched, int& n_touched,
                                           bool valid, int32_t jl, float prod) {
    bool first = false;
    if (valid) {
        const float a = acc[jl];
        first = __float_as_uint(a) == kUnset;
        acc[jl] = __fadd_rn(first ? 0.0f : a, prod);
    }
    const unsigned m = __ballot_sync(0xffffffffu, first);
    if (first)
        touched[n_touched + __popc(m & ((1u << (threadIdx.x & 31)) - 1u))] =
            static_cast<uint16_t>(jl);
    n_touched += __popc(m);
}

constexpr int kColBatch = 4;   // query columns whose first entries load together
constexpr int kEvalBatch = 4;  // chunks of touched rows whose norms load together

__global__ void __launch_bounds__(kWarps * 32) knn_sparse_kernel(SparseArgs p) {
    extern __shared__ float acc_all[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* acc = acc_all + warp * kTileRows;
    uint16_t* touched = reinterpret_cast<uint16_t*>(acc_all + kWarps * kTileRows) + warp * kTileRows;
    for (int j = lane; j < kTileRows; j += 32) acc[j] = __uint_as_float(kUnset);
    __syncwarp();
    const int64_t wstride = static_cast<int64_t>(gridDim.x) * kWarps;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kWarps + warp; i < p.nq; i += wstride) {
        const int64_t q0 = p.qptr[i], q1 = p.qptr[i + 1];
        const float qsq = p.qsq[i], ql2 = p.ql2[i];
        uint64_t list = ~0ull;
        // the self pair (distance 0, not from the formula)
        if (p.self) offer(list, lane == 0 ? knn_key(0.0f, static_cast<uint32_t>(i)) : ~0ull);
        // ---- 1. rows sharing a column with the query, tile by tile
        for (int64_t t = 0; t < p.n_tiles; ++t) {
            const int64_t* cp = p.tile_colptr + t * p.n_cols;
            int n_touched = 0;
            for (int64_t e0 = q0; e0 < q1; e0 += 32) {
                const int ne = static_cast<int>(q1 - e0 < 32 ? q1 - e0 : 32);
                // lane u holds query column u of this chunk: value and entry range
                int64_t mb0 = 0, mb1 = 0;
                float mqv = 0.0f;
                if (lane < ne) {
                    const int32_t c = p.qidx[e0 + lane];
                    mqv = p.qval[e0 + lane];
                    mb0 = cp[c];
                    mb1 = cp[c + 1];
                }
                for (int ub = 0; ub < ne; ub += kColBatch) {
                    // the first 32 entries of kColBatch columns load together; the
                    // products still enter the accumulator in column order
                    int32_t jl[kColBatch];
                    float pv[kColBatch], qv[kColBatch];
                    bool ok[kColBatch];
                    int64_t b0[kColBatch], b1[kColBatch];
#pragma unroll
                    for (int r = 0; r < kColBatch; ++r) {
                        const int u = ub + r < ne ? ub + r : ne - 1;
                        b0[r] = __shfl_sync(0xffffffffu, mb0, u);
                        b1[r] = __shfl_sync(0xffffffffu, mb1, u);
                        qv[r] = __shfl_sync(0xffffffffu, mqv, u);
                        const int64_t b = b0[r] + lane;
                        ok[r] = ub + r < ne && b < b1[r];
                        jl[r] = 0;
                        pv[r] = 0.0f;
                        if (ok[r]) {
                            jl[r] = p.tile_rows[b];
                            pv[r] = p.tile_vals[b];
                        }
                    }
#pragma unroll
                    for (int r = 0; r < kColBatch; ++r) {
                        if (ub + r >= ne) break;
                        accumulate(acc, touched, n_touched, ok[r], jl[r],
                                   __fmul_rn(qv[r], pv[r]));
                        for (int64_t base = b0[r] + 32; base < b1[r]; base += 32) {
                            const int64_t b = base + lane;
                            const bool v = b < b1[r];
                            const int32_t j2 = v ? p.tile_rows[b] : 0;
                            const float x2 = v ? p.tile_vals[b] : 0.0f;
                            accumulate(acc, touched, n_touched, v, j2, __fmul_rn(qv[r], x2));
                        }
                        __syncwarp();
                    }
                }
            }
            // every touched row: its distance, its key offered, its entry reset;
            // the norms of kEvalBatch chunks of 32 rows load together
            const int64_t row0 = t << kTileShift;
            const bool cosine = p.metric == UMAPB_METRIC_COSINE;
            for (int base = 0; base < n_touched; base += 32 * kEvalBatch) {
                float dot[kEvalBatch], nrm[kEvalBatch];
                int64_t jj[kEvalBatch];
#pragma unroll
                for (int r = 0; r < kEvalBatch; ++r) {
                    const int at = base + 32 * r + lane;
                    jj[r] = -1;
                    dot[r] = 0.0f;
                    nrm[r] = 0.0f;
                    if (at < n_touched) {
                        const int32_t jl = touched[at];
                        dot[r] = acc[jl];
                        acc[jl] = __uint_as_float(kUnset);
                        jj[r] = row0 + jl;
                        nrm[r] = cosine ? p.rl2[jj[r]] : p.rsq[jj[r]];
                    }
                }
#pragma unroll
                for (int r = 0; r < kEvalBatch; ++r) {
                    if (base + 32 * r >= n_touched) break;
                    uint64_t key = ~0ull;
                    if (jj[r] >= 0 && !(p.self && jj[r] == i)) {
                        const float d = cosine ? csr_distance_from_dot(dot[r], qsq, ql2, 0.0f,
                                                                       nrm[r], p.metric)
                                               : csr_distance_from_dot(dot[r], qsq, ql2, nrm[r],
                                                                       0.0f, p.metric);
                        key = knn_key(d, static_cast<uint32_t>(jj[r]));
                    }
                    offer(list, key);
                }
            }
            __syncwarp();
        }
        // ---- 2. rows sharing no column with the query (dot = +0.0)
        const bool by_norm = p.metric != UMAPB_METRIC_COSINE;
        const bool empty_cos = !by_norm && ql2 == 0.0f;
        for (int64_t base = 0; base < p.nr; base += 32) {
            const int64_t pos = base + lane;
            uint64_t key = ~0ull;
            float bound = 0.0f;  // the untouched distance at this position
            if (pos < p.nr) {
                const int64_t j = by_norm ? p.norm_order[pos] : pos;
                bound = csr_distance_from_dot(0.0f, qsq, ql2, p.rsq[j], p.rl2[j], p.metric);
                if (!(p.self && j == i) &&
                    (q0 == q1 || !shares_column(p.qptr, p.qidx, i, p.rptr, p.ridx, j)))
                    key = knn_key(bound, static_cast<uint32_t>(j));
            }
            offer(list, key);
            // Stop once no later row can enter the full list: in norm order
            // a later row's untouched distance is at least this block's
            // last; for cosine every untouched distance is 1 and later
            // indices are larger (an empty query can still meet distance-0
            // rows anywhere, so it walks all rows).
            const int64_t last = base + 31 < p.nr ? base + 31 : p.nr - 1;
            const uint64_t tau = __shfl_sync(0xffffffffu, list, kList - 1);
            const float dlast = __shfl_sync(0xffffffffu, bound, static_cast<int>(last - base));
            if (tau == ~0ull || empty_cos) continue;
            if (by_norm ? key_dist(tau) < dlast : tau < knn_key(1.0f, static_cast<uint32_t>(last)))
                break;
        }
        if (lane < p.k) {
            p.out_idx[i * p.k + lane] = static_cast<int32_t>(key_index(list));
            p.out_dist[i * p.k + lane] = key_dist(list);
        }
    }
}

__global__ void csr_norms_kernel(const int64_t* __restrict__ ptr, const float* __restrict__ val,
                                 int64_t n, float* __restrict__ sq, float* __restrict__ l2) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float s = 0.0f;
    for (int64_t e = ptr[r]; e < ptr[r + 1]; ++e) s = __fadd_rn(s, __fmul_rn(val[e], val[e]));
    sq[r] = s;
    l2[r] = __fsqrt_rn(s);
}

// Sort key of every stored entry: (row tile, column), entries in row order.
__global__ void tile_keys_kernel(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                 int64_t n, int64_t n_cols, int64_t* __restrict__ keys,
                                 int64_t* __restrict__ ids) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int64_t t = r >> kTileShift;
    for (int64_t e = ptr[r]; e < ptr[r + 1]; ++e) {
        keys[e] = t * n_cols + idx[e];
        ids[e] = e;
    }
}

__global__ void entry_row_kernel(const int64_t* __restrict__ ptr, int64_t n,
                                 int32_t* __restrict__ row_of) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    for (int64_t e = ptr[r]; e < ptr[r + 1]; ++e) row_of[e] = static_cast<int32_t>(r);
}

__global__ void tile_gather_kernel(const int64_t* __restrict__ order,
                                   const int32_t* __restrict__ row_of,
                                   const float* __restrict__ val, int64_t nnz,
                                   int32_t* __restrict__ rows, float* __restrict__ vals) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    const int64_t e = order[p];
    rows[p] = row_of[e] & (kTileRows - 1);
    vals[p] = val[e];
}

// tile_colptr[key] = first sorted position whose key is >= key.
__global__ void key_bounds_kernel(const int64_t* __restrict__ sorted_keys, int64_t nnz,
                                  int64_t n_keys, int64_t* __restrict__ colptr) {
    const int64_t key = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (key > n_keys) return;
    int64_t lo = 0, hi = nnz;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (sorted_keys[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    colptr[key] = lo;
}

__global__ void norm_keys_kernel(const float* __restrict__ sq, int64_t n,
                                 uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    keys[r] = knn_key(sq[r], static_cast<uint32_t>(r));
    ids[r] = static_cast<int32_t>(r);
}

// Nonzeros of each dense row (one warp per row).
__global__ void dense_nnz_kernel(const float* __restrict__ X, int64_t n, int64_t d,
                                 int64_t* __restrict__ cnt) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    int c = 0;
    for (int64_t f = lane; f < d; f += 32) c += X[row * d + f] != 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[row] = c;
}

// The nonzeros of each dense row in column order (one warp per row).
__global__ void dense_fill_kernel(const float* __restrict__ X, int64_t n, int64_t d,
                                  const int64_t* __restrict__ ptr, int32_t* __restrict__ idx,
                                  float* __restrict__ val) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    int64_t o = ptr[row];
    for (int64_t base = 0; base < d; base += 32) {
        const int64_t f = base + lane;
        const float v = f < d ? X[row * d + f] : 0.0f;
        const bool nz = f < d && v != 0.0f;
        const unsigned m = __ballot_sync(0xffffffffu, nz);
        if (nz) {
            const int64_t at = o + __popc(m & ((1u << lane) - 1u));
            idx[at] = static_cast<int32_t>(f);
            val[at] = v;
        }
        o += __popc(m);
    }
}

inline unsigned blocks_for(int64_t n, int t = 256) {
    return static_cast<unsigned>(ceil_div(std::max<int64_t>(n, 1), t));
}

}  // namespace

void csr_upload(const int64_t* indptr, const int64_t* indices, const float* values,
                int64_t n_rows, int64_t n_cols, CsrDevice& out, cudaStream_t s) {
    const int64_t nnz = indptr[n_rows];
    out.n_rows = n_rows;
    out.n_cols = n_cols;
    out.nnz = nnz;
    out.indptr.alloc(n_rows + 1, s);
    UMAPB_CUDA(cudaMemcpyAsync(out.indptr.get(), indptr, (n_rows + 1) * 8, cudaMemcpyHostToDevice,
                               s));
    std::vector<int32_t> idx32(static_cast<size_t>(nnz));
    for (int64_t e = 0; e < nnz; ++e) idx32[e] = static_cast<int32_t>(indices[e]);
    out.indices.alloc(std::max<int64_t>(nnz, 1), s);
    out.values.alloc(std::max<int64_t>(nnz, 1), s);
    if (nnz > 0) {
        UMAPB_CUDA(cudaMemcpyAsync(out.indices.get(), idx32.data(), nnz * 4,
                                   cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(out.values.get(), values, nnz * 4, cudaMemcpyHostToDevice, s));
    }
    out.sq.alloc(std::max<int64_t>(n_rows, 1), s);
    out.l2.alloc(std::max<int64_t>(n_rows, 1), s);
    if (n_rows > 0) {
        csr_norms_kernel<<<blocks_for(n_rows), 256, 0, s>>>(out.indptr.get(), out.values.get(),
                                                            n_rows, out.sq.get(), out.l2.get());
        UMAPB_LAUNCH_CHECK();
    }
    // the host copy of the indices must outlive the copy that reads it
    UMAPB_CUDA(cudaStreamSynchronize(s));
}

void csr_from_dense(const float* X, int64_t n, int64_t d, CsrDevice& out, cudaStream_t s) {
    out.n_rows = n;
    out.n_cols = d;
    DevBuf<int64_t> cnt(n + 1, s);
    UMAPB_CUDA(cudaMemsetAsync(cnt.get(), 0, (n + 1) * 8, s));
    if (n > 0) {
        dense_nnz_kernel<<<blocks_for(n * 32), 256, 0, s>>>(X, n, d, cnt.get());
        UMAPB_LAUNCH_CHECK();
    }
    out.indptr.alloc(n + 1, s);
    size_t tmp_bytes = 0;
    UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.get(), out.indptr.get(),
                                             n + 1, s));
    DevBuf<unsigned char> tmp(tmp_bytes, s);
    UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmp_bytes, cnt.get(), out.indptr.get(),
                                             n + 1, s));
    int64_t nnz = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&nnz, out.indptr.get() + n, 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    out.nnz = nnz;
    out.indices.alloc(std::max<int64_t>(nnz, 1), s);
    out.values.alloc(std::max<int64_t>(nnz, 1), s);
    out.sq.alloc(std::max<int64_t>(n, 1), s);
    out.l2.alloc(std::max<int64_t>(n, 1), s);
    if (n > 0) {
        dense_fill_kernel<<<blocks_for(n * 32), 256, 0, s>>>(X, n, d, out.indptr.get(),
                                                             out.indices.get(), out.values.get());
        UMAPB_LAUNCH_CHECK();
        csr_norms_kernel<<<blocks_for(n), 256, 0, s>>>(out.indptr.get(), out.values.get(), n,
                                                       out.sq.get(), out.l2.get());
        UMAPB_LAUNCH_CHECK();
    }
}

void csr_index(const CsrDevice& r, CsrIndex& out, cudaStream_t s) {
    const int64_t n = r.n_rows, nnz = r.nnz;
    out.n_tiles = ceil_div(std::max<int64_t>(n, 1), kTileRows);
    const int64_t n_keys = out.n_tiles * r.n_cols;
    DevBuf<int64_t> keys(std::max<int64_t>(nnz, 1), s), keys2(std::max<int64_t>(nnz, 1), s);
    DevBuf<int64_t> ids(std::max<int64_t>(nnz, 1), s), order(std::max<int64_t>(nnz, 1), s);
    DevBuf<int32_t> row_of(std::max<int64_t>(nnz, 1), s);
    out.tile_rows.alloc(std::max<int64_t>(nnz, 1), s);
    out.tile_vals.alloc(std::max<int64_t>(nnz, 1), s);
    out.tile_colptr.alloc(n_keys + 1, s);
    if (nnz > 0) {
        tile_keys_kernel<<<blocks_for(n), 256, 0, s>>>(r.indptr.get(), r.indices.get(), n, r.n_cols,
                                                       keys.get(), ids.get());
        UMAPB_LAUNCH_CHECK();
        entry_row_kernel<<<blocks_for(n), 256, 0, s>>>(r.indptr.get(), n, row_of.get());
        UMAPB_LAUNCH_CHECK();
        int bits = 1;
        while ((static_cast<int64_t>(1) << bits) <= n_keys) ++bits;
        size_t tmp_bytes = 0;
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.get(), keys2.get(),
                                                   ids.get(), order.get(), nnz, 0, bits, s));
        DevBuf<unsigned char> tmp(tmp_bytes, s);
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, keys.get(), keys2.get(),
                                                   ids.get(), order.get(), nnz, 0, bits, s));
        tile_gather_kernel<<<blocks_for(nnz), 256, 0, s>>>(order.get(), row_of.get(),
                                                           r.values.get(), nnz,
                                                           out.tile_rows.get(),
                                                           out.tile_vals.get());
        UMAPB_LAUNCH_CHECK();
    }
    key_bounds_kernel<<<blocks_for(n_keys + 1), 256, 0, s>>>(keys2.get(), nnz, n_keys,
                                                            out.tile_colptr.get());
    UMAPB_LAUNCH_CHECK();
    // rows by (squared norm, index): the euclidean walk over untouched rows
    out.norm_order.alloc(std::max<int64_t>(n, 1), s);
    DevBuf<uint64_t> nk(std::max<int64_t>(n, 1), s), nk2(std::max<int64_t>(n, 1), s);
    DevBuf<int32_t> nid(std::max<int64_t>(n, 1), s);
    norm_keys_kernel<<<blocks_for(n), 256, 0, s>>>(r.sq.get(), n, nk.get(), nid.get());
    UMAPB_LAUNCH_CHECK();
    size_t tmp_bytes = 0;
    UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, nk.get(), nk2.get(), nid.get(),
                                               out.norm_order.get(), n, 0, 64, s));
    DevBuf<unsigned char> tmp(tmp_bytes, s);
    UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, nk.get(), nk2.get(),
                                               nid.get(), out.norm_order.get(), n, 0, 64, s));
}

void knn_sparse(const CsrDevice& q, const CsrDevice& r, const CsrIndex& ri, bool self, int k,
                int metric, int32_t* out_idx, float* out_dist, cudaStream_t s) {
    if (metric != UMAPB_METRIC_EUCLIDEAN && metric != UMAPB_METRIC_COSINE)
        invalid("the sparse kNN supports the euclidean and cosine metrics");
    if (k < 1 || k > kList) invalid("the sparse kNN supports 1 <= n_neighbors <= 32");
    if (k > r.n_rows) invalid("kNN needs k <= number of reference rows");
    if (q.n_cols != r.n_cols) invalid("sparse query and reference widths differ");
    if (q.n_rows == 0) return;
    SparseArgs a{};
    a.qptr = q.indptr.get();
    a.qidx = q.indices.get();
    a.qval = q.values.get();
    a.qsq = q.sq.get();
    a.ql2 = q.l2.get();
    a.nq = q.n_rows;
    a.rptr = r.indptr.get();
    a.ridx = r.indices.get();
    a.rsq = r.sq.get();
    a.rl2 = r.l2.get();
    a.nr = r.n_rows;
    a.n_cols = r.n_cols;
    a.tile_colptr = ri.tile_colptr.get();
    a.tile_rows = ri.tile_rows.get();
    a.tile_vals = ri.tile_vals.get();
    a.n_tiles = ri.n_tiles;
    a.norm_order = ri.norm_order.get();
    a.k = k;
    a.metric = metric;
    a.self = self ? 1 : 0;
    a.out_idx = out_idx;
    a.out_dist = out_dist;
    // per warp: the FP32 accumulator and the list of touched rows (uint16)
    const size_t smem = static_cast<size_t>(kWarps) * kTileRows * (sizeof(float) + sizeof(uint16_t));
    UMAPB_CUDA(cudaFuncSetAttribute(knn_sparse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    int dev = 0, sms = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t grid = std::min<int64_t>(ceil_div(q.n_rows, kWarps), static_cast<int64_t>(sms));
    knn_sparse_kernel<<<static_cast<unsigned>(grid), kWarps * 32, smem, s>>>(a);
    UMAPB_LAUNCH_CHECK();
}

}  // namespace umapb
