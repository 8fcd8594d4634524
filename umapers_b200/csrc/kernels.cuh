// kernels.cuh - internal launcher API shared by the engine and the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"

namespace umapb {

// ---------------------------------------------------------- knn_plain.cu
// Row L2 norms in the reference's summation order (l2_norm,
// rust_umap/src/lib.rs:2604-2647); `sq` (nullable) receives the squared norm
// before the square root.
void row_norms(const float* X, int64_t n, int d, float* norms, float* sq, cudaStream_t s);

// Index of the first row holding a non-finite value, or INT64_MAX.
int64_t first_nonfinite_row(const float* X, int64_t n, int d, cudaStream_t s);

// Exact kNN on FP32 CUDA cores in the reference's summation order.
// Query row r is Q[q_rows ? q_rows[r] : r] and its result goes to output row
// q_rows ? q_rows[r] : r.  Distances: euclidean = sqrt of the FP32 squared
// distance; cosine = 1 - clamp(dot / (|q||r|)).
void knn_plain(const float* Q, const int32_t* q_rows, int64_t n_q, const float* R, int64_t n_r,
               int d, int k, int metric, const float* qnorm, const float* rnorm,
               int32_t* out_idx, float* out_dist, cudaStream_t s);

// ------------------------------------------------------------- knn_tc.cu
struct TcKnnStats {
    int64_t fallback_rows = 0;
    float kernel_ms = 0.0f;   // distance-GEMM + select kernel, CUDA events
    int64_t shortlist = 0;
};

// True when the tcgen05 path supports this shape on the current device.
bool knn_tc_supported(int d, int k, int metric);

// Exact kNN through BF16 split tensor-core tiles with a certified shortlist
// and an FP32 re-rank in reference order; rows whose shortlist cannot be
// certified are recomputed by knn_plain.  Q may equal R (self join).
void knn_tc(const float* Q, int64_t n_q, const float* R, int64_t n_r, int d, int k, int metric,
            int32_t* out_idx, float* out_dist, TcKnnStats* stats, cudaStream_t s);

// ---------------------------------------------------------- nndescent.cu
int64_t nndescent(const float* X, int64_t n, int d, int k, int metric, int64_t candidate_pool,
                  int64_t n_iters, uint64_t seed, int32_t* out_idx, float* out_dist,
                  cudaStream_t s);

// -------------------------------------------------------------- graph.cu
struct Graph {
    DevBuf<int32_t> heads, tails, row_ptr;  // row_ptr: n+1 offsets into edges
    DevBuf<float> weights;
    int64_t n = 0;
    int64_t n_edges = 0;
};

// knn_rows_include_self (rust_umap/src/lib.rs:3402-3417) on the device.
bool knn_includes_self(const int32_t* idx, const float* dist, int64_t n, int k, cudaStream_t s);

// smooth_knn_dist (rust_umap/src/lib.rs:3424-3523), one thread per row.
void smooth_knn(const float* dist, int64_t n, int k, float k_f, float local_conn, float bandwidth,
                bool include_self, float* sigmas, float* rhos, cudaStream_t s);

// compute_membership_strengths + symmetrize_fuzzy_graph (+ prune_edges when
// n_epochs > 0): the symmetric graph sorted by (head, tail).
void fuzzy_union(const int32_t* idx, const float* dist, const float* sigmas, const float* rhos,
                 int64_t n, int k, float mix, int64_t n_epochs, Graph& g, cudaStream_t s);

// Bipartite membership + prune for transform (rust_umap/src/lib.rs:1738-1761):
// edges grouped by query in kNN order; returns the edge count.
void bipartite_graph(const int32_t* idx, const float* dist, const float* sigmas,
                     const float* rhos, int64_t nq, int k, int64_t n_epochs, Graph& g,
                     cudaStream_t s);

// CSR offsets of a head-sorted edge list.
void build_row_ptr(const int32_t* heads, int64_t n_edges, int64_t n, int32_t* row_ptr,
                   cudaStream_t s);

// max over weights
float max_weight(const float* w, int64_t n, cudaStream_t s);

// ----------------------------------------------------------- spectral.cu
struct SpectralResult {
    bool used_spectral = false;
    int64_t n_components = 0;
};
// initialize_embedding with InitMethod::Spectral (rust_umap/src/lib.rs:3841-3888).
SpectralResult spectral_init(const float* X, int64_t n, int d, const Graph& g, int dim,
                             uint64_t seed, float* out, cudaStream_t s);

// random_init (rust_umap/src/lib.rs:3824-3839) with counter-based uniforms.
void random_init(int64_t n, int dim, uint64_t seed, float low, float high, float* out,
                 cudaStream_t s);

// ---------------------------------------------------------------- sgd.cu
// optimize_layout_training (rust_umap/src/lib.rs:5137-5321), Hogwild over
// edges, one launch per epoch; returns the attractive edge-sample count when
// `count_samples` is set.
double optimize_layout(float* emb, int64_t n_vertices, int dim, const Graph& g, int64_t n_epochs,
                       float a, float b, float lr, int64_t neg_rate, float repulsion,
                       uint64_t seed, bool count_samples, float* kernel_ms, cudaStream_t s);

// init_graph_transform + optimize_layout_transform
// (rust_umap/src/lib.rs:4793-4836, 5444-5544): one thread per query.
void transform_layout(float* out, int64_t nq, int dim, const float* base, int64_t n_base,
                      const Graph& g, int64_t n_epochs, float a, float b, float lr,
                      int64_t neg_rate, float repulsion, uint64_t seed, cudaStream_t s);

// ------------------------------------------------------------ engine.cu
// Records the message umapb_last_error() returns on this thread.
void set_last_error(const std::string& msg);

// ------------------------------------------------------------- hostmath
void find_ab_params(float spread, float min_dist, float* a, float* b);
// Symmetric eigendecomposition (ascending eigenvalues, eigenvectors in the
// columns of V, row-major n x n).
void symmetric_eigen(const std::vector<double>& A, int n, std::vector<double>& w,
                     std::vector<double>& V);

}  // namespace umapb
