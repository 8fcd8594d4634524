// kernels.cuh - internal launcher API shared by the engine and the kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
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
// The same scan without a host synchronisation: the first non-finite row
// index plus `row_offset` is folded into *first_row (atomic minimum; start it
// at all ones).
void nonfinite_rows_async(const float* X, int64_t n, int d, int64_t row_offset,
                          unsigned long long* first_row, cudaStream_t s);

// Exact kNN on FP32 CUDA cores in the reference's summation order.
// Query row r is Q[q_rows ? q_rows[r] : r] and its result goes to output row
// q_rows ? q_rows[r] : r.  Distances: euclidean = sqrt of the FP32 squared
// distance; cosine = 1 - clamp(dot / (|q||r|)).  Few query rows are spread
// over the candidates with partial lists in scratch, unless !allow_scratch.
void knn_plain(const float* Q, const int32_t* q_rows, int64_t n_q, const float* R, int64_t n_r,
               int d, int k, int metric, const float* qnorm, const float* rnorm,
               int32_t* out_idx, float* out_dist, cudaStream_t s, bool allow_scratch = true);

// True when the plain kernel's tiles fit shared memory for this width and k.
bool knn_plain_supported(int d, int k);

// ------------------------------------------------------------- knn_tc.cu
struct TcKnnStats {
    int64_t fallback_rows = 0;     // rows recomputed on the plain path
    int64_t second_pass_rows = 0;  // rows the first tensor-core pass could not certify
    float kernel_ms = 0.0f;        // distance-GEMM + select kernels, CUDA events
    int64_t shortlist = 0;
};

// True when the tcgen05 path supports this shape on the current device.
bool knn_tc_supported(int d, int k, int metric);

// Exact kNN (euclidean or cosine) through FP16 tensor-core tiles with a
// certified shortlist and an FP32 re-rank in reference order; rows whose
// shortlist cannot be certified run a second pass with more lists per row,
// and rows that still fail are recomputed by knn_plain.  Q may equal R
// (self join).
void knn_tc(const float* Q, int64_t n_q, const float* R, int64_t n_r, int d, int k, int metric,
            int32_t* out_idx, float* out_dist, TcKnnStats* stats, cudaStream_t s);

// --------------------------------------------------------- knn_sparse.cu
// A CSR matrix on the device: indptr (n_rows + 1), int32 column indices
// strictly increasing within a row, FP32 values, and the per-row squared and
// L2 norms of SparseCsrMatrix (rust_umap/src/sparse.rs:90-97: sum of v * v in
// stored order, and its square root).
struct CsrDevice {
    int64_t n_rows = 0, n_cols = 0, nnz = 0;
    DevBuf<int64_t> indptr;
    DevBuf<int32_t> indices;
    DevBuf<float> values;
    DevBuf<float> sq, l2;
};

// Uploads host CSR arrays (already validated) and computes the norms.
void csr_upload(const int64_t* indptr, const int64_t* indices, const float* values,
                int64_t n_rows, int64_t n_cols, CsrDevice& out, cudaStream_t s);
// The nonzeros of dense device rows (n x d) as CSR rows, with their norms.
void csr_from_dense(const float* X, int64_t n, int64_t d, CsrDevice& out, cudaStream_t s);

// The reference side of a sparse kNN: its nonzeros regrouped by (tile of
// 2048 rows, column), rows ascending within a group, and its rows ordered by
// (squared norm, index).
struct CsrIndex {
    int64_t n_tiles = 0;
    DevBuf<int64_t> tile_colptr;  // n_tiles * n_cols + 1 offsets
    DevBuf<int32_t> tile_rows;    // row within its tile
    DevBuf<float> tile_vals;
    DevBuf<int32_t> norm_order;
};
void csr_index(const CsrDevice& r, CsrIndex& out, cudaStream_t s);

// Exact kNN of the rows of q against the rows of r (euclidean or cosine,
// k <= 32), the result of exact_nearest_neighbors (self = true, q = r) or
// exact_nearest_neighbors_sparse_query (sparse.rs:605-657) bit for bit.
void knn_sparse(const CsrDevice& q, const CsrDevice& r, const CsrIndex& ri, bool self, int k,
                int metric, int32_t* out_idx, float* out_dist, cudaStream_t s);

// ------------------------------------------------------------ gemm_tc.cu
// C[M x N] = A[M x K] B[N x K]^T on tcgen05 tensor cores: BF16 operands
// (row-major, K contiguous, K % 64 == 0, 16-byte aligned), FP32 accumulation
// in TMEM, one 128 x 128 output tile per CTA, and a fused epilogue.
enum GemmEpilogue : int {
    kEpiF32 = 0,           // c = A B^T                                 (fp32, ld N)
    kEpiBiasGelu = 1,      // z = A B^T + bias (fp32, optional); act = bf16(gelu(z)); act_t
    kEpiGeluBwd = 2,       // act = bf16((A B^T) * gelu'(z_in)); act_t
    kEpiBiasGeluHead = 3,  // kEpiBiasGelu, plus head_part[tile][row][o] = sum over the tile's
                           // columns n of act[row][n] * head_w[o][n]
    kEpiRowMin = 4,        // per row and column tile: min over columns n < n_valid of
                           // col_sq[n] - 2 (A B^T)[row][n], and its n
};
constexpr int kGemmMaxHead = 4;

struct GemmOut {
    const float* bias = nullptr;           // [N]
    const float* z_in = nullptr;           // kEpiGeluBwd: [M x N] pre-activation
    float* c = nullptr;                    // kEpiF32: [M x N]
    float* z = nullptr;                    // optional pre-activation output [M x N]
    __nv_bfloat16* act = nullptr;          // optional [M x N]
    __nv_bfloat16* act_t = nullptr;        // optional transposed output [N x ld_t]
    int64_t ld_t = 0;
    const float* head_w = nullptr;         // kEpiBiasGeluHead: [head_dim x N]
    int head_dim = 0;
    float* head_part = nullptr;            // [N / 128][M][head_dim]
    const float* col_sq = nullptr;         // kEpiRowMin: [n_valid]
    int64_t n_valid = 0;
    float* min_val = nullptr;              // kEpiRowMin: [ceil(N / 128)][M]
    int32_t* min_idx = nullptr;
};

void gemm_bf16_tn(const __nv_bfloat16* A, const __nv_bfloat16* B, int64_t M, int64_t N, int64_t K,
                  int epilogue, const GemmOut& out, cudaStream_t s);

// Reads and clears the device error word the GEMM kernels set when a
// bounded wait runs out (0 = no error since the last call).
int gemm_take_error(cudaStream_t s);

// ---------------------------------------------------------- nndescent.cu
struct NdStats {
    int64_t candidates = 0;   // candidate distances evaluated, initial lists included
    double kernel_sec = 0.0;  // CUDA-event time of the initial and iteration kernels
};
int64_t nndescent(const float* X, int64_t n, int d, int k, int metric, int64_t candidate_pool,
                  int64_t n_iters, uint64_t seed, int32_t* out_idx, float* out_dist,
                  cudaStream_t s, NdStats* stats = nullptr);
struct CsrDevice;
// The same NN-descent on CSR rows: candidates scored by sparse dot products
// in the reference's column order (the exact sparse kNN's distances).
int64_t nndescent_csr(const CsrDevice& x, int k, int metric, int64_t candidate_pool,
                      int64_t n_iters, uint64_t seed, int32_t* out_idx, float* out_dist,
                      cudaStream_t s, NdStats* stats = nullptr);

// -------------------------------------------------------------- graph.cu
struct Graph {
    DevBuf<int32_t> heads, tails, row_ptr;  // row_ptr: n+1 offsets into edges
    DevBuf<float> weights;
    DevBuf<float> row_max;  // row-local bipartite graphs: each query's largest weight
    int64_t n = 0;
    int64_t n_edges = 0;
};

// knn_rows_include_self (rust_umap/src/lib.rs:3402-3417) on the device.
bool knn_includes_self(const int32_t* idx, const float* dist, int64_t n, int k, cudaStream_t s);

// smooth_knn_dist (rust_umap/src/lib.rs:3424-3523), one thread per row.
// `row_local`: every row as a request of its own (the floor of a row with
// rho = 0 uses the mean of its own distances, not of all rows').
void smooth_knn(const float* dist, int64_t n, int k, float k_f, float local_conn, float bandwidth,
                bool include_self, float* sigmas, float* rhos, cudaStream_t s,
                bool row_local = false);

// A categorical supervision target (SupervisedTarget, rust_umap/src/lib.rs:
// 109-125) on the device: int64 labels (-1 = unlabelled), the target weight
// and the two scales of apply_categorical_target_intersection, exp(-1) and
// exp(-far_dist), computed on the host in FP32.
struct CategoricalTarget {
    const int64_t* labels = nullptr;
    float weight = 0.0f;
    float unknown_scale = 0.0f;
    float far_scale = 0.0f;
};

// compute_membership_strengths + symmetrize_fuzzy_graph (+ the categorical
// target intersection when `target` has a positive weight, + prune_edges when
// n_epochs > 0): the symmetric graph sorted by (head, tail).
// `phase_sec` (nullable, 3 values): seconds of membership, symmetrisation
// and prune + CSR offsets, with a stream synchronisation after each.
void fuzzy_union(const int32_t* idx, const float* dist, const float* sigmas, const float* rhos,
                 int64_t n, int k, float mix, int64_t n_epochs, Graph& g, cudaStream_t s,
                 double* phase_sec = nullptr, const CategoricalTarget* target = nullptr);

// Bipartite membership + prune for transform (rust_umap/src/lib.rs:1738-1761):
// edges grouped by query in kNN order; returns the edge count.  With
// `row_local` every query is pruned against its own largest weight (a
// request of one row), kept in g.row_max for the sampling periods.
void bipartite_graph(const int32_t* idx, const float* dist, const float* sigmas,
                     const float* rhos, int64_t nq, int k, int64_t n_epochs, Graph& g,
                     cudaStream_t s, bool row_local = false);

// CSR offsets of a head-sorted edge list.
void build_row_ptr(const int32_t* heads, int64_t n_edges, int64_t n, int32_t* row_ptr,
                   cudaStream_t s);

// max over weights
float max_weight(const float* w, int64_t n, cudaStream_t s);

// init_inverse_points + optimize_layout_inverse (rust_umap/src/lib.rs:
// 4838-4935, 5547-5645) for nq embedded queries zq (nq x L) whose k
// neighbours in the fitted embedding are idx/dist: writes nq x D points.
void inverse_layout(const float* zq, int64_t nq, int L, const int32_t* idx, const float* dist,
                    int k, const float* emb, const float* X, int64_t n, int D, const float* sig,
                    const float* rho, float a, float b, int64_t n_epochs, float lr,
                    int64_t neg_rate, float repulsion, uint64_t seed, float* out,
                    cudaStream_t s);

// ----------------------------------------------------------- spectral.cu
struct SpectralResult {
    bool used_spectral = false;
    int64_t n_components = 0;
};
// initialize_embedding with InitMethod::Spectral (rust_umap/src/lib.rs:3841-3888).
// The input rows serve only the centroids of a disconnected graph's meta
// layout: dense X (n x d), or the CSR rows when csr is given.
SpectralResult spectral_init(const float* X, int64_t n, int d, const Graph& g, int dim,
                             uint64_t seed, float* out, cudaStream_t s,
                             const CsrDevice* csr = nullptr);

// random_init (rust_umap/src/lib.rs:3824-3839) with counter-based uniforms.
void random_init(int64_t n, int dim, uint64_t seed, float low, float high, float* out,
                 cudaStream_t s);

// ---------------------------------------------------------------- sgd.cu
// optimize_layout_training (rust_umap/src/lib.rs:5137-5321), Hogwild over
// edges, one launch per epoch; returns the attractive edge-sample count when
// `count_samples` is set.
struct DensityParams {
    const float* radii;   // local radii of the input rows (device, n)
    int64_t start_epoch;  // density_start_epoch (lib.rs:5052-5055)
    float lambda, var_shift;
};
// With `dens`, every epoch runs the densMAP kernel (lib.rs:5355-5440).
double optimize_layout(float* emb, int64_t n_vertices, int dim, const Graph& g, int64_t n_epochs,
                       float a, float b, float lr, int64_t neg_rate, float repulsion,
                       uint64_t seed, bool count_samples, float* kernel_ms, cudaStream_t s,
                       const DensityParams* dens = nullptr);

// local_radii_from_knn / embedding_radii_from_knn (lib.rs:5057-5108) and
// density_start_epoch (lib.rs:5052-5055).
void local_radii(const int32_t* idx, const float* dist, int64_t n, int k, float var_shift,
                 float* out, cudaStream_t s);
void embedding_radii(const float* emb, int dim, const int32_t* idx, int64_t n, int k,
                     float var_shift, float* out, cudaStream_t s);
int64_t density_start_epoch(int64_t n_epochs, float frac);

// init_graph_transform + optimize_layout_transform
// (rust_umap/src/lib.rs:4793-4836, 5444-5544): one thread per query.
// Query q's random stream is keyed by (qid ? qid[q] : q) + qid_offset, its
// row in the whole request.
void transform_layout(float* out, int64_t nq, int dim, const float* base, int64_t n_base,
                      const Graph& g, int64_t n_epochs, float a, float b, float lr,
                      int64_t neg_rate, float repulsion, uint64_t seed, cudaStream_t s,
                      const int32_t* qid = nullptr, int64_t qid_offset = 0);

// --------------------------------------------------------- surrogate.cu
struct Surrogate;
struct SurrogateDeleter {
    void operator()(Surrogate* s) const;
};
using SurrogatePtr = std::unique_ptr<Surrogate, SurrogateDeleter>;

// Trains the transform surrogate on fitted rows X (n x d, device), their
// embedding `emb` (n x dim, device) and the fit's fuzzy graph `g` (CSR by
// head); calibrates its gate on the held-out rows.
SurrogatePtr surrogate_train(const float* X, int64_t n, int d, const float* emb, int dim,
                             const Graph& g, float a, float b, int64_t neg_rate,
                             const umapb_surrogate_params& p, uint64_t seed,
                             umapb_surrogate_info* info, std::vector<double>* history,
                             cudaStream_t s);

// Network outputs of nq query rows (device) into out (nq x dim) and, in
// `flags` (nullable), 1 for each row the gate rejects, with no host
// synchronisation (no gate count, no GEMM status read);
// surrogate_count_flags then reads the GEMM status and counts the gated rows
// of a whole request once.
void surrogate_infer_async(const Surrogate& sg, const float* Q, int64_t nq, int d, float* out,
                           uint8_t* flags, cudaStream_t s);
// The gate alone (flags, no network outputs) and the network alone (outputs,
// no gate), queued on `s` with no host wait; surrogate_check then waits for
// `s` and reports a GEMM wait timeout.
void surrogate_gate_async(const Surrogate& sg, const float* Q, int64_t nq, int d, uint8_t* flags,
                          cudaStream_t s);
void surrogate_forward_async(const Surrogate& sg, const float* Q, int64_t nq, int d, float* out,
                             cudaStream_t s);
void surrogate_check(cudaStream_t s);
int64_t surrogate_count_flags(const uint8_t* flags, int64_t nq, cudaStream_t s);

// dst[r] = src[ids[r]] and dst[ids[r]] = src[r] for rows of d floats.
void gather_rows(const float* src, const int32_t* ids, int64_t n, int d, float* dst,
                 cudaStream_t s);
void scatter_rows(const float* src, const int32_t* ids, int64_t n, int d, float* dst,
                  cudaStream_t s);
// Ascending indices of the non-zero flags; returns their count.
int64_t select_flagged(const uint8_t* flags, int64_t n, int32_t* ids, cudaStream_t s);

// umapb_mlp_grad on host buffers.
void mlp_grad(const umapb_mlp_batch& mb, float* grads, double* loss, float* y, cudaStream_t s);

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
