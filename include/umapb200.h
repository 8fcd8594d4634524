/*
 * umapb200.h - C ABI of the B200 UMAP engine (libumapb200.so).
 *
 * This is the drop-in boundary that replaces the PyO3 class `UmapCore` of
 * umapers (umap_rs/src/lib.rs:540-1320) and the `rust_umap::UmapModel` entry
 * points it forwards to (rust_umap/src/lib.rs:570-1966).  Every function
 * takes plain pointers and sizes; no pointer passed in is retained after the
 * call returns.  Host pointers are ordinary (pageable or pinned) host memory;
 * functions with the `_device` suffix take device pointers on the device that
 * was current when the model was created.
 *
 * All functions return an `umapb_status`.  The status codes map 1:1 onto the
 * reference's `UmapError` variants (rust_umap/src/lib.rs:197-244); the binding
 * raises RuntimeError for UMAPB_NOT_FITTED and UMAPB_ERR_CUDA and ValueError
 * for the rest, as umap_rs/src/lib.rs:147-157 does.  The message of the last
 * failure on the calling thread is returned by umapb_last_error().
 */
#ifndef UMAPB200_H
#define UMAPB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every declaration below is exported from libumapb200.so even though the
 * library is compiled with hidden default visibility. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define UMAPB_ABI_VERSION 2

typedef enum umapb_status {
    UMAPB_OK = 0,
    UMAPB_ERR_EMPTY_DATA = 1,            /* UmapError::EmptyData */
    UMAPB_ERR_NEED_TWO_SAMPLES = 2,      /* UmapError::NeedAtLeastTwoSamples */
    UMAPB_ERR_INCONSISTENT_DIMS = 3,     /* UmapError::InconsistentDimensions */
    UMAPB_ERR_FEATURE_MISMATCH = 4,      /* UmapError::FeatureMismatch */
    UMAPB_ERR_EMBEDDING_DIM_MISMATCH = 5,/* UmapError::EmbeddingDimensionMismatch */
    UMAPB_ERR_NOT_FITTED = 6,            /* UmapError::NotFitted */
    UMAPB_ERR_INVALID_PARAMETER = 7,     /* UmapError::InvalidParameter(msg) */
    UMAPB_ERR_CUDA = 8,                  /* device failure (no reference counterpart) */
    UMAPB_ERR_OUT_OF_MEMORY = 9          /* device allocation failure */
} umapb_status;

/* Metric enum order follows rust_umap::Metric (rust_umap/src/lib.rs:88-101). */
typedef enum umapb_metric {
    UMAPB_METRIC_EUCLIDEAN = 0,
    UMAPB_METRIC_MANHATTAN = 1,
    UMAPB_METRIC_COSINE = 2,
    UMAPB_METRIC_CHEBYSHEV = 3,
    UMAPB_METRIC_MINKOWSKI = 4,
    UMAPB_METRIC_CORRELATION = 5,
    UMAPB_METRIC_CANBERRA = 6,
    UMAPB_METRIC_BRAYCURTIS = 7
} umapb_metric;

typedef enum umapb_init {
    UMAPB_INIT_RANDOM = 0,
    UMAPB_INIT_SPECTRAL = 1
} umapb_init;

/* How exact kNN distance tiles are computed on the GPU.  Both produce the
 * same neighbour indices (ties broken by lower index) and the same FP32
 * distances as the reference's AVX2 summation order. */
typedef enum umapb_knn_backend {
    UMAPB_KNN_AUTO = 0,    /* tensor-core path where supported, else plain */
    UMAPB_KNN_TENSOR = 1,  /* tcgen05 BF16 split GEMM + FP32 re-rank */
    UMAPB_KNN_PLAIN = 2    /* FP32 CUDA-core tiles in reference order */
} umapb_knn_backend;

/* Mirrors rust_umap::UmapParams (rust_umap/src/lib.rs:128-152) with the
 * defaults of lib.rs:170-195; umapb_params_default() fills them in. */
typedef struct umapb_params {
    int64_t n_neighbors;          /* 15 */
    int64_t n_components;         /* 2 */
    int64_t n_epochs;             /* -1 = None (500 if n<=10000 else 200) */
    int32_t metric;               /* umapb_metric, euclidean */
    float metric_p;               /* minkowski p */
    float learning_rate;          /* 1.0 */
    float min_dist;               /* 0.1 */
    float spread;                 /* 1.0 */
    float local_connectivity;     /* 1.0 */
    float set_op_mix_ratio;       /* 1.0 */
    float repulsion_strength;     /* 1.0 */
    int64_t negative_sample_rate; /* 5 */
    uint64_t random_seed;         /* 42 */
    int32_t init;                 /* umapb_init, spectral */
    int32_t use_approximate_knn;  /* 1 */
    int64_t approx_knn_candidates;/* 50 */
    int64_t approx_knn_iters;     /* 14 */
    int64_t approx_knn_threshold; /* 4096 */
    int32_t densmap;              /* 0 */
    float dens_lambda;            /* 2.0 */
    float dens_frac;              /* 0.3 */
    float dens_var_shift;         /* 0.1 */
    int32_t output_dens;          /* 0 */
    int32_t knn_backend;          /* umapb_knn_backend (B200 knob), auto */
} umapb_params;

/* Same fields as FitTimingBreakdown (rust_umap/src/lib.rs:51-68); stage times
 * are measured with CUDA events on the model's stream, in seconds. */
typedef struct umapb_timings {
    double validation_sec;
    double knn_sec;
    double curve_params_sec;
    double knn_validate_trim_sec;
    double smooth_knn_sec;
    double density_original_sec;
    double membership_sec;
    double symmetrize_sec;
    double target_intersection_sec;
    double prune_sec;
    double init_sec;
    double optimize_sec;
    double density_embedding_sec;
    double output_copy_sec;
    double store_state_sec;
    double total_sec;
} umapb_timings;

/* Fields of ProfiledFit (rust_umap/src/lib.rs:71-79) besides the embedding,
 * plus kNN counters of the B200 path. */
typedef struct umapb_fit_info {
    int32_t used_approximate_knn;
    int32_t knn_backend_used;     /* umapb_knn_backend actually run */
    int64_t n_samples;
    int64_t n_features;
    int64_t n_epochs;
    int64_t n_edges;
    int64_t knn_fallback_rows;    /* rows re-run on the plain path */
    int64_t n_components_graph;   /* connected components of the fuzzy graph */
    double knn_kernel_sec;        /* dominant kNN kernel, CUDA events */
    double sgd_edge_samples;      /* attractive edge samples over all epochs */
    int64_t knn_second_pass_rows; /* rows the first tensor-core pass could not certify */
    double stage_wait_sec;        /* with timings: host time spent waiting for the device
                                     at the stage boundaries (device still busy) */
    double stage_host_sec;        /* with timings: the rest of the staged time (host work,
                                     launch overhead) */
    double sgd_kernel_sec;        /* with timings: the layout epochs alone, CUDA events */
} umapb_fit_info;

typedef struct umapb_model umapb_model;

/* ---- library ---------------------------------------------------------- */

/* Replaces umapers.__version__ (umap_rs/src/lib.rs:1551-1558). */
const char* umapb_version(void);
int32_t umapb_abi_version(void);
/* Message of the last failing call on this thread ("" if none). */
const char* umapb_last_error(void);
/* Number of kernels this library has launched in the process so far (no
 * reference counterpart; used to attribute device work in benchmarks). */
uint64_t umapb_kernel_launches(void);
/* Bytes the current device's default stream-ordered memory pool holds mapped
 * (reserved) and hands out (used) right now; the fit's working buffers come
 * from that pool (no reference counterpart; memory diagnostics). */
int32_t umapb_pool_bytes(int64_t* reserved, int64_t* used);
/* Defaults of UmapParams::default (rust_umap/src/lib.rs:170-195). */
void umapb_params_default(umapb_params* params);
/* should_use_approximate_knn (rust_umap/src/lib.rs:2285-2311): 1 when a fit
 * of n_rows x n_cols with these parameters takes the NN-descent path.  Host
 * only; needs no device. */
int32_t umapb_should_use_approximate_knn(const umapb_params* params, int64_t n_rows,
                                         int64_t n_cols);

/* ---- model lifecycle: UmapCore.__new__ (umap_rs/src/lib.rs:549-630) ---- */

int32_t umapb_create(const umapb_params* params, umapb_model** out_model);
void umapb_destroy(umapb_model* model);

/* ---- fit / transform --------------------------------------------------- */

/* UmapCore.fit (umap_rs/src/lib.rs:632-646) -> UmapModel::fit_dense (lib.rs:705). */
int32_t umapb_fit(umapb_model* model, const float* data, int64_t n_rows, int64_t n_cols);

/* UmapCore.fit_transform / fit_transform_into (umap_rs/src/lib.rs:687-710,
 * 809-835) -> UmapModel::fit_transform_dense (rust_umap/src/lib.rs:769-794).
 * `out` is n_rows x n_components float32, row-major. */
int32_t umapb_fit_transform(umapb_model* model, const float* data, int64_t n_rows,
                            int64_t n_cols, float* out);

/* UmapCore.fit_transform_stateless (umap_rs/src/lib.rs:779-807) ->
 * rust_umap::fit_transform_dense (rust_umap/src/lib.rs:1928-1942): same as
 * fit_transform but no state is kept. */
int32_t umapb_fit_transform_stateless(const umapb_params* params, const float* data,
                                      int64_t n_rows, int64_t n_cols, float* out);

/* ---- categorical supervision ----------------------------------------------
 * UmapCore.fit_supervised / fit_transform_supervised[_into]
 * (umap_rs/src/lib.rs:647-673, 746-779, 835-868) -> UmapModel::fit_dense_supervised /
 * fit_transform_dense_supervised (rust_umap/src/lib.rs:722-767).  `labels` holds
 * n_labels int64 class labels (-1 = unlabelled), checked against n_rows by
 * validate_supervised_target (lib.rs:2260-2283) with its messages, as are
 * target_weight in [0, 1] and target_n_neighbors (>= 1, or < 0 for none; the
 * production path does not use it).  After the fuzzy union, each edge is scaled by
 * label agreement, every head's row is renormalised by its largest weight, and the
 * graph is unioned again (apply_categorical_target_intersection, lib.rs:3694-3760).
 * A target_weight of 0 leaves the graph as the unsupervised fit's. */
int32_t umapb_fit_supervised(umapb_model* model, const float* data, int64_t n_rows,
                             int64_t n_cols, const int64_t* labels, int64_t n_labels,
                             float target_weight, int64_t target_n_neighbors);
int32_t umapb_fit_transform_supervised(umapb_model* model, const float* data, int64_t n_rows,
                                       int64_t n_cols, const int64_t* labels, int64_t n_labels,
                                       float target_weight, int64_t target_n_neighbors,
                                       float* out);

/* UmapCore.inverse_transform[_into] (umap_rs/src/lib.rs:1229-1290) ->
 * UmapModel::inverse_transform_dense (rust_umap/src/lib.rs:1789-1915).
 * `embedded_query` is n_rows x n_cols float32 (n_cols must equal
 * n_components); `out` is n_rows x n_features.  Dense-fitted models only;
 * n_components <= 16 and n_neighbors <= 32 on this path. */
int32_t umapb_inverse_transform(umapb_model* model, const float* embedded_query, int64_t n_rows,
                                int64_t n_cols, float* out);

/* ---- CSR input -----------------------------------------------------------
 * indptr holds n_rows + 1 int64 offsets starting at 0; indices (int64) and
 * data (float32) hold indptr[n_rows] entries, column indices strictly
 * increasing within a row.  The checks of SparseCsrMatrix::new
 * (rust_umap/src/sparse.rs:20-105) run first, with its messages.  The B200
 * path supports the euclidean and cosine metrics and n_neighbors <= 32. */

/* UmapCore.fit_sparse_csr (umap_rs/src/lib.rs:674-686) ->
 * UmapModel::fit_sparse_csr (rust_umap/src/lib.rs:998-1014). */
int32_t umapb_fit_csr(umapb_model* model, const int64_t* indptr, const int64_t* indices,
                      const float* data, int64_t n_rows, int64_t n_cols);

/* UmapCore.fit_transform_sparse_csr[_into] (umap_rs/src/lib.rs:869-883,
 * 900-915) -> UmapModel::fit_transform_sparse_csr (rust_umap/src/lib.rs:1016-1036).
 * `out` is n_rows x n_components float32. */
int32_t umapb_fit_transform_csr(umapb_model* model, const int64_t* indptr,
                                const int64_t* indices, const float* data, int64_t n_rows,
                                int64_t n_cols, float* out);

/* UmapCore.fit_transform_sparse_csr_stateless (umap_rs/src/lib.rs:884-899) ->
 * rust_umap::fit_transform_sparse_csr (rust_umap/src/lib.rs:1944-1966). */
int32_t umapb_fit_transform_csr_stateless(const umapb_params* params, const int64_t* indptr,
                                          const int64_t* indices, const float* data,
                                          int64_t n_rows, int64_t n_cols, float* out);

/* UmapCore.transform_sparse_csr[_into] (umap_rs/src/lib.rs:1198-1227) ->
 * UmapModel::transform_sparse_csr (rust_umap/src/lib.rs:1687-1736): sparse
 * queries of a model fitted on CSR rows. */
int32_t umapb_transform_csr(umapb_model* model, const int64_t* indptr, const int64_t* indices,
                            const float* data, int64_t n_rows, int64_t n_cols, float* out);

/* UmapCore.fit_transform_with_knn[_into] (umap_rs/src/lib.rs:916-1017) ->
 * UmapModel::fit_transform_with_knn_metric_dense_i64_flat (rust_umap/src/lib.rs:1159-1212).
 * knn_indices int64 [idx_rows x idx_cols], knn_dists float32 [dist_rows x dist_cols]. */
int32_t umapb_fit_transform_with_knn(umapb_model* model, const float* data, int64_t n_rows,
                                     int64_t n_cols, const int64_t* knn_indices,
                                     int64_t idx_rows, int64_t idx_cols,
                                     const float* knn_dists, int64_t dist_rows,
                                     int64_t dist_cols, int32_t knn_metric,
                                     int32_t validate_precomputed, float* out);

/* UmapCore.transform / transform_into (umap_rs/src/lib.rs:1147-1200) ->
 * UmapModel::transform_dense (rust_umap/src/lib.rs:1593-1685). */
int32_t umapb_transform(umapb_model* model, const float* query, int64_t n_rows,
                        int64_t n_cols, float* out);

/* UmapCore.profile_fit_transform (umap_rs/src/lib.rs:712-744) ->
 * UmapModel::profile_fit_transform_dense (rust_umap/src/lib.rs:796-962). */
int32_t umapb_profile_fit_transform(umapb_model* model, const float* data, int64_t n_rows,
                                    int64_t n_cols, float* out, umapb_timings* timings,
                                    umapb_fit_info* info);

/* The deterministic stages of transform_from_knn (rust_umap/src/lib.rs:
 * 1738-1763) for query rows of a fitted model: the exact query kNN to the
 * fitted rows, smooth_knn_dist with local_connectivity - 1 (lib.rs:3424-3523),
 * compute_membership_strengths_bipartite (lib.rs:3562-3595) after prune_edges
 * with the transform's epoch count (lib.rs:3804-3822), and
 * init_graph_transform (lib.rs:4793-4836), i.e. transform's output before
 * optimize_layout_transform.  sigmas/rhos: n_rows floats; heads/tails/
 * weights: edges grouped by query in kNN order (at most edge_capacity);
 * init: n_rows x n_components. */
int32_t umapb_transform_graph(umapb_model* model, const float* query, int64_t n_rows,
                              int64_t n_cols, float* sigmas, float* rhos, int32_t* heads,
                              int32_t* tails, float* weights, int64_t edge_capacity,
                              int64_t* n_edges, float* init);

/* Device-resident variants of fit_transform / transform: `data`, `query` and
 * `out` are device pointers (no host copies inside).  They have no reference
 * counterpart; they exist so a caller that keeps its matrices in HBM pays no
 * PCIe traffic.  `timings`/`info` may be NULL. */
int32_t umapb_fit_transform_device(umapb_model* model, const float* data, int64_t n_rows,
                                   int64_t n_cols, float* out, umapb_timings* timings,
                                   umapb_fit_info* info);
int32_t umapb_transform_device(umapb_model* model, const float* query, int64_t n_rows,
                               int64_t n_cols, float* out);

/* ---- fitted-state getters (umap_rs/src/lib.rs:1260-1320) --------------- */

int64_t umapb_n_components(const umapb_model* model);
int64_t umapb_n_neighbors(const umapb_model* model);
/* -1 when the model is not fitted. */
int64_t umapb_n_features(const umapb_model* model);
int64_t umapb_n_samples(const umapb_model* model);
/* Copies the fitted embedding (n_samples x n_components) into `out`. */
int32_t umapb_get_embedding(const umapb_model* model, float* out, int64_t n_rows,
                            int64_t n_cols);
/* UmapCore.radii_original / radii_embedding (umap_rs/src/lib.rs:1306-1320) ->
 * UmapModel::radii_original / radii_embedding: the mean log neighbour radius
 * of every fitted row in the input space (local_radii_from_knn,
 * rust_umap/src/lib.rs:5057-5082) and in the embedding
 * (embedding_radii_from_knn, 5084-5108).  They exist after a fit with densmap
 * or output_dens set; umapb_has_radii tells.  Either pointer may be NULL. */
int32_t umapb_has_radii(const umapb_model* model);
int32_t umapb_get_radii(const umapb_model* model, float* radii_original, float* radii_embedding,
                        int64_t n_rows);
/* Copies the curve parameters resolved by the last fit (UmapModel::ab_params,
 * rust_umap/src/lib.rs:604-610). */
int32_t umapb_get_ab(const umapb_model* model, float* a, float* b);

/* ---- stage entry points (host buffers) --------------------------------- *
 * Each runs one stage of the fit on the current device and exists so that a
 * caller (or a parity test) can drive the stages separately. */

/* find_ab_params (rust_umap/src/lib.rs:5672-5746), host arithmetic. */
int32_t umapb_find_ab_params(float spread, float min_dist, float* a, float* b);

/* Exact kNN of every row against all rows, self included
 * (exact_nearest_neighbors, rust_umap/src/lib.rs:2911-2928).  Euclidean
 * distances are sqrt of FP32 squared distances in the reference's
 * summation order (lib.rs:2445-2492); ties go to the lower index.
 * `fallback_rows` (may be NULL) receives the number of rows the tensor path
 * could not certify and recomputed on the plain path. */
int32_t umapb_knn_exact(const float* data, int64_t n_rows, int64_t n_cols, int64_t k,
                        int32_t metric, int32_t backend, int64_t* indices, float* dists,
                        int64_t* fallback_rows);

/* Allocation-free exact kNN (euclidean, self join, tensor-core path) for
 * callers that cannot allocate device memory: for example a host that hands
 * all HBM to its own arena before loading this library, or code that runs
 * where the CUDA allocator may not be called.  It has no counterpart in the
 * reference.  `data` (n_rows x n_cols f32), `indices` (n_rows x k int32) and
 * `dists` (n_rows x k f32) are device pointers; `stream` is a cudaStream_t
 * (NULL = legacy default stream).  Results equal umapb_knn_exact's.
 * Scratch comes from one static device array of 160 MiB that every GPU
 * loading the library holds until exit: about 49,000 rows at 64 columns; larger
 * inputs are rejected with UMAPB_ERR_INVALID_PARAMETER naming the limit.  No
 * cudaMalloc/cudaFree or allocating library routine is called.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress),
 * so make that first call before any stream capture.  The call reads the
 * kernel's status and the count of rows it recomputes on the plain path back
 * to the host, so it waits for `stream` before it returns: no call may be made
 * while `stream` is being captured into a graph.  Every call reuses
 * the same array: calls that overlap on the GPU (other streams, other
 * threads) race and must be serialised by the caller. */
int32_t umapb_knn_exact_noalloc(const float* data, int64_t n_rows, int64_t n_cols, int64_t k,
                                int32_t* indices, float* dists, void* stream);

/* Exact kNN of query rows against reference rows
 * (exact_nearest_neighbors_to_reference, rust_umap/src/lib.rs:3346-3399). */
int32_t umapb_knn_query(const float* query, int64_t n_query, const float* reference,
                        int64_t n_reference, int64_t n_cols, int64_t k, int32_t metric,
                        int32_t backend, int64_t* indices, float* dists);

/* sparse::exact_nearest_neighbors (rust_umap/src/sparse.rs:605-626): exact
 * kNN of CSR rows against themselves (a row's distance to itself is 0),
 * euclidean or cosine, k <= 32; indices int64 and distances float32, n_rows x k. */
int32_t umapb_knn_csr(const int64_t* indptr, const int64_t* indices, const float* data,
                      int64_t n_rows, int64_t n_cols, int64_t k, int32_t metric,
                      int64_t* out_indices, float* out_dists);

/* sparse::exact_nearest_neighbors_sparse_query (rust_umap/src/sparse.rs:628-657):
 * CSR query rows against CSR reference rows. */
int32_t umapb_knn_csr_query(const int64_t* q_indptr, const int64_t* q_indices,
                            const float* q_data, int64_t n_query, const int64_t* r_indptr,
                            const int64_t* r_indices, const float* r_data, int64_t n_reference,
                            int64_t n_cols, int64_t k, int32_t metric, int64_t* out_indices,
                            float* out_dists);

/* NN-descent on CSR rows: the candidate rule of
 * approximate_nearest_neighbors_with_distance (rust_umap/src/lib.rs:3086-3151)
 * with candidates scored by the exact sparse kNN's distances (sparse_dot in
 * ascending column order and the row norms, rust_umap/src/sparse.rs:90-97,
 * 220-239, 605-626), euclidean or cosine.  The reference has no approximate
 * path for sparse rows; a fit takes this one on an explicit approximate
 * request (use_approximate_knn with approx_knn_threshold 0).  Outputs as
 * umapb_nndescent. */
int32_t umapb_nndescent_csr(const int64_t* indptr, const int64_t* indices, const float* data,
                            int64_t n_rows, int64_t n_cols, int64_t k, int32_t metric,
                            int64_t candidate_pool, int64_t n_iters, uint64_t seed,
                            int64_t* indices_out, float* dists, int64_t* iters_run,
                            int64_t* candidates_evaluated, double* kernel_sec);

/* NN-descent variant (approximate_nearest_neighbors_with_distance,
 * rust_umap/src/lib.rs:3086-3151) on the GPU; `seed` plays the role of
 * random_seed ^ 0xC0FE_FEED_1234_ABCD (lib.rs:2327).  `candidates_evaluated`
 * and `kernel_sec` (each may be NULL) receive the number of candidate
 * distances computed (initial lists included) and the CUDA-event time of the
 * NN-descent kernels. */
int32_t umapb_nndescent(const float* data, int64_t n_rows, int64_t n_cols, int64_t k,
                        int32_t metric, int64_t candidate_pool, int64_t n_iters,
                        uint64_t seed, int64_t* indices, float* dists, int64_t* iters_run,
                        int64_t* candidates_evaluated, double* kernel_sec);

/* smooth_knn_dist (rust_umap/src/lib.rs:3424-3523): dists is n_rows x n_cols. */
int32_t umapb_smooth_knn_dist(const float* dists, int64_t n_rows, int64_t n_cols, float k,
                              float local_connectivity, float bandwidth,
                              int32_t include_self, float* sigmas, float* rhos);

/* Fuzzy simplicial set of a kNN graph: self detection (lib.rs:3402-3417),
 * smooth_knn_dist, compute_membership_strengths (3525-3560),
 * symmetrize_fuzzy_graph (3597-3649) and, when n_epochs > 0, prune_edges
 * (3804-3822).  Edges come back sorted by (head, tail); `capacity` must be
 * >= 2 * n_rows * k.  `sigmas`/`rhos` (length n_rows) may be NULL. */
int32_t umapb_fuzzy_graph(const int64_t* indices, const float* dists, int64_t n_rows,
                          int64_t k, float set_op_mix_ratio, float local_connectivity,
                          int64_t n_epochs, int32_t* heads, int32_t* tails, float* weights,
                          int64_t capacity, int64_t* n_edges, float* sigmas, float* rhos);

/* umapb_fuzzy_graph followed by apply_categorical_target_intersection
 * (rust_umap/src/lib.rs:1426-1431, 3694-3760) for n_rows int64 `labels` at
 * `target_weight` > 0, then prune_edges when n_epochs > 0. */
int32_t umapb_fuzzy_graph_supervised(const int64_t* indices, const float* dists, int64_t n_rows,
                                     int64_t k, float set_op_mix_ratio, float local_connectivity,
                                     int64_t n_epochs, const int64_t* labels, float target_weight,
                                     int32_t* heads, int32_t* tails, float* weights,
                                     int64_t capacity, int64_t* n_edges);

/* spectral_init (rust_umap/src/lib.rs:3871-3888, connected and
 * multi-component); `data` (n_rows x n_cols) feeds the component centroids
 * of the meta layout (lib.rs:4463-4485).  Writes n_rows x n_components.
 * Returns UMAPB_OK with *used_spectral = 0 when the reference would fall
 * back to random init (out then holds random_init's layout). */
int32_t umapb_spectral_init(const float* data, int64_t n_rows, int64_t n_cols,
                            const int32_t* heads, const int32_t* tails, const float* weights,
                            int64_t n_edges, int64_t n_components, uint64_t seed, float* out,
                            int32_t* used_spectral);

/* optimize_layout_training (rust_umap/src/lib.rs:5137-5321) on the GPU:
 * embedding (n_vertices x dim) is updated in place. */
int32_t umapb_optimize_layout(float* embedding, int64_t n_vertices, int64_t dim,
                              const int32_t* heads, const int32_t* tails, const float* weights,
                              int64_t n_edges, int64_t n_epochs, float a, float b,
                              float learning_rate, int64_t negative_sample_rate,
                              float repulsion_strength, uint64_t seed);

/* ---- learned transform surrogate ---------------------------------------- *
 * No reference function: the reference's transform is UmapModel::transform_dense
 * (rust_umap/src/lib.rs:1593-1685) and its learned model, ParametricUmapModel
 * (rust_umap/src/parametric.rs:89-534), is a separate estimator that
 * Umap.transform never uses.  Here a BF16 MLP n_cols -> hidden -> hidden ->
 * n_components (GELU, FP32 master weights, Adam) is trained on the GPU on the
 * fitted model's rows and embedding, with a loss of
 *     mse_weight * |f(x_i) - e_i|^2
 *   + edge_loss_weight * (UMAP cross-entropy of f(x_i) against the fitted
 *                    positions of the row's fuzzy-graph neighbours, with
 *                    negative samples),
 * averaged over a batch.  Inputs are standardised per feature as in
 * parametric.rs:634-707.  A held-out share of the rows calibrates a per-row
 * gate: a query whose nearest anchor row (a seeded sample of the training
 * rows) is farther than any training row assigned to it, or whose anchor cell
 * showed held-out disagreement above `fallback_radius` too often, is
 * recomputed by the plain transform (umapb_transform's path). */
typedef struct umapb_surrogate_params {
    int64_t hidden;           /* hidden width, multiple of 128 (512) */
    int64_t epochs;           /* passes over the training rows (20) */
    int64_t batch_size;       /* rows per Adam step, multiple of 128 (4096) */
    float learning_rate;      /* Adam step size (1e-3; betas 0.9/0.999, eps 1e-8) */
    float mse_weight;         /* weight of the squared error to the fitted embedding (1) */
    float edge_loss_weight;   /* weight of the fuzzy-edge cross-entropy (0.1) */
    int64_t negatives;        /* negative samples per row and step (5) */
    float holdout_fraction;   /* share of rows held out for the gate (0.05) */
    int64_t n_anchors;        /* anchor rows of the gate (256) */
    float fallback_radius;    /* disagreement radius in embedding units; <= 0 picks 5% of
                                 the embedding's 1%-99% extent */
    float max_cell_failure;   /* a cell is trusted when at most this share of its held-out
                                 rows fall outside the radius (0.1) */
    uint64_t seed;            /* 0: the model's random_seed */
} umapb_surrogate_params;

typedef struct umapb_surrogate_info {
    int64_t n_train;
    int64_t n_holdout;
    int64_t steps;
    int64_t n_anchors;
    int64_t cells_trusted;
    double radius;                 /* the fallback radius used */
    double train_sec;              /* GPU training, wall clock */
    double calibrate_sec;          /* held-out check and gate tables */
    double first_epoch_loss;
    double final_epoch_loss;
    double holdout_rmse;           /* root mean square of |f(x) - e| over the held-out rows */
    double holdout_median_error;   /* median of |f(x) - e| over the held-out rows */
    double holdout_within_radius;  /* share of held-out rows within the radius */
    double holdout_gated;          /* share of held-out rows the gate sends to the plain path */
} umapb_surrogate_info;

void umapb_surrogate_params_default(umapb_surrogate_params* params);

/* Trains the surrogate of a fitted model (after umapb_fit*).  `params` may be
 * NULL (defaults), `info` may be NULL. */
int32_t umapb_surrogate_fit(umapb_model* model, const umapb_surrogate_params* params,
                            umapb_surrogate_info* info);

/* 1 when the model holds a trained surrogate. */
int32_t umapb_surrogate_ready(const umapb_model* model);

/* Transform through the surrogate.  With `use_fallback` = 1, rows the gate
 * rejects are recomputed by the plain transform, each as a request of its own
 * (its sigma floor, prune threshold and sampling periods follow its own
 * neighbours) with the request's epoch count and the random stream of its
 * row in the request, so a gated row's result does not depend on the other
 * rows; with 0 every row keeps the network's output.  `fallback` (may be
 * NULL, n_rows bytes) receives 1 for each gated row; `n_fallback` (may be
 * NULL) their count.  Host buffers: the rows go up in chunks and the network
 * runs on each chunk as it lands; the gated rows are recomputed once, after
 * the last chunk. */
int32_t umapb_surrogate_transform(umapb_model* model, const float* query, int64_t n_rows,
                                  int64_t n_cols, int32_t use_fallback, float* out,
                                  uint8_t* fallback, int64_t* n_fallback);
/* The same on device pointers (`query`, `out`, `fallback`). */
int32_t umapb_surrogate_transform_device(umapb_model* model, const float* query,
                                         int64_t n_rows, int64_t n_cols, int32_t use_fallback,
                                         float* out, uint8_t* fallback, int64_t* n_fallback);

/* Mean training loss of each epoch of the last umapb_surrogate_fit;
 * writes min(n, epochs) values and returns that count in *n_written. */
int32_t umapb_surrogate_loss_history(const umapb_model* model, double* out, int64_t n,
                                     int64_t* n_written);

/* One forward and backward pass of the surrogate's network and loss on host
 * buffers, with the GPU kernels training uses; it exists so the gradients
 * can be checked against a CPU oracle.  `params` is the flat FP32 vector
 * W1 (hidden x n_features), b1 (hidden), W2 (hidden x hidden), b2 (hidden),
 * W3 (n_out x hidden), b3 (n_out); `grads` has the same layout.  Row p's
 * edges are edge_tail/edge_weight[edge_ptr[p] .. edge_ptr[p + 1]), indices
 * into `teacher` (n_teacher x n_out); its negatives are
 * neg_tail[p * n_neg .. (p + 1) * n_neg). */
typedef struct umapb_mlp_batch {
    int64_t batch;            /* rows, multiple of 128 */
    int64_t n_features;
    int64_t hidden;           /* multiple of 128 */
    int64_t n_out;            /* 1..4 */
    const float* x;           /* batch x n_features, already standardised */
    const float* targets;     /* batch x n_out */
    const float* params;
    const float* teacher;     /* n_teacher x n_out */
    int64_t n_teacher;
    const int64_t* edge_ptr;  /* batch + 1 */
    const int32_t* edge_tail;
    const float* edge_weight;
    const int32_t* neg_tail;  /* batch x n_neg */
    int64_t n_neg;
    float a, b;               /* curve parameters of q = 1 / (1 + a d^(2b)) */
    float mse_weight, edge_loss_weight;
    float neg_scale;          /* repulsive weight per negative = neg_scale * sum of the row's
                                 edge weights / n_neg */
    const float* out_shift;   /* n_out: y = out_shift + out_scale * (W3 a2 + b3); NULL = 0 */
    const float* out_scale;   /* n_out; NULL = 1 */
} umapb_mlp_batch;
int32_t umapb_mlp_grad(const umapb_mlp_batch* batch, float* grads, double* loss, float* y);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* UMAPB200_H */
