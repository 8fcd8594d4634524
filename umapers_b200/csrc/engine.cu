// engine.cu - the C ABI of libumapb200 and the host pipeline behind it.
//
// Mirrors rust_umap::UmapModel (rust_umap/src/lib.rs:570-1966): parameter
// and data validation with the reference's messages (lib.rs:1968-2283), the
// kNN switch (lib.rs:2285-2331), build_dense_fit_artifacts (lib.rs:1367-1464)
// and transform_rows / transform_from_knn (lib.rs:1604-1780).  Every stage
// after the input upload runs on the model's CUDA stream; the training matrix,
// the embedding and the graph stay in HBM.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "kernels.cuh"

namespace umapb {
std::atomic<unsigned long long> g_kernel_launches{0};
}  // namespace umapb

using namespace umapb;

namespace {

thread_local std::string g_last_error;

constexpr const char* kVersion = "1.1.4+b200.1";
constexpr float kSmoothKTolerance = 1e-5f;  // lib.rs:19

std::string fmt_float(float v) {
    // Rust's Display for f32 prints the shortest round-trip representation.
    char buf[64];
    for (int prec = 1; prec <= 9; ++prec) {
        std::snprintf(buf, sizeof(buf), "%.*g", prec, static_cast<double>(v));
        if (std::strtof(buf, nullptr) == v) break;
    }
    std::string s(buf);
    if (s.find_first_of(".eE") == std::string::npos && s.find("inf") == std::string::npos &&
        s.find("nan") == std::string::npos)
        ;  // integers print without a decimal point in Rust's Display
    return s;
}

const char* metric_debug_name(int32_t m) {
    switch (m) {
        case UMAPB_METRIC_EUCLIDEAN: return "Euclidean";
        case UMAPB_METRIC_MANHATTAN: return "Manhattan";
        case UMAPB_METRIC_COSINE: return "Cosine";
        case UMAPB_METRIC_CHEBYSHEV: return "Chebyshev";
        case UMAPB_METRIC_MINKOWSKI: return "Minkowski";
        case UMAPB_METRIC_CORRELATION: return "Correlation";
        case UMAPB_METRIC_CANBERRA: return "Canberra";
        case UMAPB_METRIC_BRAYCURTIS: return "BrayCurtis";
        default: return "Unknown";
    }
}

std::string metric_debug(int32_t m, float p) {
    if (m == UMAPB_METRIC_MINKOWSKI) return "Minkowski { p: " + fmt_float(p) + " }";
    return metric_debug_name(m);
}

template <typename F>
int32_t guarded(F&& fn) {
    try {
        fn();
        g_last_error.clear();
        return UMAPB_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return UMAPB_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return UMAPB_ERR_CUDA;
    }
}

// ------------------------------------------------------------ validation
// validate_data (lib.rs:2113-2138) on host memory; the finiteness scan is
// split across threads for large inputs.
void validate_data_host(const float* data, int64_t n, int64_t d) {
    if (n == 0) throw Error(UMAPB_ERR_EMPTY_DATA, "input data is empty");
    if (n < 2) throw Error(UMAPB_ERR_NEED_TWO_SAMPLES, "need at least two samples");
    if (d == 0) invalid("input rows must have at least one feature");
    const int64_t total = n * d;
    int n_threads = 1;
    if (total >= (int64_t(1) << 22))
        n_threads = static_cast<int>(std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency())));
    std::vector<int64_t> first(n_threads, INT64_MAX);
    auto scan = [&](int t) {
        const int64_t rows_per = ceil_div(n, n_threads);
        const int64_t r0 = t * rows_per, r1 = std::min(n, r0 + rows_per);
        for (int64_t r = r0; r < r1; ++r) {
            const uint32_t* row = reinterpret_cast<const uint32_t*>(data + r * d);
            uint32_t bad = 0;
            for (int64_t c = 0; c < d; ++c) bad |= ((row[c] & 0x7f800000u) == 0x7f800000u);
            if (bad) {
                first[t] = r;
                return;
            }
        }
    };
    if (n_threads == 1) {
        scan(0);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < n_threads; ++t) th.emplace_back(scan, t);
        for (auto& t : th) t.join();
    }
    const int64_t bad = *std::min_element(first.begin(), first.end());
    if (bad != INT64_MAX)
        invalid("input contains non-finite value at row " + std::to_string(bad));
}

void validate_data_device(const float* data, int64_t n, int64_t d, cudaStream_t s) {
    if (n == 0) throw Error(UMAPB_ERR_EMPTY_DATA, "input data is empty");
    if (n < 2) throw Error(UMAPB_ERR_NEED_TWO_SAMPLES, "need at least two samples");
    if (d == 0) invalid("input rows must have at least one feature");
    const int64_t bad = first_nonfinite_row(data, n, static_cast<int>(d), s);
    if (bad != INT64_MAX)
        invalid("input contains non-finite value at row " + std::to_string(bad));
}

bool finite(float v) { return std::isfinite(v); }

// validate_params (lib.rs:2140-2228) and validate_metric (lib.rs:2230-2239).
void validate_params(const umapb_params& p, int64_t n_samples) {
    if (p.metric == UMAPB_METRIC_MINKOWSKI && (!finite(p.metric_p) || p.metric_p <= 0.0f))
        invalid("minkowski metric requires finite p > 0");
    if (p.n_neighbors < 2) invalid("n_neighbors must be >= 2");
    if (p.n_neighbors >= n_samples)
        invalid("n_neighbors (" + std::to_string(p.n_neighbors) +
                ") must be smaller than number of samples (" + std::to_string(n_samples) + ")");
    if (p.n_components <= 0) invalid("n_components must be >= 1");
    if (!finite(p.learning_rate) || p.learning_rate <= 0.0f)
        invalid("learning_rate must be finite and > 0");
    if (!finite(p.min_dist) || p.min_dist < 0.0f) invalid("min_dist must be finite and >= 0");
    if (!finite(p.spread) || p.spread <= 0.0f) invalid("spread must be finite and > 0");
    if (p.min_dist > p.spread) invalid("min_dist must be <= spread");
    if (!finite(p.set_op_mix_ratio) || p.set_op_mix_ratio < 0.0f || p.set_op_mix_ratio > 1.0f)
        invalid("set_op_mix_ratio must be finite and in [0, 1]");
    if (!finite(p.repulsion_strength) || p.repulsion_strength < 0.0f)
        invalid("repulsion_strength must be finite and >= 0");
    if (p.negative_sample_rate <= 0) invalid("negative_sample_rate must be >= 1");
    if (!finite(p.local_connectivity) || p.local_connectivity < 0.0f)
        invalid("local_connectivity must be finite and >= 0");
    if (p.approx_knn_candidates <= 0) invalid("approx_knn_candidates must be >= 1");
    if (p.approx_knn_iters <= 0) invalid("approx_knn_iters must be >= 1");
    if (!finite(p.dens_lambda) || p.dens_lambda < 0.0f) invalid("dens_lambda must be finite and >= 0");
    if (!finite(p.dens_frac) || p.dens_frac < 0.0f || p.dens_frac > 1.0f)
        invalid("dens_frac must be finite and in [0, 1]");
    if (!finite(p.dens_var_shift) || p.dens_var_shift <= 0.0f)
        invalid("dens_var_shift must be finite and > 0");
}

// The parts of the reference surface the GPU engine does not implement.
void check_engine_support(const umapb_params& p) {
    if (p.metric != UMAPB_METRIC_EUCLIDEAN && p.metric != UMAPB_METRIC_COSINE)
        invalid(std::string("metric ") + metric_debug_name(p.metric) +
                " is not supported by the B200 engine (supported: euclidean, cosine)");
    if (p.n_components > 16) invalid("n_components above 16 is not supported by the B200 engine");
}

// SparseCsrMatrix::new (rust_umap/src/sparse.rs:20-105) on host arrays:
// indptr holds n_rows + 1 offsets, indices and data indptr[n_rows] entries.
void validate_csr_host(const int64_t* indptr, const int64_t* indices, const float* data,
                       int64_t n_rows, int64_t n_cols) {
    if (n_cols <= 0) invalid("csr n_cols must be >= 1");
    if (!indptr || (indptr[n_rows] > 0 && (!indices || !data))) invalid("null csr array");
    if (indptr[0] != 0) invalid("csr indptr must start from 0");
    for (int64_t row = 0; row < n_rows; ++row) {
        if (indptr[row] > indptr[row + 1])
            invalid("csr indptr must be non-decreasing, got indptr[" + std::to_string(row) +
                    "]=" + std::to_string(indptr[row]) + " > indptr[" + std::to_string(row + 1) +
                    "]=" + std::to_string(indptr[row + 1]));
        for (int64_t e = indptr[row] + 1; e < indptr[row + 1]; ++e)
            if (indices[e - 1] >= indices[e])
                invalid("csr row " + std::to_string(row) + " indices must be strictly increasing");
        for (int64_t e = indptr[row]; e < indptr[row + 1]; ++e)
            if (indices[e] < 0 || indices[e] >= n_cols)
                invalid("csr row " + std::to_string(row) + " has column index " +
                        std::to_string(indices[e]) + " out of bounds for n_cols=" +
                        std::to_string(n_cols));
    }
    for (int64_t e = 0; e < indptr[n_rows]; ++e)
        if (!std::isfinite(data[e])) invalid("csr data must be finite");
    if (indptr[n_rows] > 0x7FFFFFFFll) invalid("csr input above 2^31 nonzeros is not supported");
}

// validate_sparse_metric and validate_sparse_density_params
// (lib.rs:2241-2258), then the B200 sparse kNN's own limits.
void check_sparse_support(const umapb_params& p) {
    if (p.metric == UMAPB_METRIC_CANBERRA || p.metric == UMAPB_METRIC_BRAYCURTIS)
        invalid(std::string(metric_debug_name(p.metric)) +
                " metric is currently supported for dense input only");
    if (p.densmap || p.output_dens)
        invalid("densmap and output_dens are currently supported for dense input only");
    check_engine_support(p);
    if (p.n_neighbors > 32)
        invalid("n_neighbors above 32 is not supported by the B200 sparse kNN");
}

// should_use_approximate_knn (lib.rs:2285-2311).
bool should_use_approximate_knn(const umapb_params& p, int64_t n, int64_t d) {
    if (!p.use_approximate_knn || n <= p.approx_knn_threshold) return false;
    if (p.approx_knn_threshold > 0) {
        const int64_t mult = 4;  // both branches of lib.rs:2300-2307 use 4
        (void)d;
        if (n <= p.approx_knn_threshold * mult) return false;
    }
    return true;
}

// CSR fits take NN-descent only on an explicit approximate request.
bool sparse_uses_nndescent(const umapb_params& p, int64_t n) {
    return p.use_approximate_knn && p.approx_knn_threshold == 0 && n > p.n_neighbors + 1;
}

int64_t default_epochs(const umapb_params& p, int64_t n) {
    return p.n_epochs >= 0 ? p.n_epochs : (n <= 10000 ? 500 : 200);
}

double now_sec() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Stage timer: each lap synchronises the stream and returns the wall time
// since the previous lap.  It also splits that time into the part the host
// spent waiting inside the synchronisation (the device still busy) and the
// rest (host-side work and launch overhead), summed over the laps.
struct StageClock {
    cudaStream_t s;
    bool on;
    double t0;
    double wait_sec = 0.0;  // inside cudaStreamSynchronize
    double host_sec = 0.0;  // outside it
    StageClock(cudaStream_t st, bool enabled) : s(st), on(enabled), t0(now_sec()) {}
    double lap() {
        if (!on) return 0.0;
        const double tb = now_sec();
        UMAPB_CUDA(cudaStreamSynchronize(s));
        const double t = now_sec();
        const double dt = t - t0;
        wait_sec += t - tb;
        host_sec += tb - t0;
        t0 = t;
        return dt;
    }
};

}  // namespace

namespace umapb {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace umapb

struct umapb_model {
    umapb_params p{};
    int device = -1;
    cudaStream_t stream = nullptr;
    // A second stream at the device's lowest priority, for work beside the
    // model's stream: the chunked uploads of a host surrogate transform and
    // the surrogate's network beside the gated rows' plain transform.  It
    // lives as long as the model, so the device blocks freed on it stay
    // cached for the next call.
    cudaStream_t side = nullptr;
    std::mutex mu;
    float a = 0.0f, b = 0.0f;
    bool fitted = false;
    int64_t n_fit = 0, d_fit = 0;
    DevBuf<float> X;    // training rows, n_fit x d_fit (dense fits)
    umapb::CsrDevice csr;      // training rows of a sparse fit
    umapb::CsrIndex csr_idx;   // their kNN index (tiles by column, norm order)
    bool sparse = false;       // fitted from CSR rows
    DevBuf<float> emb;  // fitted embedding, n_fit x n_components
    DevBuf<float> fit_sig, fit_rho;  // the fit's smooth_knn_dist sigmas / rhos (inverse_transform)
    Graph graph;        // the fit's fuzzy graph (CSR by head), the surrogate's edge loss
    DevBuf<float> radii_orig, radii_emb;  // densMAP / output_dens radii (n_fit each)
    SurrogatePtr surrogate;
    std::vector<double> surrogate_loss;

    void ensure_device() {
        if (stream) {
            UMAPB_CUDA(cudaSetDevice(device));
            return;
        }
        UMAPB_CUDA(cudaGetDevice(&device));
        // The model's stream has the device's highest priority: where a call
        // runs work beside it on another stream (the surrogate's network
        // beside the gated rows' plain transform), the latency-bound chain on
        // this stream gets freed SMs first.
        int least = 0, greatest = 0;
        UMAPB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        UMAPB_CUDA(cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, greatest));
        UMAPB_CUDA(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, least));
        // keep freed pool memory cached across fits
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    // A new fit replaces every fitted array: release the old ones first so the
    // fit's peak memory holds one generation only.
    void begin_fit() {
        fitted = false;
        surrogate.reset();
        surrogate_loss.clear();
        graph = Graph();
        radii_orig.release();
        radii_emb.release();
        fit_sig.release();
        fit_rho.release();
        emb.release();
        X.release();
        csr = umapb::CsrDevice();
        csr_idx = umapb::CsrIndex();
        sparse = false;
    }
    void resolve_ab() {
        // resolve_ab_params (lib.rs:613-622): computed once, reused by later fits
        if (a > 0.0f && b > 0.0f) return;
        umapb::find_ab_params(p.spread, p.min_dist, &a, &b);
    }
};

namespace {

struct FitOutputs {
    umapb_timings t{};
    umapb_fit_info info{};
};

// Exact kNN on the device (exact_nearest_neighbors{,_to_reference}).
void knn_exact_device(const float* Q, int64_t nq, const float* R, int64_t nr, int d, int k,
                      int metric, int backend, int32_t* idx, float* dist, int64_t* fallback,
                      double* kernel_sec, int32_t* backend_used, cudaStream_t s,
                      int64_t* second_pass = nullptr) {
    const bool use_tc = backend == UMAPB_KNN_TENSOR ||
                        (backend == UMAPB_KNN_AUTO && knn_tc_supported(d, k, metric));
    if (backend == UMAPB_KNN_TENSOR && !knn_tc_supported(d, k, metric))
        invalid("the tensor-core kNN path does not support this metric/shape on this device");
    if (use_tc) {
        TcKnnStats st;
        knn_tc(Q, nq, R, nr, d, k, metric, idx, dist, &st, s);
        if (fallback) *fallback = st.fallback_rows;
        if (second_pass) *second_pass = st.second_pass_rows;
        if (kernel_sec) *kernel_sec = st.kernel_ms * 1e-3;
        if (backend_used) *backend_used = UMAPB_KNN_TENSOR;
        return;
    }
    DevBuf<float> qn, rn;
    if (metric == UMAPB_METRIC_COSINE) {
        qn.alloc(nq, s);
        row_norms(Q, nq, d, qn.get(), nullptr, s);
        if (R == Q) {
            rn.ptr = nullptr;
        } else {
            rn.alloc(nr, s);
            row_norms(R, nr, d, rn.get(), nullptr, s);
        }
    }
    cudaEvent_t e0, e1;
    UMAPB_CUDA(cudaEventCreate(&e0));
    UMAPB_CUDA(cudaEventCreate(&e1));
    UMAPB_CUDA(cudaEventRecord(e0, s));
    knn_plain(Q, nullptr, nq, R, nr, d, k, metric, qn.get(), rn.get() ? rn.get() : qn.get(), idx,
              dist, s);
    UMAPB_CUDA(cudaEventRecord(e1, s));
    UMAPB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    UMAPB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (fallback) *fallback = 0;
    if (second_pass) *second_pass = 0;
    if (kernel_sec) *kernel_sec = ms * 1e-3;
    if (backend_used) *backend_used = UMAPB_KNN_PLAIN;
}

// build_dense_fit_artifacts (lib.rs:1367-1464) from a device kNN graph;
// writes the embedding into model->emb.
void fit_from_knn(umapb_model* m, const float* Xd, int64_t n, int64_t d, const int32_t* idx,
                  const float* dist, int k, FitOutputs* out, StageClock& clk,
                  const CsrDevice* csr = nullptr, const CategoricalTarget* target = nullptr) {
    cudaStream_t s = m->stream;
    const umapb_params& p = m->p;
    const int64_t n_epochs = default_epochs(p, n);
    m->resolve_ab();
    if (out) out->t.curve_params_sec = clk.lap();
    const bool self = knn_includes_self(idx, dist, n, k, s);
    if (out) out->t.knn_validate_trim_sec = clk.lap();
    DevBuf<float> sig(n, s), rho(n, s);
    smooth_knn(dist, n, k, static_cast<float>(p.n_neighbors), p.local_connectivity, 1.0f, self,
               sig.get(), rho.get(), s);
    if (out) out->t.smooth_knn_sec = clk.lap();
    // densMAP / output_dens (lib.rs:1401-1422): radii of the input neighbourhoods
    const bool dens_outputs = p.densmap || p.output_dens;
    DevBuf<float> r_orig;
    if (dens_outputs) {
        r_orig.alloc(n, s);
        local_radii(idx, dist, n, k, p.dens_var_shift, r_orig.get(), s);
    }
    Graph g;
    double phases[3] = {0.0, 0.0, 0.0};
    fuzzy_union(idx, dist, sig.get(), rho.get(), n, k, p.set_op_mix_ratio, n_epochs, g, s,
                out ? phases : nullptr, target);
    if (out) {
        clk.lap();
        out->t.membership_sec = phases[0];
        out->t.symmetrize_sec = phases[1];
        out->t.prune_sec = phases[2];
        out->info.n_edges = g.n_edges;
    }
    const int dim = static_cast<int>(p.n_components);
    DevBuf<float> emb(n * dim, s);
    bool spectral_ok = false;
    if (p.init == UMAPB_INIT_SPECTRAL) {
        const SpectralResult r =
            spectral_init(Xd, n, static_cast<int>(d), g, dim, p.random_seed, emb.get(), s, csr);
        spectral_ok = r.used_spectral;
        if (out) out->info.n_components_graph = r.n_components;
    }
    if (!spectral_ok) random_init(n, dim, p.random_seed, -10.0f, 10.0f, emb.get(), s);
    if (out) out->t.init_sec = clk.lap();
    float sgd_ms = 0.0f;
    DensityParams dens{r_orig.get(), density_start_epoch(n_epochs, p.dens_frac), p.dens_lambda,
                       p.dens_var_shift};
    const bool with_density = p.densmap && p.dens_lambda > 0.0f;
    const double samples = optimize_layout(
        emb.get(), n, dim, g, n_epochs, m->a, m->b, p.learning_rate, p.negative_sample_rate,
        p.repulsion_strength, p.random_seed ^ 0x9E3779B97F4A7C15ULL, out != nullptr,
        out ? &sgd_ms : nullptr, s, with_density ? &dens : nullptr);
    if (dens_outputs) {
        // radii of the same neighbourhoods in the embedding (lib.rs:1454-1462)
        DevBuf<float> r_emb(n, s);
        embedding_radii(emb.get(), dim, idx, n, k, p.dens_var_shift, r_emb.get(), s);
        m->radii_orig = std::move(r_orig);
        m->radii_emb = std::move(r_emb);
    }
    if (out) {
        out->t.optimize_sec = clk.lap();
        out->info.sgd_edge_samples = samples;
        out->info.sgd_kernel_sec = sgd_ms * 1e-3;
        out->info.n_epochs = n_epochs;
    }
    m->emb = std::move(emb);
    m->fit_sig = std::move(sig);
    m->fit_rho = std::move(rho);
    g.heads.release();
    m->graph = std::move(g);
    m->surrogate.reset();
    m->surrogate_loss.clear();
}

// Full dense fit on device-resident rows `Xd` (owned copy is taken).
void fit_device(umapb_model* m, const float* Xd, int64_t n, int64_t d, bool copy_rows,
                FitOutputs* out, StageClock& clk, const CategoricalTarget* target = nullptr) {
    cudaStream_t s = m->stream;
    const umapb_params& p = m->p;
    const int k = static_cast<int>(p.n_neighbors);
    DevBuf<float> Xown;
    const float* X = Xd;
    if (copy_rows) {
        Xown.alloc(n * d, s);
        UMAPB_CUDA(cudaMemcpyAsync(Xown.get(), Xd, n * d * 4, cudaMemcpyDeviceToDevice, s));
        X = Xown.get();
    }
    DevBuf<int32_t> idx(n * k, s);
    DevBuf<float> dist(n * k, s);
    const bool approx = should_use_approximate_knn(p, n, d);
    if (out) out->info.used_approximate_knn = approx;
    if (approx) {
        nndescent(X, n, static_cast<int>(d), k, p.metric, p.approx_knn_candidates,
                  p.approx_knn_iters, p.random_seed ^ 0xC0FEFEED1234ABCDULL, idx.get(),
                  dist.get(), s);
        if (out) out->info.knn_backend_used = -1;
    } else {
        int64_t fb = 0, second = 0;
        double ks = 0.0;
        int32_t used = 0;
        knn_exact_device(X, n, X, n, static_cast<int>(d), k, p.metric, p.knn_backend, idx.get(),
                         dist.get(), &fb, &ks, &used, s, &second);
        if (out) {
            out->info.knn_fallback_rows = fb;
            out->info.knn_second_pass_rows = second;
            out->info.knn_kernel_sec = ks;
            out->info.knn_backend_used = used;
        }
    }
    if (out) out->t.knn_sec = clk.lap();
    fit_from_knn(m, X, n, d, idx.get(), dist.get(), k, out, clk, nullptr, target);
    if (copy_rows) m->X = std::move(Xown);
    m->n_fit = n;
    m->d_fit = d;
    m->fitted = true;
}

void upload(DevBuf<float>& dst, const float* src, int64_t count, cudaStream_t s) {
    dst.alloc(count, s);
    if (count > 0)
        UMAPB_CUDA(cudaMemcpyAsync(dst.get(), src, count * 4, cudaMemcpyHostToDevice, s));
}

void copy_embedding_out(umapb_model* m, float* out) {
    const int64_t cnt = m->n_fit * m->p.n_components;
    UMAPB_CUDA(cudaMemcpyAsync(out, m->emb.get(), cnt * 4, cudaMemcpyDeviceToHost, m->stream));
    UMAPB_CUDA(cudaStreamSynchronize(m->stream));
}

void fit_host(umapb_model* m, const float* data, int64_t n, int64_t d, FitOutputs* out,
              float* emb_out) {
    StageClock clk(nullptr, out != nullptr);
    const double t_start = now_sec();
    // validate_data, validate_params and the engine's own limits, in that
    // order; the fitted state is replaced only once all of them pass
    auto checks = [&] {
        validate_data_host(data, n, d);
        validate_params(m->p, n);
        check_engine_support(m->p);
    };
    if (n == 0 || d == 0) checks();  // nothing to upload
    try {
        m->ensure_device();
    } catch (...) {
        checks();  // without a usable device the input's own errors come first
        throw;
    }
    clk.s = m->stream;
    DevBuf<float> X;
    // the copy of pinned rows runs while the host scans them; a rejected
    // input waits for its copy, so the caller's rows are not read afterwards
    upload(X, data, n * d, m->stream);
    try {
        checks();
    } catch (...) {
        cudaStreamSynchronize(m->stream);
        throw;
    }
    m->begin_fit();
    if (out) out->t.validation_sec = clk.lap();
    fit_device(m, X.get(), n, d, false, out, clk);
    m->X = std::move(X);
    if (emb_out) copy_embedding_out(m, emb_out);
    if (out) {
        out->t.output_copy_sec = clk.lap();
        out->t.total_sec = now_sec() - t_start;
        out->info.n_samples = n;
        out->info.n_features = d;
        out->info.stage_wait_sec = clk.wait_sec;
        out->info.stage_host_sec = clk.host_sec;
    }
}

// validate_supervised_target (lib.rs:2260-2283), with its messages.
// `target_n_neighbors` < 0 means none; the production path does not use it
// (only the reference's test-only target graph does, lib.rs:3651-3692).
void validate_supervised_target(int64_t n_labels, float weight, int64_t target_n_neighbors,
                                int64_t n_samples) {
    if (n_labels != n_samples)
        invalid("target label length (" + std::to_string(n_labels) +
                ") must match number of samples (" + std::to_string(n_samples) + ")");
    if (!std::isfinite(weight) || !(weight >= 0.0f && weight <= 1.0f))
        invalid("target_weight must be finite and in [0, 1]");
    if (target_n_neighbors == 0) invalid("target_n_neighbors must be >= 1 when provided");
}

// The scales of apply_categorical_target_intersection (lib.rs:3702-3708),
// FP32 as in the reference: exp(-1) for an unlabelled end, exp(-far_dist)
// with far_dist = 2.5 / (1 - weight) (1e12 at weight 1) for different labels.
void categorical_scales(float weight, float* unknown_scale, float* far_scale) {
    const float far_dist = weight < 1.0f ? 2.5f / (1.0f - weight) : 1.0e12f;
    *unknown_scale = std::exp(-1.0f);
    *far_scale = std::exp(-far_dist);
}

// fit_dense_supervised / fit_transform_dense_supervised (lib.rs:722-767,
// 1367-1431): the dense fit with the categorical target intersection between
// the fuzzy union and prune.  A weight of 0 leaves the graph as it is.
void fit_supervised_host(umapb_model* m, const float* data, int64_t n, int64_t d,
                         const int64_t* labels, int64_t n_labels, float weight,
                         int64_t target_n_neighbors, float* emb_out) {
    validate_data_host(data, n, d);
    validate_params(m->p, n);
    validate_supervised_target(n_labels, weight, target_n_neighbors, n);
    check_engine_support(m->p);
    m->ensure_device();
    cudaStream_t s = m->stream;
    StageClock clk(s, false);
    m->begin_fit();
    DevBuf<float> X;
    upload(X, data, n * d, s);
    DevBuf<int64_t> lab;
    CategoricalTarget target;
    if (weight > 0.0f) {
        lab.alloc(n, s);
        UMAPB_CUDA(cudaMemcpyAsync(lab.get(), labels, n * 8, cudaMemcpyHostToDevice, s));
        target.labels = lab.get();
        target.weight = weight;
        categorical_scales(weight, &target.unknown_scale, &target.far_scale);
    }
    fit_device(m, X.get(), n, d, false, nullptr, clk, weight > 0.0f ? &target : nullptr);
    m->X = std::move(X);
    if (emb_out) copy_embedding_out(m, emb_out);
    UMAPB_CUDA(cudaStreamSynchronize(s));
}

// inverse_transform_dense (lib.rs:1789-1915): checks in the reference's
// order, exact kNN of the embedded queries among the fitted embedding
// (exact_nearest_neighbors_to_reference, euclidean), then init_inverse_points
// and optimize_layout_inverse on the device.  `out` is nq x n_features.
void inverse_transform_host(umapb_model* m, const float* zq, int64_t nq, int64_t L, float* out) {
    if (m->fitted && m->sparse)
        invalid("inverse_transform is not supported for sparse-trained models yet");
    if (!m->fitted || m->fit_sig.get() == nullptr)
        throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
    if (nq == 0) return;
    if (L != m->p.n_components)
        throw Error(UMAPB_ERR_EMBEDDING_DIM_MISMATCH,
                    "embedding dimension mismatch: expected " + std::to_string(m->p.n_components) +
                        ", got " + std::to_string(L));
    for (int64_t i = 0; i < nq; ++i)
        for (int64_t c = 0; c < L; ++c)
            if (!std::isfinite(zq[i * L + c]))
                invalid("input contains non-finite value at row " + std::to_string(i));
    const umapb_params& p = m->p;
    cudaStream_t s = m->stream;
    UMAPB_CUDA(cudaSetDevice(m->device));
    const int64_t n = m->n_fit;
    const int64_t D = m->d_fit;
    // inverse_neighbor_count (lib.rs:3420-3422)
    const int k = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(p.n_neighbors, n)));
    const int64_t n_epochs = p.n_epochs < 0 ? (nq <= 10000 ? 100 : 30)
                                            : std::max<int64_t>(p.n_epochs / 3, 1);
    DevBuf<float> Z;
    upload(Z, zq, nq * L, s);
    DevBuf<int32_t> idx(nq * k, s);
    DevBuf<float> dist(nq * k, s);
    knn_exact_device(Z.get(), nq, m->emb.get(), n, static_cast<int>(L), k, UMAPB_METRIC_EUCLIDEAN,
                     UMAPB_KNN_PLAIN, idx.get(), dist.get(), nullptr, nullptr, nullptr, s);
    DevBuf<float> o(nq * D, s);
    inverse_layout(Z.get(), nq, static_cast<int>(L), idx.get(), dist.get(), k, m->emb.get(),
                   m->X.get(), n, static_cast<int>(D), m->fit_sig.get(), m->fit_rho.get(), m->a,
                   m->b, n_epochs, p.learning_rate, p.negative_sample_rate, p.repulsion_strength,
                   p.random_seed ^ 0xD1B54A32D192ED03ULL, o.get(), s);
    UMAPB_CUDA(cudaMemcpyAsync(out, o.get(), nq * D * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
}

// fit_sparse_csr / fit_transform_sparse_csr (lib.rs:998-1036, 1479-1549):
// exact sparse kNN, then the dense pipeline from the kNN table with the
// centroids of a disconnected graph taken from the CSR rows.
void fit_csr_host(umapb_model* m, const int64_t* indptr, const int64_t* indices,
                  const float* data, int64_t n, int64_t d, float* emb_out) {
    validate_csr_host(indptr, indices, data, n, d);
    if (n == 0) throw Error(UMAPB_ERR_EMPTY_DATA, "input data is empty");
    if (n < 2) throw Error(UMAPB_ERR_NEED_TWO_SAMPLES, "need at least two samples");
    validate_params(m->p, n);
    check_sparse_support(m->p);
    m->ensure_device();
    cudaStream_t s = m->stream;
    m->begin_fit();
    CsrDevice csr;
    csr_upload(indptr, indices, data, n, d, csr, s);
    CsrIndex ci;
    csr_index(csr, ci, s);
    const int k = static_cast<int>(m->p.n_neighbors);
    DevBuf<int32_t> idx(n * k, s);
    DevBuf<float> dist(n * k, s);
    // The reference always runs the exact kNN on CSR rows.  An explicit
    // approximate request (ann_mode="approximate": use_approximate_knn with a
    // zero threshold) runs NN-descent on them instead, with the reference's
    // candidate rule and the exact kNN's sparse distances.
    if (sparse_uses_nndescent(m->p, n))
        nndescent_csr(csr, k, m->p.metric, m->p.approx_knn_candidates, m->p.approx_knn_iters,
                      m->p.random_seed ^ 0xC0FEFEED1234ABCDULL, idx.get(), dist.get(), s);
    else
        knn_sparse(csr, csr, ci, true, k, m->p.metric, idx.get(), dist.get(), s);
    StageClock clk(s, false);
    fit_from_knn(m, nullptr, n, d, idx.get(), dist.get(), k, nullptr, clk, &csr);
    m->csr = std::move(csr);
    m->csr_idx = std::move(ci);
    m->sparse = true;
    m->n_fit = n;
    m->d_fit = d;
    m->fitted = true;
    if (emb_out) copy_embedding_out(m, emb_out);
}

// validate_and_trim_precomputed_knn (lib.rs:1968-2040) on host arrays that
// already passed the shape checks; writes the trimmed k columns.
void trim_precomputed(const int64_t* idx, const float* dist, int64_t n, int64_t cols, int64_t k,
                      std::vector<int32_t>& idx_out, std::vector<float>& dist_out) {
    idx_out.resize(n * k);
    dist_out.resize(n * k);
    std::unordered_set<int64_t> seen;
    seen.reserve(k * 2);
    for (int64_t r = 0; r < n; ++r) {
        seen.clear();
        float prev = -INFINITY;
        for (int64_t c = 0; c < k; ++c) {
            const int64_t j = idx[r * cols + c];
            const float dv = dist[r * cols + c];
            if (j >= n)
                invalid("precomputed knn index out of range at row " + std::to_string(r) +
                        ", col " + std::to_string(c));
            if (!std::isfinite(dv) || dv < 0.0f)
                invalid("precomputed knn distance must be finite and >= 0 at row " +
                        std::to_string(r) + ", col " + std::to_string(c));
            if (!seen.insert(j).second)
                invalid("precomputed knn row " + std::to_string(r) + " contains duplicate index " +
                        std::to_string(j));
            if (c > 0 && dv + kSmoothKTolerance < prev)
                invalid("precomputed knn distances must be non-decreasing within each row; row " +
                        std::to_string(r) + " has dist[" + std::to_string(c) + "]=" +
                        fmt_float(dv) + " < dist[" + std::to_string(c - 1) + "]=" +
                        fmt_float(prev));
            prev = dv;
            idx_out[r * k + c] = static_cast<int32_t>(j);
            dist_out[r * k + c] = dv;
        }
    }
}

// Work on the model's side stream with one completion event per chunk.  Its
// destructor waits for everything queued on the stream, so buffers that work
// reads or writes outlive it, on error paths too.
struct SideWork {
    cudaStream_t s = nullptr;
    cudaEvent_t ready = nullptr;
    std::vector<cudaEvent_t> done;
    SideWork(cudaStream_t side, int64_t n) : s(side), done(static_cast<size_t>(n), nullptr) {
        UMAPB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        for (auto& e : done) UMAPB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    SideWork(const SideWork&) = delete;
    SideWork& operator=(const SideWork&) = delete;
    ~SideWork() {
        if (s) cudaStreamSynchronize(s);
        for (auto e : done)
            if (e) cudaEventDestroy(e);
        if (ready) cudaEventDestroy(ready);
    }
};

// Host buffers for the deterministic transform stages (umapb_transform_graph).
struct TransformStages {
    float* sigmas = nullptr;
    float* rhos = nullptr;
    int32_t* heads = nullptr;
    int32_t* tails = nullptr;
    float* weights = nullptr;
    int64_t capacity = 0;
    int64_t* n_edges = nullptr;
};

// transform_from_knn (lib.rs:1738-1780) on a device kNN table: bipartite
// membership, weighted init and the per-query SGD.  The default epoch count
// follows the size of the whole request, `epoch_rows` (lib.rs:1650-1657).
// With `stages`, sigma, rho and the pruned edges are copied out and out_dev
// receives init_graph_transform's positions: the same transform kernel runs
// with no SGD epoch.  With `row_local` every query is transformed as a
// request of its own (its sigma floor, prune threshold and sampling periods
// follow its own distances and weights, not the batch's).
void transform_from_knn_device(umapb_model* m, const int32_t* idx, const float* dist, int64_t nq,
                               int k, int64_t epoch_rows, float* out_dev,
                               const TransformStages* stages = nullptr,
                               const int32_t* qid = nullptr, int64_t qid_offset = 0,
                               bool row_local = false) {
    cudaStream_t s = m->stream;
    const umapb_params& p = m->p;
    const int dim = static_cast<int>(p.n_components);
    const int64_t n_epochs = p.n_epochs >= 0 ? std::max<int64_t>(p.n_epochs, 1)
                                             : (epoch_rows <= 10000 ? 100 : 30);
    DevBuf<float> sig(nq, s), rho(nq, s);
    const float lc = std::max(p.local_connectivity - 1.0f, 0.0f);
    smooth_knn(dist, nq, k, static_cast<float>(k), lc, 1.0f, false, sig.get(), rho.get(), s,
               row_local);
    Graph g;
    bipartite_graph(idx, dist, sig.get(), rho.get(), nq, k, n_epochs, g, s, row_local);
    if (stages) {
        if (g.n_edges > stages->capacity)
            invalid("edge capacity " + std::to_string(stages->capacity) + " below the " +
                    std::to_string(g.n_edges) + " transform edges");
        UMAPB_CUDA(cudaMemcpyAsync(stages->sigmas, sig.get(), nq * 4, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaMemcpyAsync(stages->rhos, rho.get(), nq * 4, cudaMemcpyDeviceToHost, s));
        if (g.n_edges > 0) {
            UMAPB_CUDA(cudaMemcpyAsync(stages->heads, g.heads.get(), g.n_edges * 4,
                                       cudaMemcpyDeviceToHost, s));
            UMAPB_CUDA(cudaMemcpyAsync(stages->tails, g.tails.get(), g.n_edges * 4,
                                       cudaMemcpyDeviceToHost, s));
            UMAPB_CUDA(cudaMemcpyAsync(stages->weights, g.weights.get(), g.n_edges * 4,
                                       cudaMemcpyDeviceToHost, s));
        }
        *stages->n_edges = g.n_edges;
        transform_layout(out_dev, nq, dim, m->emb.get(), m->n_fit, g, 0, m->a, m->b,
                         p.learning_rate / 4.0f, p.negative_sample_rate, p.repulsion_strength,
                         p.random_seed ^ 0xA24BAED40B53C117ULL, s);
        return;
    }
    transform_layout(out_dev, nq, dim, m->emb.get(), m->n_fit, g, n_epochs, m->a, m->b,
                     p.learning_rate / 4.0f, p.negative_sample_rate, p.repulsion_strength,
                     p.random_seed ^ 0xA24BAED40B53C117ULL, s, qid, qid_offset);
}

// transform_dense (lib.rs:1593-1685) on device rows.  A model fitted on CSR
// rows takes the dense queries' nonzeros as CSR rows
// (exact_nearest_neighbors_dense_query, sparse.rs:753-910, gives the same
// distances).
// `qid`/`qid_offset` give each query's row in the whole request (the key of
// its random stream) when Qd holds a subset of the request's rows;
// `row_local` transforms every row as a request of its own.
void transform_device(umapb_model* m, const float* Qd, int64_t nq, int64_t d, float* out_dev,
                      int64_t epoch_rows = -1, const TransformStages* stages = nullptr,
                      const int32_t* qid = nullptr, int64_t qid_offset = 0,
                      bool row_local = false) {
    cudaStream_t s = m->stream;
    const umapb_params& p = m->p;
    const int k = static_cast<int>(std::min<int64_t>(p.n_neighbors, m->n_fit));
    if (epoch_rows < 0) epoch_rows = nq;
    DevBuf<int32_t> idx(nq * k, s);
    DevBuf<float> dist(nq * k, s);
    if (m->sparse) {
        CsrDevice q;
        csr_from_dense(Qd, nq, d, q, s);
        knn_sparse(q, m->csr, m->csr_idx, false, k, p.metric, idx.get(), dist.get(), s);
    } else {
        knn_exact_device(Qd, nq, m->X.get(), m->n_fit, static_cast<int>(d), k, p.metric,
                         p.knn_backend, idx.get(), dist.get(), nullptr, nullptr, nullptr, s);
    }
    transform_from_knn_device(m, idx.get(), dist.get(), nq, k, epoch_rows, out_dev, stages, qid,
                              qid_offset, row_local);
}

void surrogate_fallback(umapb_model* m, const float* Qd, int64_t nq, int64_t d, float* out,
                        const uint8_t* flags, int64_t nf, int64_t epoch_rows = -1,
                        int64_t row_offset = 0, cudaEvent_t before_scatter = nullptr);

// Surrogate transform of device rows: network outputs for every row, then
// (use_fallback) the plain transform for the rows the gate rejects.  The gate
// needs only the input rows, so it runs first; with gated rows, the network
// then runs on a second stream while the plain transform of the gated rows
// runs on the model's stream, and its results are scattered over the
// network's once both are done.
void surrogate_transform_device(umapb_model* m, const float* Qd, int64_t nq, int64_t d,
                                bool use_fallback, float* out, uint8_t* flags_out,
                                int64_t* n_fallback) {
    cudaStream_t s = m->stream;
    DevBuf<uint8_t> own;
    uint8_t* flags = flags_out;
    if (!flags) {
        own.alloc(nq, s);
        flags = own.get();
    }
    const Surrogate& sg = *m->surrogate;
    surrogate_gate_async(sg, Qd, nq, static_cast<int>(d), flags, s);
    const int64_t nf = surrogate_count_flags(flags, nq, s);  // synchronises s
    if (n_fallback) *n_fallback = nf;
    if (!use_fallback || nf == 0) {
        surrogate_forward_async(sg, Qd, nq, static_cast<int>(d), out, s);
        surrogate_check(s);
        return;
    }
    SideWork net(m->side, 1);
    UMAPB_CUDA(cudaEventRecord(net.ready, s));
    UMAPB_CUDA(cudaStreamWaitEvent(net.s, net.ready, 0));
    surrogate_forward_async(sg, Qd, nq, static_cast<int>(d), out, net.s);
    UMAPB_CUDA(cudaEventRecord(net.done[0], net.s));
    surrogate_fallback(m, Qd, nq, d, out, flags, nf, -1, 0, net.done[0]);
    surrogate_check(net.s);
}

// The plain transform for the `nf` rows the gate flagged, scattered into out.
// Each gated row is transformed as a request of its own (its sigma floor,
// prune threshold and sampling periods follow its own neighbours, not the
// other rows'), with the epoch count of `epoch_rows` rows (the whole
// request, default nq) and the random stream of its row in the request (row
// i of Qd is row row_offset + i).  A gated row's result therefore does not
// depend on which other rows were gated, nor on how the request is split.
void surrogate_fallback(umapb_model* m, const float* Qd, int64_t nq, int64_t d, float* out,
                        const uint8_t* flags, int64_t nf, int64_t epoch_rows,
                        int64_t row_offset, cudaEvent_t before_scatter) {
    if (nf == 0) return;
    if (epoch_rows < 0) epoch_rows = nq;
    cudaStream_t s = m->stream;
    const int dim = static_cast<int>(m->p.n_components);
    DevBuf<int32_t> ids(nf, s);
    select_flagged(flags, nq, ids.get(), s);
    DevBuf<float> sub(nf * d, s), sub_out(nf * dim, s);
    gather_rows(Qd, ids.get(), nf, static_cast<int>(d), sub.get(), s);
    transform_device(m, sub.get(), nf, d, sub_out.get(), epoch_rows, nullptr, ids.get(),
                     row_offset, true);
    // the network's outputs for these rows (another stream) land first
    if (before_scatter) UMAPB_CUDA(cudaStreamWaitEvent(s, before_scatter, 0));
    scatter_rows(sub_out.get(), ids.get(), nf, dim, out, s);
}

void check_surrogate_query(umapb_model* m, int64_t n_cols) {
    if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
    if (!m->surrogate) throw Error(UMAPB_ERR_NOT_FITTED, "the transform surrogate is not trained");
    if (n_cols != m->d_fit)
        throw Error(UMAPB_ERR_FEATURE_MISMATCH, "feature mismatch: expected " +
                                                    std::to_string(m->d_fit) + ", got " +
                                                    std::to_string(n_cols));
}

// transform_rows checks (lib.rs:1608-1643)
void check_transform(umapb_model* m, int64_t n_cols) {
    if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
    (void)n_cols;
}

// Rows per upload chunk of a host surrogate transform (64 MB at 128 features).
constexpr int64_t kUploadChunkRows = 131072;


}  // namespace

// ====================================================================== C ABI
extern "C" {

const char* umapb_version(void) { return kVersion; }
int32_t umapb_abi_version(void) { return UMAPB_ABI_VERSION; }

int32_t umapb_should_use_approximate_knn(const umapb_params* params, int64_t n_rows,
                                         int64_t n_cols) {
    if (!params) return 0;
    return should_use_approximate_knn(*params, n_rows, n_cols) ? 1 : 0;
}
const char* umapb_last_error(void) { return g_last_error.c_str(); }
uint64_t umapb_kernel_launches(void) { return g_kernel_launches.load(); }

int32_t umapb_pool_bytes(int64_t* reserved, int64_t* used) {
    return guarded([&] {
        if (!reserved || !used) invalid("null output pointer");
        int dev = 0;
        UMAPB_CUDA(cudaGetDevice(&dev));
        cudaMemPool_t pool;
        UMAPB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        unsigned long long r = 0, u = 0;
        UMAPB_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
        UMAPB_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
        *reserved = static_cast<int64_t>(r);
        *used = static_cast<int64_t>(u);
    });
}

void umapb_params_default(umapb_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->n_neighbors = 15;
    p->n_components = 2;
    p->n_epochs = -1;
    p->metric = UMAPB_METRIC_EUCLIDEAN;
    p->metric_p = 0.0f;
    p->learning_rate = 1.0f;
    p->min_dist = 0.1f;
    p->spread = 1.0f;
    p->local_connectivity = 1.0f;
    p->set_op_mix_ratio = 1.0f;
    p->repulsion_strength = 1.0f;
    p->negative_sample_rate = 5;
    p->random_seed = 42;
    p->init = UMAPB_INIT_SPECTRAL;
    p->use_approximate_knn = 1;
    p->approx_knn_candidates = 50;
    p->approx_knn_iters = 14;
    p->approx_knn_threshold = 4096;
    p->densmap = 0;
    p->dens_lambda = 2.0f;
    p->dens_frac = 0.3f;
    p->dens_var_shift = 0.1f;
    p->output_dens = 0;
    p->knn_backend = UMAPB_KNN_AUTO;
}

int32_t umapb_create(const umapb_params* params, umapb_model** out_model) {
    return guarded([&] {
        if (!params || !out_model) invalid("null argument");
        if (params->init != UMAPB_INIT_RANDOM && params->init != UMAPB_INIT_SPECTRAL)
            invalid("unsupported init, expected random|spectral");
        if (params->metric < 0 || params->metric > UMAPB_METRIC_BRAYCURTIS)
            invalid("unsupported metric");
        auto* m = new umapb_model();
        m->p = *params;
        *out_model = m;
    });
}

void umapb_destroy(umapb_model* m) {
    if (!m) return;
    {
        std::lock_guard<std::mutex> lk(m->mu);
        if (m->stream) {
            cudaSetDevice(m->device);
            // every device array is freed on the model's stream, before it goes
            m->begin_fit();
            cudaStreamSynchronize(m->stream);
            dev_release_stream(m->stream);
            cudaStreamDestroy(m->stream);
            m->stream = nullptr;
            if (m->side) {
                cudaStreamSynchronize(m->side);
                dev_release_stream(m->side);
                cudaStreamDestroy(m->side);
                m->side = nullptr;
            }
        }
    }
    delete m;
}

int32_t umapb_fit(umapb_model* m, const float* data, int64_t n_rows, int64_t n_cols) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        fit_host(m, data, n_rows, n_cols, nullptr, nullptr);
    });
}

int32_t umapb_fit_transform(umapb_model* m, const float* data, int64_t n_rows, int64_t n_cols,
                            float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        fit_host(m, data, n_rows, n_cols, nullptr, out);
    });
}

int32_t umapb_fit_supervised(umapb_model* m, const float* data, int64_t n_rows, int64_t n_cols,
                             const int64_t* labels, int64_t n_labels, float target_weight,
                             int64_t target_n_neighbors) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        fit_supervised_host(m, data, n_rows, n_cols, labels, n_labels, target_weight,
                            target_n_neighbors, nullptr);
    });
}

int32_t umapb_fit_transform_supervised(umapb_model* m, const float* data, int64_t n_rows,
                                       int64_t n_cols, const int64_t* labels, int64_t n_labels,
                                       float target_weight, int64_t target_n_neighbors,
                                       float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        fit_supervised_host(m, data, n_rows, n_cols, labels, n_labels, target_weight,
                            target_n_neighbors, out);
    });
}

int32_t umapb_inverse_transform(umapb_model* m, const float* embedded_query, int64_t n_rows,
                                int64_t n_cols, float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        inverse_transform_host(m, embedded_query, n_rows, n_cols, out);
    });
}

int32_t umapb_fit_csr(umapb_model* m, const int64_t* indptr, const int64_t* indices,
                      const float* data, int64_t n_rows, int64_t n_cols) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        fit_csr_host(m, indptr, indices, data, n_rows, n_cols, nullptr);
    });
}

int32_t umapb_fit_transform_csr(umapb_model* m, const int64_t* indptr, const int64_t* indices,
                                const float* data, int64_t n_rows, int64_t n_cols, float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        fit_csr_host(m, indptr, indices, data, n_rows, n_cols, out);
    });
}

int32_t umapb_fit_transform_csr_stateless(const umapb_params* params, const int64_t* indptr,
                                          const int64_t* indices, const float* data,
                                          int64_t n_rows, int64_t n_cols, float* out) {
    umapb_model* m = nullptr;
    int32_t st = umapb_create(params, &m);
    if (st != UMAPB_OK) return st;
    st = umapb_fit_transform_csr(m, indptr, indices, data, n_rows, n_cols, out);
    const std::string err = g_last_error;
    umapb_destroy(m);
    g_last_error = err;
    return st;
}

int32_t umapb_transform_csr(umapb_model* m, const int64_t* indptr, const int64_t* indices,
                            const float* data, int64_t n_rows, int64_t n_cols, float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        validate_csr_host(indptr, indices, data, n_rows, n_cols);
        // transform_sparse_csr (lib.rs:1687-1736)
        if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        if (n_cols != m->d_fit)
            throw Error(UMAPB_ERR_FEATURE_MISMATCH,
                        "feature mismatch: expected " + std::to_string(m->d_fit) + ", got " +
                            std::to_string(n_cols));
        if (!m->sparse)
            invalid("sparse query transform is supported only for sparse-fitted models");
        if (n_rows == 0) return;
        m->ensure_device();
        cudaStream_t s = m->stream;
        CsrDevice q;
        csr_upload(indptr, indices, data, n_rows, n_cols, q, s);
        const int k = static_cast<int>(std::min<int64_t>(m->p.n_neighbors, m->n_fit));
        DevBuf<int32_t> idx(n_rows * k, s);
        DevBuf<float> dist(n_rows * k, s);
        knn_sparse(q, m->csr, m->csr_idx, false, k, m->p.metric, idx.get(), dist.get(), s);
        DevBuf<float> outd(n_rows * m->p.n_components, s);
        transform_from_knn_device(m, idx.get(), dist.get(), n_rows, k, n_rows, outd.get());
        UMAPB_CUDA(cudaMemcpyAsync(out, outd.get(), n_rows * m->p.n_components * 4,
                                   cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
    });
}

int32_t umapb_fit_transform_stateless(const umapb_params* params, const float* data,
                                      int64_t n_rows, int64_t n_cols, float* out) {
    umapb_model* m = nullptr;
    int32_t st = umapb_create(params, &m);
    if (st != UMAPB_OK) return st;
    st = umapb_fit_transform(m, data, n_rows, n_cols, out);
    const std::string err = g_last_error;
    umapb_destroy(m);
    g_last_error = err;
    return st;
}

int32_t umapb_profile_fit_transform(umapb_model* m, const float* data, int64_t n_rows,
                                    int64_t n_cols, float* out, umapb_timings* timings,
                                    umapb_fit_info* info) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        FitOutputs fo;
        fit_host(m, data, n_rows, n_cols, &fo, out);
        if (timings) *timings = fo.t;
        if (info) *info = fo.info;
    });
}

int32_t umapb_fit_transform_device(umapb_model* m, const float* data, int64_t n_rows,
                                   int64_t n_cols, float* out, umapb_timings* timings,
                                   umapb_fit_info* info) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        m->ensure_device();
        FitOutputs fo;
        StageClock clk(m->stream, timings != nullptr || info != nullptr);
        const double t_start = now_sec();
        validate_data_device(data, n_rows, n_cols, m->stream);
        validate_params(m->p, n_rows);
        check_engine_support(m->p);
        fo.t.validation_sec = clk.lap();
        m->begin_fit();
        // profile outputs (stage laps, sampled-edge counts) only when asked for
        fit_device(m, data, n_rows, n_cols, true, timings || info ? &fo : nullptr, clk);
        if (out)
            UMAPB_CUDA(cudaMemcpyAsync(out, m->emb.get(), n_rows * m->p.n_components * 4,
                                       cudaMemcpyDeviceToDevice, m->stream));
        UMAPB_CUDA(cudaStreamSynchronize(m->stream));
        fo.t.total_sec = now_sec() - t_start;
        fo.info.n_samples = n_rows;
        fo.info.n_features = n_cols;
        fo.info.stage_wait_sec = clk.wait_sec;
        fo.info.stage_host_sec = clk.host_sec;
        if (timings) *timings = fo.t;
        if (info) *info = fo.info;
    });
}

int32_t umapb_fit_transform_with_knn(umapb_model* m, const float* data, int64_t n_rows,
                                     int64_t n_cols, const int64_t* knn_indices,
                                     int64_t idx_rows, int64_t idx_cols,
                                     const float* knn_dists, int64_t dist_rows,
                                     int64_t dist_cols, int32_t knn_metric,
                                     int32_t validate_precomputed, float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        const umapb_params& p = m->p;
        // fit_transform_with_knn_metric_dense_i64_flat (lib.rs:1159-1212)
        if (knn_metric != p.metric)
            invalid("precomputed knn metric (" + metric_debug(knn_metric, p.metric_p) +
                    ") must match model metric (" + metric_debug(p.metric, p.metric_p) + ")");
        validate_data_host(data, n_rows, n_cols);
        validate_params(p, n_rows);
        // validate_precomputed_array_shapes (lib.rs:2042-2066)
        if (idx_rows != dist_rows || idx_cols != dist_cols)
            invalid("knn_indices and knn_dists must have identical shapes");
        if (idx_rows != n_rows) invalid("knn row count must match data row count");
        if (idx_cols < p.n_neighbors)
            invalid("knn columns must be >= n_neighbors (" + std::to_string(p.n_neighbors) + ")");
        if (validate_precomputed) {
            // validate_precomputed_distance_values_flat (lib.rs:2068-2082)
            const int64_t total = dist_rows * dist_cols;
            for (int64_t i = 0; i < total; ++i) {
                if (!std::isfinite(knn_dists[i])) invalid("knn_dists must contain only finite values");
                if (knn_dists[i] < 0.0f) invalid("knn_dists must be non-negative");
            }
        }
        // precomputed_knn_indices_from_i64_flat (lib.rs:2084-2111)
        for (int64_t i = 0; i < idx_rows * idx_cols; ++i)
            if (knn_indices[i] < 0) invalid("knn indices must be non-negative integers");
        check_engine_support(p);
        const int64_t k = p.n_neighbors;
        std::vector<int32_t> idx_h;
        std::vector<float> dist_h;
        trim_precomputed(knn_indices, knn_dists, n_rows, idx_cols, k, idx_h, dist_h);
        m->ensure_device();
        cudaStream_t s = m->stream;
        DevBuf<float> X;
        upload(X, data, n_rows * n_cols, s);
        DevBuf<int32_t> idx(n_rows * k, s);
        DevBuf<float> dist;
        upload(dist, dist_h.data(), n_rows * k, s);
        UMAPB_CUDA(cudaMemcpyAsync(idx.get(), idx_h.data(), n_rows * k * 4, cudaMemcpyHostToDevice, s));
        m->begin_fit();
        StageClock clk(s, false);
        fit_from_knn(m, X.get(), n_rows, n_cols, idx.get(), dist.get(), static_cast<int>(k),
                     nullptr, clk);
        m->X = std::move(X);
        m->n_fit = n_rows;
        m->d_fit = n_cols;
        m->fitted = true;
        if (out) copy_embedding_out(m, out);
    });
}

int32_t umapb_transform(umapb_model* m, const float* query, int64_t n_rows, int64_t n_cols,
                        float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        if (n_rows == 0) return;
        if (n_cols != m->d_fit)
            throw Error(UMAPB_ERR_FEATURE_MISMATCH,
                        "feature mismatch: expected " + std::to_string(m->d_fit) + ", got " +
                            std::to_string(n_cols));
        m->ensure_device();
        cudaStream_t s = m->stream;
        DevBuf<float> Q, outd(n_rows * m->p.n_components, s);
        upload(Q, query, n_rows * n_cols, s);
        // the finiteness scan of transform_rows (lib.rs:1630-1640) runs on the uploaded rows
        const int64_t bad = first_nonfinite_row(Q.get(), n_rows, static_cast<int>(n_cols), s);
        if (bad != INT64_MAX) invalid("input contains non-finite value at row " + std::to_string(bad));
        transform_device(m, Q.get(), n_rows, n_cols, outd.get());
        UMAPB_CUDA(cudaMemcpyAsync(out, outd.get(), n_rows * m->p.n_components * 4,
                                   cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
    });
}

int32_t umapb_transform_graph(umapb_model* m, const float* query, int64_t n_rows, int64_t n_cols,
                              float* sigmas, float* rhos, int32_t* heads, int32_t* tails,
                              float* weights, int64_t edge_capacity, int64_t* n_edges,
                              float* init) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        if (!n_edges) invalid("n_edges must not be null");
        *n_edges = 0;
        if (n_rows == 0) return;
        if (n_cols != m->d_fit)
            throw Error(UMAPB_ERR_FEATURE_MISMATCH,
                        "feature mismatch: expected " + std::to_string(m->d_fit) + ", got " +
                            std::to_string(n_cols));
        m->ensure_device();
        cudaStream_t s = m->stream;
        DevBuf<float> Q, outd(n_rows * m->p.n_components, s);
        upload(Q, query, n_rows * n_cols, s);
        const int64_t bad = first_nonfinite_row(Q.get(), n_rows, static_cast<int>(n_cols), s);
        if (bad != INT64_MAX) invalid("input contains non-finite value at row " + std::to_string(bad));
        TransformStages st;
        st.sigmas = sigmas;
        st.rhos = rhos;
        st.heads = heads;
        st.tails = tails;
        st.weights = weights;
        st.capacity = edge_capacity;
        st.n_edges = n_edges;
        transform_device(m, Q.get(), n_rows, n_cols, outd.get(), -1, &st);
        UMAPB_CUDA(cudaMemcpyAsync(init, outd.get(), n_rows * m->p.n_components * 4,
                                   cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
    });
}

int32_t umapb_transform_device(umapb_model* m, const float* query, int64_t n_rows,
                               int64_t n_cols, float* out) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        if (n_rows == 0) return;
        if (n_cols != m->d_fit)
            throw Error(UMAPB_ERR_FEATURE_MISMATCH,
                        "feature mismatch: expected " + std::to_string(m->d_fit) + ", got " +
                            std::to_string(n_cols));
        m->ensure_device();
        const int64_t bad = first_nonfinite_row(query, n_rows, static_cast<int>(n_cols), m->stream);
        if (bad != INT64_MAX) invalid("input contains non-finite value at row " + std::to_string(bad));
        transform_device(m, query, n_rows, n_cols, out);
        UMAPB_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int64_t umapb_n_components(const umapb_model* m) { return m ? m->p.n_components : -1; }
int64_t umapb_n_neighbors(const umapb_model* m) { return m ? m->p.n_neighbors : -1; }
int64_t umapb_n_features(const umapb_model* m) { return (m && m->fitted) ? m->d_fit : -1; }
int64_t umapb_n_samples(const umapb_model* m) { return (m && m->fitted) ? m->n_fit : -1; }

int32_t umapb_get_embedding(const umapb_model* cm, float* out, int64_t n_rows, int64_t n_cols) {
    auto* m = const_cast<umapb_model*>(cm);
    return guarded([&] {
        std::lock_guard<std::mutex> lk(m->mu);
        if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        if (n_rows != m->n_fit || n_cols != m->p.n_components)
            invalid("output buffer shape mismatch");
        UMAPB_CUDA(cudaSetDevice(m->device));
        copy_embedding_out(m, out);
    });
}

int32_t umapb_has_radii(const umapb_model* m) {
    return (m && m->fitted && m->radii_orig.get() && m->radii_emb.get()) ? 1 : 0;
}

int32_t umapb_get_radii(const umapb_model* cm, float* radii_original, float* radii_embedding,
                        int64_t n_rows) {
    auto* m = const_cast<umapb_model*>(cm);
    return guarded([&] {
        if (!m || !m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        if (!m->radii_orig.get())
            invalid("radii are computed only when densmap or output_dens is set");
        if (n_rows != m->n_fit) invalid("radii buffers must hold n_samples values");
        std::lock_guard<std::mutex> lk(m->mu);
        if (radii_original)
            UMAPB_CUDA(cudaMemcpyAsync(radii_original, m->radii_orig.get(), n_rows * 4,
                                       cudaMemcpyDeviceToHost, m->stream));
        if (radii_embedding)
            UMAPB_CUDA(cudaMemcpyAsync(radii_embedding, m->radii_emb.get(), n_rows * 4,
                                       cudaMemcpyDeviceToHost, m->stream));
        UMAPB_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int32_t umapb_get_ab(const umapb_model* m, float* a, float* b) {
    return guarded([&] {
        if (!(m->a > 0.0f && m->b > 0.0f)) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        *a = m->a;
        *b = m->b;
    });
}

// ----------------------------------------------------------- stage APIs

int32_t umapb_find_ab_params(float spread, float min_dist, float* a, float* b) {
    return guarded([&] { umapb::find_ab_params(spread, min_dist, a, b); });
}

namespace {
struct ScopedStream {
    cudaStream_t s = nullptr;
    ScopedStream() { UMAPB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~ScopedStream() {
        if (s) {
            cudaStreamSynchronize(s);
            dev_release_stream(s);
            cudaStreamDestroy(s);
        }
    }
};

void to_i64(const std::vector<int32_t>& v, int64_t* out) {
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
}
}  // namespace

int32_t umapb_knn_exact(const float* data, int64_t n, int64_t d, int64_t k, int32_t metric,
                        int32_t backend, int64_t* indices, float* dists, int64_t* fallback_rows) {
    return guarded([&] {
        if (n <= 0 || d <= 0) invalid("empty input");
        if (k < 1 || k > n) invalid("k must be in [1, n_rows]");
        ScopedStream ss;
        DevBuf<float> X;
        upload(X, data, n * d, ss.s);
        DevBuf<int32_t> idx(n * k, ss.s);
        DevBuf<float> dist(n * k, ss.s);
        int64_t fb = 0;
        knn_exact_device(X.get(), n, X.get(), n, static_cast<int>(d), static_cast<int>(k), metric,
                         backend, idx.get(), dist.get(), &fb, nullptr, nullptr, ss.s);
        std::vector<int32_t> ih(n * k);
        UMAPB_CUDA(cudaMemcpyAsync(ih.data(), idx.get(), n * k * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaMemcpyAsync(dists, dist.get(), n * k * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        to_i64(ih, indices);
        if (fallback_rows) *fallback_rows = fb;
    });
}

int32_t umapb_knn_query(const float* query, int64_t nq, const float* reference, int64_t nr,
                        int64_t d, int64_t k, int32_t metric, int32_t backend, int64_t* indices,
                        float* dists) {
    return guarded([&] {
        if (nr <= 0 || d <= 0) invalid("empty reference");
        if (k < 1 || k > nr) invalid("k must be in [1, n_reference]");
        if (nq == 0) return;
        ScopedStream ss;
        DevBuf<float> Q, R;
        upload(Q, query, nq * d, ss.s);
        upload(R, reference, nr * d, ss.s);
        DevBuf<int32_t> idx(nq * k, ss.s);
        DevBuf<float> dist(nq * k, ss.s);
        knn_exact_device(Q.get(), nq, R.get(), nr, static_cast<int>(d), static_cast<int>(k),
                         metric, backend, idx.get(), dist.get(), nullptr, nullptr, nullptr, ss.s);
        std::vector<int32_t> ih(nq * k);
        UMAPB_CUDA(cudaMemcpyAsync(ih.data(), idx.get(), nq * k * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaMemcpyAsync(dists, dist.get(), nq * k * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        to_i64(ih, indices);
    });
}

int32_t umapb_knn_csr(const int64_t* indptr, const int64_t* indices, const float* data,
                      int64_t n_rows, int64_t n_cols, int64_t k, int32_t metric,
                      int64_t* out_idx, float* out_dist) {
    return guarded([&] {
        validate_csr_host(indptr, indices, data, n_rows, n_cols);
        if (n_rows == 0) return;
        if (k < 1 || k > n_rows) invalid("k must be in [1, n_rows]");
        ScopedStream ss;
        CsrDevice csr;
        csr_upload(indptr, indices, data, n_rows, n_cols, csr, ss.s);
        CsrIndex ci;
        csr_index(csr, ci, ss.s);
        DevBuf<int32_t> idx(n_rows * k, ss.s);
        DevBuf<float> dist(n_rows * k, ss.s);
        knn_sparse(csr, csr, ci, true, static_cast<int>(k), metric, idx.get(), dist.get(), ss.s);
        std::vector<int32_t> ih(n_rows * k);
        UMAPB_CUDA(cudaMemcpyAsync(ih.data(), idx.get(), n_rows * k * 4, cudaMemcpyDeviceToHost,
                                   ss.s));
        UMAPB_CUDA(cudaMemcpyAsync(out_dist, dist.get(), n_rows * k * 4, cudaMemcpyDeviceToHost,
                                   ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        to_i64(ih, out_idx);
    });
}

int32_t umapb_nndescent_csr(const int64_t* indptr, const int64_t* indices, const float* data,
                            int64_t n_rows, int64_t n_cols, int64_t k, int32_t metric,
                            int64_t candidate_pool, int64_t n_iters, uint64_t seed,
                            int64_t* out_idx, float* out_dist, int64_t* iters_run,
                            int64_t* candidates_evaluated, double* kernel_sec) {
    return guarded([&] {
        validate_csr_host(indptr, indices, data, n_rows, n_cols);
        if (n_rows <= 1) invalid("need at least two rows");
        if (k < 1 || k >= n_rows) invalid("k must be in [1, n_rows)");
        ScopedStream ss;
        CsrDevice csr;
        csr_upload(indptr, indices, data, n_rows, n_cols, csr, ss.s);
        DevBuf<int32_t> idx(n_rows * k, ss.s);
        DevBuf<float> dist(n_rows * k, ss.s);
        NdStats st;
        const int64_t ran = nndescent_csr(csr, static_cast<int>(k), metric, candidate_pool,
                                          n_iters, seed, idx.get(), dist.get(), ss.s, &st);
        std::vector<int32_t> ih(n_rows * k);
        UMAPB_CUDA(cudaMemcpyAsync(ih.data(), idx.get(), n_rows * k * 4, cudaMemcpyDeviceToHost,
                                   ss.s));
        UMAPB_CUDA(cudaMemcpyAsync(out_dist, dist.get(), n_rows * k * 4, cudaMemcpyDeviceToHost,
                                   ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        to_i64(ih, out_idx);
        if (iters_run) *iters_run = ran;
        if (candidates_evaluated) *candidates_evaluated = st.candidates;
        if (kernel_sec) *kernel_sec = st.kernel_sec;
    });
}

int32_t umapb_knn_csr_query(const int64_t* q_indptr, const int64_t* q_indices,
                            const float* q_data, int64_t n_q, const int64_t* r_indptr,
                            const int64_t* r_indices, const float* r_data, int64_t n_r,
                            int64_t n_cols, int64_t k, int32_t metric, int64_t* out_idx,
                            float* out_dist) {
    return guarded([&] {
        validate_csr_host(q_indptr, q_indices, q_data, n_q, n_cols);
        validate_csr_host(r_indptr, r_indices, r_data, n_r, n_cols);
        if (n_q == 0) return;
        if (k < 1 || k > n_r) invalid("k must be in [1, n_reference]");
        ScopedStream ss;
        CsrDevice q, r;
        csr_upload(q_indptr, q_indices, q_data, n_q, n_cols, q, ss.s);
        csr_upload(r_indptr, r_indices, r_data, n_r, n_cols, r, ss.s);
        CsrIndex ri;
        csr_index(r, ri, ss.s);
        DevBuf<int32_t> idx(n_q * k, ss.s);
        DevBuf<float> dist(n_q * k, ss.s);
        knn_sparse(q, r, ri, false, static_cast<int>(k), metric, idx.get(), dist.get(), ss.s);
        std::vector<int32_t> ih(n_q * k);
        UMAPB_CUDA(cudaMemcpyAsync(ih.data(), idx.get(), n_q * k * 4, cudaMemcpyDeviceToHost,
                                   ss.s));
        UMAPB_CUDA(cudaMemcpyAsync(out_dist, dist.get(), n_q * k * 4, cudaMemcpyDeviceToHost,
                                   ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        to_i64(ih, out_idx);
    });
}


int32_t umapb_nndescent(const float* data, int64_t n, int64_t d, int64_t k, int32_t metric,
                        int64_t candidate_pool, int64_t n_iters, uint64_t seed, int64_t* indices,
                        float* dists, int64_t* iters_run, int64_t* candidates_evaluated,
                        double* kernel_sec) {
    return guarded([&] {
        if (n <= 1 || d <= 0) invalid("need at least two rows");
        if (k < 1 || k >= n) invalid("k must be in [1, n_rows)");
        ScopedStream ss;
        DevBuf<float> X;
        upload(X, data, n * d, ss.s);
        DevBuf<int32_t> idx(n * k, ss.s);
        DevBuf<float> dist(n * k, ss.s);
        NdStats st;
        const int64_t ran = umapb::nndescent(X.get(), n, static_cast<int>(d), static_cast<int>(k),
                                             metric, candidate_pool, n_iters, seed, idx.get(),
                                             dist.get(), ss.s, &st);
        if (candidates_evaluated) *candidates_evaluated = st.candidates;
        if (kernel_sec) *kernel_sec = st.kernel_sec;
        std::vector<int32_t> ih(n * k);
        UMAPB_CUDA(cudaMemcpyAsync(ih.data(), idx.get(), n * k * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaMemcpyAsync(dists, dist.get(), n * k * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        to_i64(ih, indices);
        if (iters_run) *iters_run = ran;
    });
}

int32_t umapb_smooth_knn_dist(const float* dists, int64_t n, int64_t cols, float k,
                              float local_connectivity, float bandwidth, int32_t include_self,
                              float* sigmas, float* rhos) {
    return guarded([&] {
        if (n == 0) return;
        ScopedStream ss;
        DevBuf<float> D, sg(n, ss.s), rh(n, ss.s);
        upload(D, dists, n * cols, ss.s);
        smooth_knn(D.get(), n, static_cast<int>(cols), k, local_connectivity, bandwidth,
                   include_self != 0, sg.get(), rh.get(), ss.s);
        UMAPB_CUDA(cudaMemcpyAsync(sigmas, sg.get(), n * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaMemcpyAsync(rhos, rh.get(), n * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
    });
}

int32_t umapb_fuzzy_graph(const int64_t* indices, const float* dists, int64_t n, int64_t k,
                          float set_op_mix_ratio, float local_connectivity, int64_t n_epochs,
                          int32_t* heads, int32_t* tails, float* weights, int64_t capacity,
                          int64_t* n_edges, float* sigmas, float* rhos) {
    return guarded([&] {
        if (n <= 0 || k <= 0) invalid("empty kNN graph");
        if (capacity < 2 * n * k) invalid("capacity must be >= 2 * n_rows * k");
        ScopedStream ss;
        std::vector<int32_t> ih(n * k);
        for (int64_t i = 0; i < n * k; ++i) {
            if (indices[i] < 0 || indices[i] >= n) invalid("kNN index out of range");
            ih[i] = static_cast<int32_t>(indices[i]);
        }
        DevBuf<int32_t> idx(n * k, ss.s);
        DevBuf<float> dist;
        UMAPB_CUDA(cudaMemcpyAsync(idx.get(), ih.data(), n * k * 4, cudaMemcpyHostToDevice, ss.s));
        upload(dist, dists, n * k, ss.s);
        const bool self = knn_includes_self(idx.get(), dist.get(), n, static_cast<int>(k), ss.s);
        DevBuf<float> sg(n, ss.s), rh(n, ss.s);
        smooth_knn(dist.get(), n, static_cast<int>(k), static_cast<float>(k), local_connectivity,
                   1.0f, self, sg.get(), rh.get(), ss.s);
        Graph g;
        fuzzy_union(idx.get(), dist.get(), sg.get(), rh.get(), n, static_cast<int>(k),
                    set_op_mix_ratio, n_epochs, g, ss.s);
        if (g.n_edges > 0) {
            UMAPB_CUDA(cudaMemcpyAsync(heads, g.heads.get(), g.n_edges * 4, cudaMemcpyDeviceToHost, ss.s));
            UMAPB_CUDA(cudaMemcpyAsync(tails, g.tails.get(), g.n_edges * 4, cudaMemcpyDeviceToHost, ss.s));
            UMAPB_CUDA(cudaMemcpyAsync(weights, g.weights.get(), g.n_edges * 4, cudaMemcpyDeviceToHost, ss.s));
        }
        if (sigmas) UMAPB_CUDA(cudaMemcpyAsync(sigmas, sg.get(), n * 4, cudaMemcpyDeviceToHost, ss.s));
        if (rhos) UMAPB_CUDA(cudaMemcpyAsync(rhos, rh.get(), n * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        *n_edges = g.n_edges;
    });
}

int32_t umapb_fuzzy_graph_supervised(const int64_t* indices, const float* dists, int64_t n,
                                     int64_t k, float set_op_mix_ratio, float local_connectivity,
                                     int64_t n_epochs, const int64_t* labels, float target_weight,
                                     int32_t* heads, int32_t* tails, float* weights,
                                     int64_t capacity, int64_t* n_edges) {
    return guarded([&] {
        if (n <= 0 || k <= 0) invalid("empty kNN graph");
        if (capacity < 2 * n * k) invalid("capacity must be >= 2 * n_rows * k");
        validate_supervised_target(n, target_weight, -1, n);
        ScopedStream ss;
        std::vector<int32_t> ih(n * k);
        for (int64_t i = 0; i < n * k; ++i) {
            if (indices[i] < 0 || indices[i] >= n) invalid("kNN index out of range");
            ih[i] = static_cast<int32_t>(indices[i]);
        }
        DevBuf<int32_t> idx(n * k, ss.s);
        DevBuf<float> dist;
        UMAPB_CUDA(cudaMemcpyAsync(idx.get(), ih.data(), n * k * 4, cudaMemcpyHostToDevice, ss.s));
        upload(dist, dists, n * k, ss.s);
        DevBuf<int64_t> lab(n, ss.s);
        UMAPB_CUDA(cudaMemcpyAsync(lab.get(), labels, n * 8, cudaMemcpyHostToDevice, ss.s));
        CategoricalTarget target;
        target.labels = lab.get();
        target.weight = target_weight;
        categorical_scales(target_weight, &target.unknown_scale, &target.far_scale);
        const bool self = knn_includes_self(idx.get(), dist.get(), n, static_cast<int>(k), ss.s);
        DevBuf<float> sg(n, ss.s), rh(n, ss.s);
        smooth_knn(dist.get(), n, static_cast<int>(k), static_cast<float>(k), local_connectivity,
                   1.0f, self, sg.get(), rh.get(), ss.s);
        Graph g;
        fuzzy_union(idx.get(), dist.get(), sg.get(), rh.get(), n, static_cast<int>(k),
                    set_op_mix_ratio, n_epochs, g, ss.s, nullptr, &target);
        if (g.n_edges > 0) {
            UMAPB_CUDA(cudaMemcpyAsync(heads, g.heads.get(), g.n_edges * 4, cudaMemcpyDeviceToHost, ss.s));
            UMAPB_CUDA(cudaMemcpyAsync(tails, g.tails.get(), g.n_edges * 4, cudaMemcpyDeviceToHost, ss.s));
            UMAPB_CUDA(cudaMemcpyAsync(weights, g.weights.get(), g.n_edges * 4, cudaMemcpyDeviceToHost, ss.s));
        }
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        *n_edges = g.n_edges;
    });
}

namespace {
void graph_from_host(const int32_t* heads, const int32_t* tails, const float* weights,
                     int64_t ne, int64_t n, Graph& g, cudaStream_t s) {
    for (int64_t e = 0; e < ne; ++e) {
        if (heads[e] < 0 || heads[e] >= n || tails[e] < 0 || tails[e] >= n)
            invalid("edge endpoint out of range");
        if (e > 0 && heads[e] < heads[e - 1]) invalid("edges must be sorted by head");
    }
    g.n = n;
    g.n_edges = ne;
    g.heads.alloc(std::max<int64_t>(ne, 1), s);
    g.tails.alloc(std::max<int64_t>(ne, 1), s);
    g.weights.alloc(std::max<int64_t>(ne, 1), s);
    if (ne > 0) {
        UMAPB_CUDA(cudaMemcpyAsync(g.heads.get(), heads, ne * 4, cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(g.tails.get(), tails, ne * 4, cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(g.weights.get(), weights, ne * 4, cudaMemcpyHostToDevice, s));
    }
    g.row_ptr.alloc(n + 1, s);
    build_row_ptr(g.heads.get(), ne, n, g.row_ptr.get(), s);
}
}  // namespace

int32_t umapb_spectral_init(const float* data, int64_t n, int64_t d, const int32_t* heads,
                            const int32_t* tails, const float* weights, int64_t n_edges,
                            int64_t n_components, uint64_t seed, float* out,
                            int32_t* used_spectral) {
    return guarded([&] {
        if (n <= 0 || d <= 0 || n_components <= 0) invalid("empty input");
        ScopedStream ss;
        DevBuf<float> X, emb(n * n_components, ss.s);
        upload(X, data, n * d, ss.s);
        Graph g;
        graph_from_host(heads, tails, weights, n_edges, n, g, ss.s);
        const SpectralResult r = spectral_init(X.get(), n, static_cast<int>(d), g,
                                               static_cast<int>(n_components), seed, emb.get(), ss.s);
        if (!r.used_spectral)
            random_init(n, static_cast<int>(n_components), seed, -10.0f, 10.0f, emb.get(), ss.s);
        UMAPB_CUDA(cudaMemcpyAsync(out, emb.get(), n * n_components * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
        if (used_spectral) *used_spectral = r.used_spectral ? 1 : 0;
    });
}

int32_t umapb_optimize_layout(float* embedding, int64_t n, int64_t dim, const int32_t* heads,
                              const int32_t* tails, const float* weights, int64_t n_edges,
                              int64_t n_epochs, float a, float b, float learning_rate,
                              int64_t negative_sample_rate, float repulsion_strength,
                              uint64_t seed) {
    return guarded([&] {
        if (n <= 0 || dim <= 0) invalid("empty embedding");
        if (negative_sample_rate <= 0) invalid("negative_sample_rate must be >= 1");
        ScopedStream ss;
        DevBuf<float> emb;
        upload(emb, embedding, n * dim, ss.s);
        Graph g;
        graph_from_host(heads, tails, weights, n_edges, n, g, ss.s);
        optimize_layout(emb.get(), n, static_cast<int>(dim), g, n_epochs, a, b, learning_rate,
                        negative_sample_rate, repulsion_strength, seed, false, nullptr, ss.s);
        UMAPB_CUDA(cudaMemcpyAsync(embedding, emb.get(), n * dim * 4, cudaMemcpyDeviceToHost, ss.s));
        UMAPB_CUDA(cudaStreamSynchronize(ss.s));
    });
}

// ------------------------------------------------------------ surrogate
void umapb_surrogate_params_default(umapb_surrogate_params* p) {
    if (!p) return;
    p->hidden = 512;
    p->epochs = 20;
    p->batch_size = 4096;
    p->learning_rate = 1e-3f;
    p->mse_weight = 1.0f;
    p->edge_loss_weight = 0.1f;
    p->negatives = 5;
    p->holdout_fraction = 0.05f;
    p->n_anchors = 256;
    p->fallback_radius = 0.0f;
    p->max_cell_failure = 0.1f;
    p->seed = 0;
}

int32_t umapb_surrogate_fit(umapb_model* m, const umapb_surrogate_params* params,
                            umapb_surrogate_info* info) {
    return guarded([&] {
        if (!m) invalid("null model");
        std::lock_guard<std::mutex> lk(m->mu);
        if (!m->fitted) throw Error(UMAPB_ERR_NOT_FITTED, "model is not fitted yet");
        if (m->sparse) invalid("the transform surrogate needs a model fitted on dense rows");
        if (!m->X.get() || !m->graph.row_ptr.get())
            invalid("the surrogate needs a model fitted on rows (not a stateless fit)");
        umapb_surrogate_params p;
        umapb_surrogate_params_default(&p);
        if (params) p = *params;
        m->ensure_device();
        const uint64_t seed = p.seed != 0 ? p.seed : (m->p.random_seed ^ 0x51A7E5EEDull);
        umapb_surrogate_info local{};
        m->surrogate.reset();
        m->surrogate = surrogate_train(m->X.get(), m->n_fit, static_cast<int>(m->d_fit),
                                       m->emb.get(), static_cast<int>(m->p.n_components),
                                       m->graph, m->a, m->b, m->p.negative_sample_rate, p, seed,
                                       &local, &m->surrogate_loss, m->stream);
        if (info) *info = local;
    });
}

int32_t umapb_surrogate_ready(const umapb_model* m) { return (m && m->surrogate) ? 1 : 0; }

int32_t umapb_surrogate_transform(umapb_model* m, const float* query, int64_t n_rows,
                                  int64_t n_cols, int32_t use_fallback, float* out,
                                  uint8_t* fallback, int64_t* n_fallback) {
    return guarded([&] {
        if (!m) invalid("null model");
        std::lock_guard<std::mutex> lk(m->mu);
        check_surrogate_query(m, n_cols);
        if (n_fallback) *n_fallback = 0;
        if (n_rows == 0) return;
        m->ensure_device();
        cudaStream_t s = m->stream;
        const int64_t dim = m->p.n_components;
        DevBuf<float> Q(n_rows * n_cols, s), outd(n_rows * dim, s);
        DevBuf<uint8_t> fl(n_rows, s);
        // The rows go up in chunks on a second stream, and the model's stream
        // checks and infers each chunk as soon as it has landed, so the copy
        // of the next chunk overlaps the network on this one.  The guard
        // waits for every copy before Q can be freed, errors included.
        const int64_t chunk = n_rows >= 4 * kUploadChunkRows ? kUploadChunkRows : n_rows;
        const int64_t n_chunks = ceil_div(n_rows, chunk);
        SideWork cs(m->side, n_chunks);
        UMAPB_CUDA(cudaEventRecord(cs.ready, s));  // Q is allocated on s
        UMAPB_CUDA(cudaStreamWaitEvent(cs.s, cs.ready, 0));
        for (int64_t c = 0; c < n_chunks; ++c) {
            const int64_t r0 = c * chunk, rows = std::min(chunk, n_rows - r0);
            UMAPB_CUDA(cudaMemcpyAsync(Q.get() + r0 * n_cols, query + r0 * n_cols,
                                       rows * n_cols * 4, cudaMemcpyHostToDevice, cs.s));
            UMAPB_CUDA(cudaEventRecord(cs.done[c], cs.s));
        }
        // The checks and the network are queued chunk by chunk with no host
        // wait; the first non-finite row and the gate count are read back
        // once, after the last chunk.  (Copies from pageable host memory are
        // staged by the driver and keep the host busy until they land; pinned
        // rows let the queueing run ahead.)  Every gated row is transformed
        // as a request of its own, so one fallback over the gated rows of
        // all chunks gives each the result a per-chunk fallback would, and
        // pays the fallback's fixed latency once.
        DevBuf<unsigned long long> bad_row(1, s);
        UMAPB_CUDA(cudaMemsetAsync(bad_row.get(), 0xFF, 8, s));
        for (int64_t c = 0; c < n_chunks; ++c) {
            const int64_t r0 = c * chunk, rows = std::min(chunk, n_rows - r0);
            UMAPB_CUDA(cudaStreamWaitEvent(s, cs.done[c], 0));
            nonfinite_rows_async(Q.get() + r0 * n_cols, rows, static_cast<int>(n_cols), r0,
                                 bad_row.get(), s);
            surrogate_infer_async(*m->surrogate, Q.get() + r0 * n_cols, rows,
                                  static_cast<int>(n_cols), outd.get() + r0 * dim, fl.get() + r0,
                                  s);
        }
        unsigned long long bad = 0;
        UMAPB_CUDA(cudaMemcpyAsync(&bad, bad_row.get(), 8, cudaMemcpyDeviceToHost, s));
        const int64_t nf = surrogate_count_flags(fl.get(), n_rows, s);  // synchronises s
        if (bad != ~0ull) invalid("input contains non-finite value at row " + std::to_string(bad));
        if (use_fallback != 0)
            surrogate_fallback(m, Q.get(), n_rows, n_cols, outd.get(), fl.get(), nf);
        if (n_fallback) *n_fallback = nf;
        UMAPB_CUDA(cudaMemcpyAsync(out, outd.get(), n_rows * dim * 4, cudaMemcpyDeviceToHost, s));
        if (fallback)
            UMAPB_CUDA(cudaMemcpyAsync(fallback, fl.get(), n_rows, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
    });
}

int32_t umapb_surrogate_transform_device(umapb_model* m, const float* query, int64_t n_rows,
                                         int64_t n_cols, int32_t use_fallback, float* out,
                                         uint8_t* fallback, int64_t* n_fallback) {
    return guarded([&] {
        if (!m) invalid("null model");
        std::lock_guard<std::mutex> lk(m->mu);
        check_surrogate_query(m, n_cols);
        if (n_fallback) *n_fallback = 0;
        if (n_rows == 0) return;
        m->ensure_device();
        const int64_t bad =
            first_nonfinite_row(query, n_rows, static_cast<int>(n_cols), m->stream);
        if (bad != INT64_MAX)
            invalid("input contains non-finite value at row " + std::to_string(bad));
        surrogate_transform_device(m, query, n_rows, n_cols, use_fallback != 0, out, fallback,
                                   n_fallback);
        UMAPB_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int32_t umapb_surrogate_loss_history(const umapb_model* m, double* out, int64_t n,
                                     int64_t* n_written) {
    return guarded([&] {
        if (!m) invalid("null model");
        if (!m->surrogate) throw Error(UMAPB_ERR_NOT_FITTED, "the transform surrogate is not trained");
        const int64_t cnt = std::min<int64_t>(n, static_cast<int64_t>(m->surrogate_loss.size()));
        for (int64_t i = 0; i < cnt; ++i) out[i] = m->surrogate_loss[i];
        if (n_written) *n_written = cnt;
    });
}

int32_t umapb_mlp_grad(const umapb_mlp_batch* batch, float* grads, double* loss, float* y) {
    return guarded([&] {
        if (!batch || !grads) invalid("null argument");
        ScopedStream ss;
        mlp_grad(*batch, grads, loss, y, ss.s);
    });
}

}  // extern "C"
