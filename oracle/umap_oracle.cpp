// umap_oracle.cpp - CPU restatement of the umapers (rust_umap v1.1.4) UMAP
// path, used ONLY as test infrastructure: the parity tests, smoke() and the
// CPU-baseline leg of bench.py load it as the checker.  Nothing in the
// product (umapers_b200/, libumapb200.so) links, imports or calls it.
//
// Every function cites the reference file:line it restates.  Paths are
// relative to the reference project root.  Arithmetic follows the reference
// operation by operation in FP32 (no FMA contraction: build with
// -ffp-contract=off) so that deterministic stages match bit for bit:
//   * exact kNN: squared distance in the AVX2 8-lane order for dim >= 64
//     (rust_umap/src/lib.rs:2468-2492) and the scalar order below that
//     (lib.rs:2457-2466); ties by lower index (lib.rs:2768-2772);
//   * find_ab_params (lib.rs:5672-5746) through glibc powf/expf, as the Rust
//     build calls the same libm symbols;
//   * smooth_knn_dist, membership, symmetrize, prune (lib.rs:3424-3822).
// Stages that consume random numbers use the documented algorithms of the
// reference's pinned dependencies (rand 0.8.5 SmallRng = Xoshiro256++ seeded
// by SplitMix64; UniformInt/UniformFloat single-sample rules), except the
// Normal noise of rand_distr 0.4.3 (ziggurat), which is replaced by
// Box-Muller.  No reference test fixes those streams against vectors, so
// RNG-consuming stages are parity-unpinned at the bit level and are compared
// statistically.  SymmetricEigen (nalgebra 0.33.3) is replaced by a
// Householder tridiagonalisation + implicit QL solver; eigenvector signs may
// differ, which the spectral tests of the reference do not constrain.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <unordered_map>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/umapb200.h"

namespace {

constexpr float SMOOTH_K_TOLERANCE = 1e-5f;          // lib.rs:19
constexpr float MIN_K_DIST_SCALE = 1e-3f;            // lib.rs:20
constexpr float DEFAULT_BANDWIDTH = 1.0f;            // lib.rs:21
constexpr float INIT_MAX_COORD = 10.0f;              // lib.rs:22
constexpr float INIT_NOISE = 1e-4f;                  // lib.rs:23
constexpr size_t SPECTRAL_ITERATIVE_CONNECTED_THRESHOLD = 0;  // lib.rs:27
constexpr size_t SPECTRAL_EXACT_LOW_DIM_MAX_FEATURES = 8;     // lib.rs:28
constexpr size_t SPECTRAL_EXACT_LOW_DIM_MAX_SAMPLES = 2048;   // lib.rs:29
constexpr size_t SPECTRAL_ITERATIVE_COMPONENT_THRESHOLD = 128;  // lib.rs:30
constexpr size_t SPECTRAL_ITERATIVE_MAX_ITERS = 256;          // lib.rs:31
constexpr size_t SPECTRAL_ITERATIVE_OVERSAMPLING = 6;         // lib.rs:32
constexpr size_t SPECTRAL_DENSE_FALLBACK_MAX_SAMPLES = 4096;  // lib.rs:33
constexpr double SPECTRAL_ORTHO_EPS = 1e-12;                  // lib.rs:34

// ---------------------------------------------------------------- RNG ----
// rand 0.8.5 SmallRng on 64-bit targets is Xoshiro256++; seed_from_u64 fills
// the 256-bit state with four SplitMix64 outputs.
struct SmallRng {
    uint64_t s[4];
    static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    explicit SmallRng(uint64_t state) {
        for (int i = 0; i < 4; ++i) {
            state += 0x9e3779b97f4a7c15ULL;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            s[i] = z ^ (z >> 31);
        }
    }
    uint64_t next_u64() {
        const uint64_t result = rotl(s[0] + s[3], 23) + s[0];
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return result;
    }
    uint32_t next_u32() { return static_cast<uint32_t>(next_u64() >> 32); }
    // UniformInt<usize>::sample_single(low, high): widening multiply with the
    // "leading zeros" rejection zone.
    uint64_t gen_range(uint64_t low, uint64_t high) {
        const uint64_t range = high - low;  // (high-1) - low + 1
        if (range == 0) return next_u64();
        const uint64_t zone = (range << __builtin_clzll(range)) - 1;
        for (;;) {
            const uint64_t v = next_u64();
            const unsigned __int128 m = static_cast<unsigned __int128>(v) * range;
            const uint64_t hi = static_cast<uint64_t>(m >> 64);
            const uint64_t lo = static_cast<uint64_t>(m);
            if (lo <= zone) return low + hi;
        }
    }
    // UniformFloat<f32>::sample_single(low, high).
    float gen_range_f32(float low, float high) {
        float scale = high - low;
        for (;;) {
            uint32_t bits = (next_u32() >> 9) | 0x3f800000u;
            float v12;
            std::memcpy(&v12, &bits, 4);
            const float v01 = v12 - 1.0f;
            const float res = v01 * scale + low;
            if (res < high) return res;
            uint32_t sb;
            std::memcpy(&sb, &scale, 4);
            sb -= 1;
            std::memcpy(&scale, &sb, 4);
        }
    }
    // UniformFloat<f64>::sample_single(low, high).
    double gen_range_f64(double low, double high) {
        double scale = high - low;
        for (;;) {
            uint64_t bits = (next_u64() >> 12) | 0x3ff0000000000000ULL;
            double v12;
            std::memcpy(&v12, &bits, 8);
            const double v01 = v12 - 1.0;
            const double res = v01 * scale + low;
            if (res < high) return res;
            uint64_t sb;
            std::memcpy(&sb, &scale, 8);
            sb -= 1;
            std::memcpy(&scale, &sb, 8);
        }
    }
    // Normal(0, std) sample.  rand_distr's ziggurat is not restated; this is
    // the Box-Muller transform on two uniforms (parity unpinned).
    double normal(double std_dev) {
        double u1 = gen_range_f64(0.0, 1.0);
        double u2 = gen_range_f64(0.0, 1.0);
        if (u1 < 1e-300) u1 = 1e-300;
        return std_dev * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// ---------------------------------------------------------- distances ----
// squared_distance (lib.rs:2445-2454): AVX2 path for len >= 64 on x86_64.
inline float squared_distance_scalar(const float* x, const float* y, size_t n) {
    // lib.rs:2457-2466
    float acc = 0.0f;
    for (size_t i = 0; i < n; ++i) {
        const float d = x[i] - y[i];
        acc += d * d;
    }
    return acc;
}

inline float squared_distance_avx2_order(const float* x, const float* y, size_t n) {
    // lib.rs:2468-2492: 8 lanes of (acc + diff*diff), lanes summed in order,
    // then the scalar tail.
    float lane[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t idx = 0;
    for (; idx + 8 <= n; idx += 8) {
        for (int l = 0; l < 8; ++l) {
            const float d = x[idx + l] - y[idx + l];
            lane[l] = lane[l] + d * d;
        }
    }
    float sum = lane[0];
    for (int l = 1; l < 8; ++l) sum += lane[l];
    for (; idx < n; ++idx) {
        const float d = x[idx] - y[idx];
        sum += d * d;
    }
    return sum;
}

inline float squared_distance(const float* x, const float* y, size_t n) {
    return n >= 64 ? squared_distance_avx2_order(x, y, n) : squared_distance_scalar(x, y, n);
}

// l2_norm (lib.rs:2604-2647).
inline float l2_norm(const float* x, size_t n) {
    if (n >= 64) {
        float lane[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        size_t idx = 0;
        for (; idx + 8 <= n; idx += 8)
            for (int l = 0; l < 8; ++l) lane[l] = lane[l] + x[idx + l] * x[idx + l];
        float sum = lane[0];
        for (int l = 1; l < 8; ++l) sum += lane[l];
        for (; idx < n; ++idx) sum += x[idx] * x[idx];
        return std::sqrt(sum);
    }
    float acc = 0.0f;
    for (size_t i = 0; i < n; ++i) acc += x[i] * x[i];
    return std::sqrt(acc);
}

// dot_product_avx2 (lib.rs:2717-2738) / dot_product_scalar (lib.rs:2655-2664).
inline float dot_product(const float* x, const float* y, size_t n) {
    if (n >= 64) {
        float lane[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        size_t idx = 0;
        for (; idx + 8 <= n; idx += 8)
            for (int l = 0; l < 8; ++l) lane[l] = lane[l] + x[idx + l] * y[idx + l];
        float dot = lane[0];
        for (int l = 1; l < 8; ++l) dot += lane[l];
        for (; idx < n; ++idx) dot += x[idx] * y[idx];
        return dot;
    }
    float dot = 0.0f;
    for (size_t i = 0; i < n; ++i) dot += x[i] * y[i];
    return dot;
}

// cosine_distance_with_norms (lib.rs:2740-2765).
inline float cosine_distance_with_norms(const float* x, const float* y, size_t n, float xn,
                                        float yn) {
    const float dot = dot_product(x, y, n);
    if (xn == 0.0f && yn == 0.0f) return 0.0f;
    if (xn == 0.0f || yn == 0.0f) return 1.0f;
    float c = dot / (xn * yn);
    c = std::min(std::max(c, -1.0f), 1.0f);
    return 1.0f - c;
}

// f32::total_cmp order key for the non-NaN values used here.
inline int32_t total_key(float v) {
    int32_t b;
    std::memcpy(&b, &v, 4);
    return b ^ static_cast<int32_t>(static_cast<uint32_t>(b >> 31) >> 1);
}

// neighbor_cmp (lib.rs:2768-2772): (dist.total_cmp, index).
inline bool neighbor_less(size_t li, float ld, size_t ri, float rd) {
    const int32_t a = total_key(ld), b = total_key(rd);
    if (a != b) return a < b;
    return li < ri;
}

// push_top_k_neighbor (lib.rs:2775-2808).
inline void push_top_k(std::vector<size_t>& ri, std::vector<float>& rd, size_t idx, float dist,
                       size_t k) {
    if (ri.size() == k && !neighbor_less(idx, dist, ri[k - 1], rd[k - 1])) return;
    size_t at = ri.size();
    while (at > 0 && neighbor_less(idx, dist, ri[at - 1], rd[at - 1])) --at;
    ri.insert(ri.begin() + at, idx);
    rd.insert(rd.begin() + at, dist);
    if (ri.size() > k) {
        ri.pop_back();
        rd.pop_back();
    }
}

struct Knn {
    std::vector<std::vector<size_t>> idx;
    std::vector<std::vector<float>> dist;
};

// exact_top_k_neighbors{,_euclidean,_to_reference_euclidean} (lib.rs:2810-2861)
// and the cosine variants (lib.rs:2874-2889, 3321-3344).
void exact_row(const float* q, const float* ref, size_t n_ref, size_t d, size_t k, int metric,
               float qnorm, const float* ref_norms, std::vector<size_t>& ri,
               std::vector<float>& rd) {
    ri.clear();
    rd.clear();
    ri.reserve(k + 1);
    rd.reserve(k + 1);
    for (size_t j = 0; j < n_ref; ++j) {
        float dist;
        if (metric == UMAPB_METRIC_COSINE)
            dist = cosine_distance_with_norms(q, ref + j * d, d, qnorm, ref_norms[j]);
        else
            dist = squared_distance(q, ref + j * d, d);
        push_top_k(ri, rd, j, dist, k);
    }
    if (metric != UMAPB_METRIC_COSINE)
        for (auto& v : rd) v = std::sqrt(v);  // sqrt_row_dists (lib.rs:2830-2834)
}

Knn exact_knn_query(const float* q, size_t nq, const float* ref, size_t nr, size_t d, size_t k,
                    int metric) {
    Knn out;
    out.idx.resize(nq);
    out.dist.resize(nq);
    std::vector<float> qn, rn;
    if (metric == UMAPB_METRIC_COSINE) {
        qn.resize(nq);
        rn.resize(nr);
        for (size_t i = 0; i < nq; ++i) qn[i] = l2_norm(q + i * d, d);
        for (size_t i = 0; i < nr; ++i) rn[i] = l2_norm(ref + i * d, d);
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < static_cast<int64_t>(nq); ++i) {
        exact_row(q + i * d, ref, nr, d, k, metric, qn.empty() ? 0.0f : qn[i],
                  rn.empty() ? nullptr : rn.data(), out.idx[i], out.dist[i]);
    }
    return out;
}

// ------------------------------------------------------------ NN-descent --
// mix_approx_seed (lib.rs:3017-3024).
uint64_t mix_approx_seed(uint64_t seed, uint64_t row, uint64_t iteration) {
    uint64_t v = seed ^ (row * 0x9E3779B97F4A7C15ULL) ^ (iteration * 0xBF58476D1CE4E5B9ULL);
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}

inline bool push_unique(std::vector<size_t>& out, size_t idx) {  // lib.rs:3026-3033
    if (std::find(out.begin(), out.end(), idx) != out.end()) return false;
    out.push_back(idx);
    return true;
}

// sorted_unique_neighbors (lib.rs:2932-2938).
void sorted_unique(std::vector<std::pair<size_t, float>>& pairs, size_t k) {
    std::sort(pairs.begin(), pairs.end(), [](const auto& a, const auto& b) {
        return neighbor_less(a.first, a.second, b.first, b.second);
    });
    if (pairs.size() > k) pairs.resize(k);
}

// approximate_nearest_neighbors_with_distance (lib.rs:3086-3151).
Knn nndescent(const float* x, size_t n, size_t d, size_t k, int metric, size_t candidate_pool,
              size_t n_iters, uint64_t seed, size_t* iters_run) {
    std::vector<float> norms;
    if (metric == UMAPB_METRIC_COSINE) {
        norms.resize(n);
        for (size_t i = 0; i < n; ++i) norms[i] = l2_norm(x + i * d, d);
    }
    auto dist_fn = [&](size_t i, size_t j) -> float {
        if (metric == UMAPB_METRIC_COSINE)
            return cosine_distance_with_norms(x + i * d, x + j * d, d, norms[i], norms[j]);
        return std::sqrt(squared_distance(x + i * d, x + j * d, d));  // lib.rs:3167
    };
    const size_t pool = std::min(std::max(candidate_pool, k), n - 1);
    const size_t max_candidates = std::max(candidate_pool, k) * 4 + 1;
    std::vector<size_t> nb_idx(n * k);
    std::vector<float> nb_dist(n * k);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
        const size_t i = static_cast<size_t>(ii);
        SmallRng rng(mix_approx_seed(seed, i, 0));
        std::vector<size_t> cand;
        cand.reserve(pool + 1);
        cand.push_back(i);  // sample_unique_candidates (lib.rs:3035-3048)
        while (cand.size() < pool + 1) push_unique(cand, rng.gen_range(0, n));
        std::vector<std::pair<size_t, float>> pairs;
        for (size_t j : cand) pairs.emplace_back(j, dist_fn(i, j));
        sorted_unique(pairs, k);
        for (size_t c = 0; c < k; ++c) {
            nb_idx[i * k + c] = pairs[c].first;
            nb_dist[i * k + c] = pairs[c].second;
        }
    }
    size_t ran = 0;
    for (size_t iteration = 0; iteration < n_iters; ++iteration) {
        std::vector<size_t> next_idx(n * k);
        std::vector<float> next_dist(n * k);
        int changed = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : changed)
        for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
            const size_t i = static_cast<size_t>(ii);
            SmallRng rng(mix_approx_seed(seed, i, iteration + 1));
            std::vector<size_t> out;
            out.reserve(max_candidates + k * k + 8);
            // collect_approx_candidate_indices (lib.rs:3051-3084)
            for (size_t c = 0; c < k; ++c) {
                const size_t idx = nb_idx[i * k + c];
                push_unique(out, idx);
                for (size_t c2 = 0; c2 < k; ++c2) push_unique(out, nb_idx[idx * k + c2]);
            }
            push_unique(out, i);
            const size_t exploration = std::min(std::max(k / 2, size_t(4)), max_candidates);
            for (size_t e = 0; e < exploration; ++e) push_unique(out, rng.gen_range(0, n));
            std::sort(out.begin(), out.end());
            if (out.size() > max_candidates) {
                for (size_t s = 0; s < max_candidates; ++s) {
                    const size_t r = rng.gen_range(s, out.size());
                    std::swap(out[s], out[r]);
                }
                out.resize(max_candidates);
            }
            std::vector<std::pair<size_t, float>> pairs;
            pairs.reserve(out.size());
            for (size_t j : out) pairs.emplace_back(j, dist_fn(i, j));
            sorted_unique(pairs, k);
            bool row_changed = pairs.size() != k;
            for (size_t c = 0; c < k && c < pairs.size(); ++c) {
                if (nb_idx[i * k + c] != pairs[c].first || nb_dist[i * k + c] != pairs[c].second)
                    row_changed = true;
                next_idx[i * k + c] = pairs[c].first;
                next_dist[i * k + c] = pairs[c].second;
            }
            if (row_changed) changed = 1;
        }
        nb_idx.swap(next_idx);
        nb_dist.swap(next_dist);
        ran = iteration + 1;
        if (!changed) break;
    }
    if (iters_run) *iters_run = ran;
    Knn out;
    out.idx.resize(n);
    out.dist.resize(n);
    for (size_t i = 0; i < n; ++i) {
        out.idx[i].assign(nb_idx.begin() + i * k, nb_idx.begin() + (i + 1) * k);
        out.dist[i].assign(nb_dist.begin() + i * k, nb_dist.begin() + (i + 1) * k);
    }
    return out;
}

// ------------------------------------------------------- find_ab_params ---
// curve_loss (lib.rs:5647-5658).
float curve_loss(float a, float b, const std::vector<float>& xv, const std::vector<float>& yv) {
    float loss = 0.0f;
    const float exponent = 2.0f * b;
    for (size_t i = 0; i < xv.size(); ++i) {
        const float model = 1.0f / (1.0f + a * powf(xv[i], exponent));
        const float e = model - yv[i];
        loss += e * e;
    }
    return loss / static_cast<float>(xv.size());
}

// curve_loss_from_powers (lib.rs:5660-5670).
float curve_loss_from_powers(float a, const std::vector<float>& xp, const std::vector<float>& yv) {
    float loss = 0.0f;
    for (size_t i = 0; i < xp.size(); ++i) {
        const float model = 1.0f / (1.0f + a * xp[i]);
        const float e = model - yv[i];
        loss += e * e;
    }
    return loss / static_cast<float>(xp.size());
}

// find_ab_params (lib.rs:5672-5746).
void find_ab_params(float spread, float min_dist, float* out_a, float* out_b) {
    const int n = 300;
    const float xmax = spread * 3.0f;
    std::vector<float> xv(n), yv(n);
    for (int i = 0; i < n; ++i) {
        const float x = xmax * static_cast<float>(i) / (static_cast<float>(n) - 1.0f);
        xv[i] = x;
        yv[i] = x < min_dist ? 1.0f : expf(-(x - min_dist) / spread);
    }
    float best_a = 1.0f, best_b = 1.0f, best_loss = std::numeric_limits<float>::infinity();
    std::vector<float> xp(n);
    for (int bi = 0; bi <= 70; ++bi) {
        const float b = 0.3f + 2.7f * static_cast<float>(bi) / 70.0f;
        const float exponent = 2.0f * b;
        for (int i = 0; i < n; ++i) xp[i] = powf(xv[i], exponent);
        for (int ai = 0; ai <= 120; ++ai) {
            const float log_a = -3.0f + 6.0f * static_cast<float>(ai) / 120.0f;
            const float a = powf(10.0f, log_a);
            const float loss = curve_loss_from_powers(a, xp, yv);
            if (loss < best_loss) {
                best_loss = loss;
                best_a = a;
                best_b = b;
            }
        }
    }
    float step_a = std::max(best_a * 0.35f, 0.05f);
    float step_b = 0.2f;
    for (int it = 0; it < 80; ++it) {
        const float am = std::max(best_a - step_a, 1e-6f);
        const float bm = std::max(best_b - step_b, 1e-6f);
        const float cand[8][2] = {
            {best_a + step_a, best_b}, {am, best_b},
            {best_a, best_b + step_b}, {best_a, bm},
            {best_a + step_a, best_b + step_b}, {best_a + step_a, bm},
            {am, best_b + step_b}, {am, bm}};
        bool improved = false;
        for (auto& c : cand) {
            const float loss = curve_loss(c[0], c[1], xv, yv);
            if (loss < best_loss) {
                best_loss = loss;
                best_a = c[0];
                best_b = c[1];
                improved = true;
            }
        }
        if (!improved) {
            step_a *= 0.7f;
            step_b *= 0.7f;
            if (step_a < 1e-5f && step_b < 1e-5f) break;
        }
    }
    *out_a = best_a;
    *out_b = best_b;
}

// ----------------------------------------------------- smooth_knn_dist ----
// knn_rows_include_self (lib.rs:3402-3417).
bool knn_rows_include_self(const Knn& knn) {
    for (size_t i = 0; i < knn.idx.size(); ++i) {
        if (knn.idx[i].empty() || knn.dist[i].empty()) return false;
        if (knn.idx[i][0] != i || std::fabs(knn.dist[i][0]) > SMOOTH_K_TOLERANCE) return false;
    }
    return true;
}

// smooth_knn_dist (lib.rs:3424-3523), templated so the same statement runs
// in FP32 (the reference) and FP64 (the precision oracle).
template <typename T>
void smooth_knn_dist_t(const std::vector<std::vector<float>>& distances, T k, T local_conn,
                       T bandwidth, bool include_self, std::vector<T>& sigmas,
                       std::vector<T>& rhos) {
    const T target = std::log2(k) * bandwidth;
    const size_t n = distances.size();
    T total = 0;
    size_t count = 0;
    for (const auto& row : distances) {
        const size_t start = (include_self && !row.empty()) ? 1 : 0;
        for (size_t c = start; c < row.size(); ++c) {
            total += static_cast<T>(row[c]);
            count++;
        }
    }
    const T mean_distances = count > 0 ? total / static_cast<T>(count) : T(0);
    sigmas.assign(n, T(0));
    rhos.assign(n, T(0));
    std::vector<T> nz;
    for (size_t i = 0; i < n; ++i) {
        const auto& row = distances[i];
        const size_t start = (include_self && !row.empty()) ? 1 : 0;
        const size_t m = row.size() - start;
        nz.clear();
        for (size_t c = start; c < row.size(); ++c)
            if (row[c] > 0.0f) nz.push_back(static_cast<T>(row[c]));
        T mean_ith = 0;
        if (m > 0) {
            T s = 0;
            for (size_t c = start; c < row.size(); ++c) s += static_cast<T>(row[c]);
            mean_ith = s / static_cast<T>(m);
        }
        if (static_cast<T>(nz.size()) >= local_conn) {
            const size_t index = static_cast<size_t>(std::floor(local_conn));
            const T interpolation = local_conn - static_cast<T>(index);
            if (index > 0) {
                rhos[i] = nz[index - 1];
                if (interpolation > static_cast<T>(SMOOTH_K_TOLERANCE) && index < nz.size())
                    rhos[i] += interpolation * (nz[index] - nz[index - 1]);
            } else if (!nz.empty()) {
                rhos[i] = interpolation * nz[0];
            }
        } else if (!nz.empty()) {
            T mx = nz[0];
            for (T v : nz) mx = std::max(mx, v);
            rhos[i] = mx;
        }
        T lo = 0, hi = std::numeric_limits<T>::infinity(), mid = 1;
        for (int it = 0; it < 64; ++it) {
            T psum = 0;
            for (size_t c = start; c < row.size(); ++c) {
                const T dd = static_cast<T>(row[c]) - rhos[i];
                if (dd > 0)
                    psum += std::exp(-(dd / mid));
                else
                    psum += 1;
            }
            if (std::fabs(psum - target) < static_cast<T>(SMOOTH_K_TOLERANCE)) break;
            if (psum > target) {
                hi = mid;
                mid = (lo + hi) / 2;
            } else {
                lo = mid;
                if (std::isinf(hi))
                    mid *= 2;
                else
                    mid = (lo + hi) / 2;
            }
        }
        const T min_scale = rhos[i] > 0 ? static_cast<T>(MIN_K_DIST_SCALE) * mean_ith
                                        : static_cast<T>(MIN_K_DIST_SCALE) * mean_distances;
        sigmas[i] = std::max(mid, min_scale);
    }
}

inline float expf_ref(float x) { return expf(x); }

struct Edge {
    size_t head, tail;
    float weight;
};

// compute_membership_strengths (lib.rs:3525-3560).
std::vector<Edge> membership(const Knn& knn, const std::vector<float>& sig,
                             const std::vector<float>& rho) {
    std::vector<Edge> out;
    for (size_t i = 0; i < knn.idx.size(); ++i) {
        for (size_t j = 0; j < knn.idx[i].size(); ++j) {
            const size_t nb = knn.idx[i][j];
            const float d = knn.dist[i][j];
            float val;
            if (nb == i)
                val = 0.0f;
            else if (d - rho[i] <= 0.0f || sig[i] == 0.0f)
                val = 1.0f;
            else
                val = expf(-(d - rho[i]) / sig[i]);
            if (val > 0.0f) out.push_back({i, nb, val});
        }
    }
    return out;
}

// compute_membership_strengths_bipartite (lib.rs:3562-3595).
std::vector<Edge> membership_bipartite(const Knn& knn, const std::vector<float>& sig,
                                       const std::vector<float>& rho) {
    std::vector<Edge> out;
    for (size_t i = 0; i < knn.idx.size(); ++i) {
        for (size_t j = 0; j < knn.idx[i].size(); ++j) {
            const float d = knn.dist[i][j];
            float val;
            if (d - rho[i] <= 0.0f || sig[i] == 0.0f)
                val = 1.0f;
            else
                val = expf(-(d - rho[i]) / sig[i]);
            if (val > 0.0f) out.push_back({i, knn.idx[i][j], val});
        }
    }
    return out;
}

// symmetrize_fuzzy_graph (lib.rs:3597-3649).
std::vector<Edge> symmetrize(const std::vector<Edge>& directed, float mix) {
    struct P {
        size_t i, j;
        float wij, wji;
    };
    std::vector<P> by_pair;
    by_pair.reserve(directed.size());
    for (const auto& e : directed) {
        if (e.head == e.tail) continue;
        if (e.head < e.tail)
            by_pair.push_back({e.head, e.tail, e.weight, 0.0f});
        else
            by_pair.push_back({e.tail, e.head, 0.0f, e.weight});
    }
    std::stable_sort(by_pair.begin(), by_pair.end(), [](const P& a, const P& b) {
        return a.i != b.i ? a.i < b.i : a.j < b.j;
    });
    std::vector<Edge> edges;
    edges.reserve(by_pair.size() * 2);
    size_t idx = 0;
    while (idx < by_pair.size()) {
        const size_t i = by_pair[idx].i, j = by_pair[idx].j;
        float wij = 0.0f, wji = 0.0f;
        while (idx < by_pair.size() && by_pair[idx].i == i && by_pair[idx].j == j) {
            if (by_pair[idx].wij > 0.0f) wij = by_pair[idx].wij;
            if (by_pair[idx].wji > 0.0f) wji = by_pair[idx].wji;
            idx++;
        }
        const float prod = wij * wji;
        const float sym = mix * (wij + wji - prod) + (1.0f - mix) * prod;
        if (sym > 0.0f) {
            edges.push_back({i, j, sym});
            edges.push_back({j, i, sym});
        }
    }
    std::stable_sort(edges.begin(), edges.end(), [](const Edge& a, const Edge& b) {
        return a.head != b.head ? a.head < b.head : a.tail < b.tail;
    });
    return edges;
}

// prune_edges (lib.rs:3804-3822).
void prune_edges(std::vector<Edge>& edges, size_t n_epochs) {
    if (edges.empty()) return;
    float mx = -std::numeric_limits<float>::infinity();
    for (const auto& e : edges) mx = std::max(mx, e.weight);
    const float denom = n_epochs > 10 ? static_cast<float>(n_epochs) : 500.0f;
    const float thr = mx / denom;
    std::vector<Edge> kept;
    kept.reserve(edges.size());
    for (const auto& e : edges)
        if (e.weight >= thr && e.weight > 0.0f) kept.push_back(e);
    edges.swap(kept);
}

// apply_categorical_target_intersection + reset_local_connectivity_edges
// (lib.rs:3694-3760): every edge's weight times 1 (same label), exp(-1)
// (either label -1) or exp(-far_dist) (different labels), with
// far_dist = 2.5 / (1 - weight) (1e12 at weight 1), all in FP32; edges whose
// product is not positive and finite are dropped; each head's edges are
// divided by its largest weight; the result is the fuzzy union (mix 1) of
// those directed edges.  A weight <= 0 or an empty graph returns the input.
std::vector<Edge> categorical_intersection(const std::vector<Edge>& edges, const int64_t* labels,
                                           size_t n, float weight) {
    if (weight <= 0.0f || edges.empty()) return edges;
    const float far_dist = weight < 1.0f ? 2.5f / (1.0f - weight) : 1.0e12f;
    const float unknown_scale = std::exp(-1.0f);
    const float far_scale = std::exp(-far_dist);
    std::vector<Edge> scaled;
    scaled.reserve(edges.size());
    for (const auto& e : edges) {
        const int64_t lhs = labels[e.head], rhs = labels[e.tail];
        const float scale =
            (lhs == -1 || rhs == -1) ? unknown_scale : (lhs != rhs ? far_scale : 1.0f);
        const float w = e.weight * scale;
        if (w > 0.0f && std::isfinite(w)) scaled.push_back({e.head, e.tail, w});
    }
    if (scaled.empty()) return {};
    std::vector<float> row_max(n, 0.0f);
    for (const auto& e : scaled) row_max[e.head] = std::max(row_max[e.head], e.weight);
    std::vector<Edge> directed;
    directed.reserve(scaled.size());
    for (const auto& e : scaled) {
        const float mx = row_max[e.head];
        if (mx <= 0.0f || !std::isfinite(mx)) continue;
        directed.push_back({e.head, e.tail, e.weight / mx});
    }
    return symmetrize(directed, 1.0f);
}

// random_init (lib.rs:3824-3839).
std::vector<std::vector<float>> random_init(size_t n, size_t dim, uint64_t seed, float low,
                                            float high) {
    SmallRng rng(seed);
    std::vector<std::vector<float>> out(n, std::vector<float>(dim));
    for (size_t i = 0; i < n; ++i)
        for (size_t c = 0; c < dim; ++c) out[i][c] = rng.gen_range_f32(low, high);
    return out;
}

// ------------------------------------------------------- eigensolver -----
// Symmetric eigendecomposition: Householder reduction to tridiagonal form
// followed by the implicit QL algorithm (the EISPACK tred2/tql2 pair).
// A is n x n row-major; returns ascending eigenvalues in `w` and the
// eigenvectors as columns of `V` (row-major, V[r*n + c]).
void symmetric_eigen(const std::vector<double>& A, size_t n, std::vector<double>& w,
                     std::vector<double>& V) {
    V = A;
    std::vector<double> d(n), e(n);
    auto v = [&](size_t r, size_t c) -> double& { return V[r * n + c]; };
    for (size_t j = 0; j < n; ++j) d[j] = v(n - 1, j);
    for (size_t i = n - 1; i > 0; --i) {
        double scale = 0.0, h = 0.0;
        for (size_t k = 0; k < i; ++k) scale += std::fabs(d[k]);
        if (scale == 0.0) {
            e[i] = d[i - 1];
            for (size_t j = 0; j < i; ++j) {
                d[j] = v(i - 1, j);
                v(i, j) = 0.0;
                v(j, i) = 0.0;
            }
        } else {
            for (size_t k = 0; k < i; ++k) {
                d[k] /= scale;
                h += d[k] * d[k];
            }
            double f = d[i - 1];
            double g = std::sqrt(h);
            if (f > 0) g = -g;
            e[i] = scale * g;
            h = h - f * g;
            d[i - 1] = f - g;
            for (size_t j = 0; j < i; ++j) e[j] = 0.0;
            for (size_t j = 0; j < i; ++j) {
                f = d[j];
                v(j, i) = f;
                g = e[j] + v(j, j) * f;
                for (size_t k = j + 1; k <= i - 1; ++k) {
                    g += v(k, j) * d[k];
                    e[k] += v(k, j) * f;
                }
                e[j] = g;
            }
            f = 0.0;
            for (size_t j = 0; j < i; ++j) {
                e[j] /= h;
                f += e[j] * d[j];
            }
            const double hh = f / (h + h);
            for (size_t j = 0; j < i; ++j) e[j] -= hh * d[j];
            for (size_t j = 0; j < i; ++j) {
                f = d[j];
                g = e[j];
                for (size_t k = j; k <= i - 1; ++k) v(k, j) -= (f * e[k] + g * d[k]);
                d[j] = v(i - 1, j);
                v(i, j) = 0.0;
            }
        }
        d[i] = h;
    }
    for (size_t i = 0; i + 1 < n; ++i) {
        v(n - 1, i) = v(i, i);
        v(i, i) = 1.0;
        const double h = d[i + 1];
        if (h != 0.0) {
            for (size_t k = 0; k <= i; ++k) d[k] = v(k, i + 1) / h;
            for (size_t j = 0; j <= i; ++j) {
                double g = 0.0;
                for (size_t k = 0; k <= i; ++k) g += v(k, i + 1) * v(k, j);
                for (size_t k = 0; k <= i; ++k) v(k, j) -= g * d[k];
            }
        }
        for (size_t k = 0; k <= i; ++k) v(k, i + 1) = 0.0;
    }
    for (size_t j = 0; j < n; ++j) {
        d[j] = v(n - 1, j);
        v(n - 1, j) = 0.0;
    }
    v(n - 1, n - 1) = 1.0;
    e[0] = 0.0;
    // tql2
    for (size_t i = 1; i < n; ++i) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    double f = 0.0, tst1 = 0.0;
    const double eps = std::ldexp(1.0, -52);
    for (size_t l = 0; l < n; ++l) {
        tst1 = std::max(tst1, std::fabs(d[l]) + std::fabs(e[l]));
        size_t m = l;
        while (m < n) {
            if (std::fabs(e[m]) <= eps * tst1) break;
            m++;
        }
        if (m == n) m = n - 1;
        if (m > l) {
            int iter = 0;
            do {
                iter++;
                double g = d[l];
                double p = (d[l + 1] - g) / (2.0 * e[l]);
                double r = std::hypot(p, 1.0);
                if (p < 0) r = -r;
                d[l] = e[l] / (p + r);
                d[l + 1] = e[l] * (p + r);
                const double dl1 = d[l + 1];
                double h = g - d[l];
                for (size_t i = l + 2; i < n; ++i) d[i] -= h;
                f += h;
                p = d[m];
                double c = 1.0, c2 = 1.0, c3 = 1.0, s = 0.0, s2 = 0.0;
                const double el1 = e[l + 1];
                for (size_t ii = m; ii-- > l;) {
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    g = c * e[ii];
                    h = c * p;
                    r = std::hypot(p, e[ii]);
                    e[ii + 1] = s * r;
                    s = e[ii] / r;
                    c = p / r;
                    p = c * d[ii] - s * g;
                    d[ii + 1] = h + s * (c * g + s * d[ii]);
                    for (size_t k = 0; k < n; ++k) {
                        h = v(k, ii + 1);
                        v(k, ii + 1) = s * v(k, ii) + c * h;
                        v(k, ii) = c * v(k, ii) - s * h;
                    }
                }
                p = -s * s2 * c3 * el1 * e[l] / dl1;
                e[l] = s * p;
                d[l] = c * p;
            } while (std::fabs(e[l]) > eps * tst1 && iter < 200);
        }
        d[l] = d[l] + f;
        e[l] = 0.0;
    }
    // sort ascending (stable on ties, keeps the QL column order)
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return d[a] < d[b]; });
    w.resize(n);
    std::vector<double> Vs(n * n);
    for (size_t c = 0; c < n; ++c) {
        w[c] = d[order[c]];
        for (size_t r = 0; r < n; ++r) Vs[r * n + c] = V[r * n + order[c]];
    }
    V.swap(Vs);
}

// ------------------------------------------------------------ spectral ---
using Coords = std::vector<std::vector<float>>;

bool all_finite(const Coords& c) {
    for (const auto& r : c)
        for (float v : r)
            if (!std::isfinite(v)) return false;
    return true;
}

// spectral_embedding_from_laplacian (lib.rs:3917-3957).
bool embedding_from_laplacian(const std::vector<double>& L, size_t n, size_t dim,
                              bool drop_first, Coords& out) {
    if (n == 0) return false;
    std::vector<double> w, V;
    symmetric_eigen(L, n, w, V);
    const size_t offset = drop_first ? 1 : 0;
    if (n <= dim + offset) return false;
    out.assign(n, std::vector<float>(dim));
    for (size_t c = 0; c < dim; ++c)
        for (size_t r = 0; r < n; ++r) out[r][c] = static_cast<float>(V[r * n + c + offset]);
    return all_finite(out);
}

// normalized_laplacian_from_affinity (lib.rs:3959-4005).
bool laplacian_from_affinity(const std::vector<double>& aff, size_t n, std::vector<double>& L) {
    if (n == 0) return false;
    std::vector<double> deg(n, 0.0);
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) deg[i] += aff[i * n + j];
    bool any = false;
    for (double v : deg) any |= v > 0.0;
    if (!any) return false;
    std::vector<double> inv(n);
    for (size_t i = 0; i < n; ++i) inv[i] = deg[i] > 0 ? 1.0 / std::sqrt(deg[i]) : 0.0;
    L.assign(n * n, 0.0);
    for (size_t i = 0; i < n; ++i) L[i * n + i] = 1.0;
    for (size_t i = 0; i < n; ++i) {
        if (deg[i] <= 0) continue;
        for (size_t j = 0; j < n; ++j) {
            if (deg[j] <= 0) continue;
            const double wgt = aff[i * n + j];
            if (wgt > 0.0) L[i * n + j] -= wgt * inv[i] * inv[j];
        }
    }
    return true;
}

// normalized_laplacian_from_edges (lib.rs:4007-4069).
bool laplacian_from_edges(size_t n, const std::vector<Edge>& edges, std::vector<double>& L) {
    if (n == 0 || edges.empty()) return false;
    L.assign(n * n, 0.0);
    for (size_t i = 0; i < n; ++i) L[i * n + i] = 1.0;
    std::vector<double> deg(n, 0.0);
    std::vector<std::pair<size_t, size_t>> pairs;
    for (const auto& e : edges) {
        if (e.head == e.tail) continue;
        const double wgt = static_cast<double>(std::max(e.weight, 0.0f));
        if (wgt <= 0.0) continue;
        const size_t i = std::min(e.head, e.tail), j = std::max(e.head, e.tail);
        const double prev = L[i * n + j];
        if (wgt > prev) {
            if (prev == 0.0) pairs.emplace_back(i, j);
            const double delta = wgt - prev;
            L[i * n + j] = wgt;
            L[j * n + i] = wgt;
            deg[i] += delta;
            deg[j] += delta;
        }
    }
    bool any = false;
    for (double v : deg) any |= v > 0.0;
    if (!any) return false;
    std::vector<double> inv(n);
    for (size_t i = 0; i < n; ++i) inv[i] = deg[i] > 0 ? 1.0 / std::sqrt(deg[i]) : 0.0;
    for (auto [i, j] : pairs) {
        const double nv = L[i * n + j] * inv[i] * inv[j];
        L[i * n + j] = -nv;
        L[j * n + i] = -nv;
    }
    for (size_t i = 0; i < n; ++i) L[i * n + i] = 1.0;
    return true;
}

// orthonormalize_columns (lib.rs:4161-4199): MGS applied twice per column.
bool orthonormalize(std::vector<double>& B, size_t rows, size_t cols) {
    if (rows == 0 || cols == 0) return false;
    for (size_t c = 0; c < cols; ++c) {
        for (int pass = 0; pass < 2; ++pass) {
            for (size_t p = 0; p < c; ++p) {
                double dot = 0.0;
                for (size_t r = 0; r < rows; ++r) dot += B[r * cols + c] * B[r * cols + p];
                for (size_t r = 0; r < rows; ++r) B[r * cols + c] -= dot * B[r * cols + p];
            }
        }
        double nsq = 0.0;
        for (size_t r = 0; r < rows; ++r) nsq += B[r * cols + c] * B[r * cols + c];
        if (!std::isfinite(nsq) || nsq <= SPECTRAL_ORTHO_EPS) return false;
        const double inv = 1.0 / std::sqrt(nsq);
        for (size_t r = 0; r < rows; ++r) B[r * cols + c] *= inv;
    }
    return true;
}

struct UEdge {
    size_t i, j;
    double w;
};

// symmetrized_undirected_edges (lib.rs:4107-4159).
bool undirected_edges(size_t n, const std::vector<Edge>& edges, std::vector<UEdge>& out,
                      std::vector<double>& deg) {
    if (n == 0 || edges.empty()) return false;
    std::map<std::pair<size_t, size_t>, double> by_pair;
    for (const auto& e : edges) {
        if (e.head == e.tail) continue;
        const double w = static_cast<double>(std::max(e.weight, 0.0f));
        if (w <= 0.0) continue;
        const auto key = std::make_pair(std::min(e.head, e.tail), std::max(e.head, e.tail));
        auto it = by_pair.find(key);
        if (it == by_pair.end())
            by_pair.emplace(key, w);
        else if (w > it->second)
            it->second = w;
    }
    if (by_pair.empty()) return false;
    deg.assign(n, 0.0);
    out.clear();
    for (const auto& [k, w] : by_pair) {
        deg[k.first] += w;
        deg[k.second] += w;
        out.push_back({k.first, k.second, w});
    }
    bool any = false;
    for (double v : deg) any |= v > 0.0;
    return any;
}

// shifted_normalized_adjacency_mul (lib.rs:4201-4225).
void shifted_mul(const std::vector<double>& X, size_t n, size_t s, const std::vector<UEdge>& ue,
                 const std::vector<double>& inv, std::vector<double>& out) {
    out = X;
    for (const auto& e : ue) {
        const double nv = e.w * inv[e.i] * inv[e.j];
        if (nv == 0.0) continue;
        for (size_t c = 0; c < s; ++c) {
            const double xi = X[e.i * s + c], xj = X[e.j * s + c];
            out[e.i * s + c] += nv * xj;
            out[e.j * s + c] += nv * xi;
        }
    }
}

// spectral_embedding_from_edges_iterative (lib.rs:4227-4326).
bool spectral_iterative(size_t n, size_t dim, const std::vector<Edge>& edges, uint64_t seed,
                        Coords& out) {
    const size_t s = std::max((dim + 1) * SPECTRAL_ITERATIVE_OVERSAMPLING, dim + 1);
    if (n <= s || edges.empty()) return false;
    std::vector<UEdge> ue;
    std::vector<double> deg;
    if (!undirected_edges(n, edges, ue, deg)) return false;
    std::vector<double> inv(n);
    for (size_t i = 0; i < n; ++i) inv[i] = deg[i] > 0 ? 1.0 / std::sqrt(deg[i]) : 0.0;
    SmallRng rng(seed ^ 0x7A5B3D91CE42A117ULL);
    std::vector<double> B(n * s, 0.0);
    for (size_t r = 0; r < n; ++r) {
        B[r * s] = std::sqrt(deg[r]);
        for (size_t c = 1; c < s; ++c) B[r * s + c] = rng.gen_range_f64(-1.0, 1.0);
    }
    if (!orthonormalize(B, n, s)) return false;
    std::vector<double> scratch;
    for (size_t it = 0; it < SPECTRAL_ITERATIVE_MAX_ITERS; ++it) {
        shifted_mul(B, n, s, ue, inv, scratch);
        if (!orthonormalize(scratch, n, s)) return false;
        B.swap(scratch);
    }
    shifted_mul(B, n, s, ue, inv, scratch);
    std::vector<double> ritz(s * s, 0.0);
    for (size_t i = 0; i < s; ++i)
        for (size_t j = i; j < s; ++j) {
            double v = 0.0;
            for (size_t r = 0; r < n; ++r) v += B[r * s + i] * scratch[r * s + j];
            ritz[i * s + j] = v;
            ritz[j * s + i] = v;
        }
    std::vector<double> w, V;
    symmetric_eigen(ritz, s, w, V);
    // descending eigenvalue order; reversed ascending order (stable on ties)
    std::vector<size_t> order(s);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return w[a] > w[b]; });
    if (order.size() <= dim) return false;
    out.assign(n, std::vector<float>(dim));
    for (size_t oc = 0; oc < dim; ++oc) {
        const size_t ec = order[oc + 1];
        for (size_t r = 0; r < n; ++r) {
            double v = 0.0;
            for (size_t b = 0; b < s; ++b) v += B[r * s + b] * V[b * s + ec];
            out[r][oc] = static_cast<float>(v);
        }
    }
    return all_finite(out);
}

// spectral_embedding_from_edges (lib.rs:4328-4353).
bool spectral_from_edges(size_t n, size_t dim, const std::vector<Edge>& edges, uint64_t seed,
                         size_t iterative_threshold, Coords& out) {
    if (n <= dim + 1 || edges.empty()) return false;
    if (n >= iterative_threshold) {
        if (spectral_iterative(n, dim, edges, seed, out)) return true;
        if (n > SPECTRAL_DENSE_FALLBACK_MAX_SAMPLES) return false;
    }
    std::vector<double> L;
    if (!laplacian_from_edges(n, edges, L)) return false;
    return embedding_from_laplacian(L, n, dim, true, out);
}

// add_noise (lib.rs:4580-4593).
void add_noise(Coords& c, uint64_t seed, float noise) {
    if (c.empty() || c[0].empty()) return;
    SmallRng rng(seed);
    for (auto& r : c)
        for (auto& v : r) v += static_cast<float>(rng.normal(noise));
}

// noisy_scale_coords (lib.rs:4766-4791).
void noisy_scale_coords(Coords& c, uint64_t seed, float max_coord, float noise) {
    if (c.empty() || c[0].empty()) return;
    float mx = 0.0f;
    for (const auto& r : c)
        for (float v : r) mx = std::max(mx, std::fabs(v));
    const float expansion = mx > 0.0f ? max_coord / mx : 1.0f;
    SmallRng rng(seed);
    for (auto& r : c)
        for (auto& v : r) v = v * expansion + static_cast<float>(rng.normal(noise));
}

// connected_components_from_edges (lib.rs:4383-4435): components sorted by
// smallest member, members ascending.
std::vector<std::vector<size_t>> connected_components(size_t n, const std::vector<Edge>& edges) {
    std::vector<size_t> parent(n);
    std::iota(parent.begin(), parent.end(), 0);
    std::vector<uint8_t> rank(n, 0);
    auto find = [&](size_t x) {
        size_t r = x;
        while (parent[r] != r) r = parent[r];
        while (parent[x] != r) {
            const size_t nx = parent[x];
            parent[x] = r;
            x = nx;
        }
        return r;
    };
    for (const auto& e : edges) {
        if (e.head == e.tail) continue;
        const size_t a = find(e.head), b = find(e.tail);
        if (a == b) continue;
        if (rank[a] < rank[b])
            parent[a] = b;
        else if (rank[a] > rank[b])
            parent[b] = a;
        else {
            parent[b] = a;
            rank[a]++;
        }
    }
    std::unordered_map<size_t, std::vector<size_t>> groups;
    for (size_t i = 0; i < n; ++i) groups[find(i)].push_back(i);
    std::vector<std::vector<size_t>> comps;
    for (auto& [k, v] : groups) comps.push_back(std::move(v));
    std::sort(comps.begin(), comps.end(),
              [](const auto& a, const auto& b) { return a[0] < b[0]; });
    return comps;
}

// meta_component_layout_from_centroids (lib.rs:4519-4554) with
// spectral_embedding_from_affinity (lib.rs:4576-4592).
bool meta_layout(const std::vector<std::vector<double>>& cents, size_t dim, uint64_t seed,
                 Coords& out) {
    const size_t m = cents.size();
    if (m == 0) return false;
    if (m == 1) {
        out.assign(1, std::vector<float>(dim, 0.0f));
        return true;
    }
    if (m <= 2 * dim) {
        const size_t k = (m + 1) / 2;
        out.assign(m, std::vector<float>(dim, 0.0f));
        for (size_t i = 0; i < m; ++i) out[i][i % k] = i < k ? 1.0f : -1.0f;
        return true;
    }
    std::vector<double> aff(m * m, 0.0);
    for (size_t i = 0; i < m; ++i) {
        aff[i * m + i] = 1.0;
        for (size_t j = i + 1; j < m; ++j) {
            double d2 = 0.0;
            for (size_t f = 0; f < cents[i].size(); ++f) {
                const double dd = cents[i][f] - cents[j][f];
                d2 += dd * dd;
            }
            const double w = std::exp(-d2);
            aff[i * m + j] = w;
            aff[j * m + i] = w;
        }
    }
    std::vector<double> L;
    if (!laplacian_from_affinity(aff, m, L)) return false;
    if (!embedding_from_laplacian(L, m, dim, true, out)) return false;
    noisy_scale_coords(out, seed ^ 0xC85E7D6ADA318F21ULL, INIT_MAX_COORD, INIT_NOISE);
    return all_finite(out);
}

// multi_component_spectral_init{,_with_layout} (lib.rs:4594-4764).
bool multi_component_init(const float* data, size_t n, size_t d, size_t dim,
                          const std::vector<Edge>& edges,
                          const std::vector<std::vector<size_t>>& comps, uint64_t seed,
                          Coords& result) {
    std::vector<std::vector<double>> cents;  // component_centroids_dense (lib.rs:4463-4485)
    for (const auto& comp : comps) {
        std::vector<double> c(d, 0.0);
        for (size_t idx : comp)
            for (size_t f = 0; f < d; ++f) c[f] += static_cast<double>(data[idx * d + f]);
        const double sc = 1.0 / static_cast<double>(comp.size());
        for (auto& v : c) v *= sc;
        cents.push_back(std::move(c));
    }
    Coords layout;
    if (!meta_layout(cents, dim, seed ^ 0xA13F52A92D4CB801ULL, layout)) return false;
    if (layout.size() != comps.size()) return false;
    std::vector<size_t> labels(n, SIZE_MAX);
    for (size_t c = 0; c < comps.size(); ++c)
        for (size_t idx : comps[c]) labels[idx] = c;
    result.assign(n, std::vector<float>(dim, 0.0f));
    for (size_t cid = 0; cid < comps.size(); ++cid) {
        const auto& comp = comps[cid];
        const auto& anchor = layout[cid];
        float data_range = std::numeric_limits<float>::infinity();
        for (size_t o = 0; o < layout.size(); ++o) {
            if (o == cid) continue;
            const float dist = std::sqrt(squared_distance(anchor.data(), layout[o].data(), dim));
            if (dist > 0.0f) data_range = std::min(data_range, dist / 2.0f);
        }
        if (!std::isfinite(data_range) || data_range <= 0.0f) data_range = 1.0f;
        Coords local;
        if (comp.size() < 2 * dim || comp.size() <= dim + 1) {
            local = random_init(comp.size(), dim, seed ^ ((cid + 1) * 0x9E3779B9ULL), -data_range,
                                data_range);
        } else {
            // remap_component_edges (lib.rs:4437-4461)
            std::vector<size_t> map(n, SIZE_MAX);
            for (size_t li = 0; li < comp.size(); ++li) map[comp[li]] = li;
            std::vector<Edge> ce;
            for (const auto& e : edges)
                if (labels[e.head] == cid && labels[e.tail] == cid)
                    ce.push_back({map[e.head], map[e.tail], e.weight});
            if (!spectral_from_edges(comp.size(), dim, ce,
                                     seed ^ ((cid + 1) * 0xBF58476D1CE4E5B9ULL),
                                     SPECTRAL_ITERATIVE_COMPONENT_THRESHOLD, local))
                return false;
            float mx = 0.0f;
            for (const auto& r : local)
                for (float v : r) mx = std::max(mx, std::fabs(v));
            const float expansion = mx > 0.0f ? data_range / mx : 1.0f;
            for (auto& r : local)
                for (auto& v : r) v *= expansion;
            add_noise(local, seed ^ ((cid + 1) * 0x94D049BBULL), INIT_NOISE);
        }
        for (size_t li = 0; li < comp.size(); ++li)
            for (size_t c = 0; c < dim; ++c) result[comp[li]][c] = local[li][c] + anchor[c];
    }
    return all_finite(result);
}

// spectral_init (lib.rs:3871-3888) + spectral_init_connected (lib.rs:4360-4381).
bool spectral_init(const float* data, size_t n, size_t d, size_t dim,
                   const std::vector<Edge>& edges, uint64_t seed, Coords& out,
                   size_t* n_components) {
    if (n <= dim + 1 || edges.empty()) return false;
    const auto comps = connected_components(n, edges);
    if (n_components) *n_components = comps.size();
    if (comps.size() > 1) return multi_component_init(data, n, d, dim, edges, comps, seed, out);
    const size_t thr = d <= SPECTRAL_EXACT_LOW_DIM_MAX_FEATURES
                           ? SPECTRAL_EXACT_LOW_DIM_MAX_SAMPLES + 1
                           : SPECTRAL_ITERATIVE_CONNECTED_THRESHOLD;
    if (!spectral_from_edges(n, dim, edges, seed, thr, out)) return false;
    noisy_scale_coords(out, seed ^ 0x5DEECE66DULL, INIT_MAX_COORD, INIT_NOISE);
    return all_finite(out);
}

// initialize_embedding (lib.rs:3841-3854).
Coords initialize_embedding(const float* data, size_t n, size_t d, size_t dim,
                            const std::vector<Edge>& edges, int init, uint64_t seed,
                            int* used_spectral, size_t* n_components) {
    Coords out;
    if (init == UMAPB_INIT_SPECTRAL && spectral_init(data, n, d, dim, edges, seed, out,
                                                     n_components)) {
        if (used_spectral) *used_spectral = 1;
        return out;
    }
    if (used_spectral) *used_spectral = 0;
    return random_init(n, dim, seed, -10.0f, 10.0f);
}

// ---------------------------------------------------------------- SGD -----
// make_epochs_per_sample (lib.rs:4937-4960).
std::vector<float> epochs_per_sample(const std::vector<float>& w, size_t n_epochs) {
    if (w.empty()) return {};
    float mx = -std::numeric_limits<float>::infinity();
    for (float v : w) mx = std::max(mx, v);
    mx = std::max(mx, 1e-12f);
    std::vector<float> out(w.size());
    for (size_t i = 0; i < w.size(); ++i) {
        const float ns = static_cast<float>(n_epochs) * (w[i] / mx);
        out[i] = ns > 0.0f ? static_cast<float>(n_epochs) / ns
                           : std::numeric_limits<float>::infinity();
    }
    return out;
}

inline float clip4(float v) { return std::min(std::max(v, -4.0f), 4.0f); }  // lib.rs:4962

inline size_t floor_to_usize(float v) {
    const float f = std::floor(v);
    if (!(f > 0.0f)) return 0;  // NaN and negatives saturate to 0
    if (f >= 1.8446744e19f) return SIZE_MAX;
    return static_cast<size_t>(f);
}

// optimize_layout_training_flat (lib.rs:5137-5321), dim == 2 fast path and
// the general path; strictly sequential with one RNG stream.
double optimize_layout_training(std::vector<float>& flat, size_t n_vertices, size_t dim,
                                const std::vector<Edge>& edges, size_t n_epochs, float a, float b,
                                float initial_alpha, size_t neg_rate, float repulsion,
                                uint64_t seed) {
    if (edges.empty() || n_vertices == 0 || n_epochs == 0) return 0.0;
    std::vector<float> w(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) w[i] = edges[i].weight;
    const auto eps = epochs_per_sample(w, n_epochs);
    auto next = eps;
    std::vector<float> eps_neg(eps.size());
    for (size_t i = 0; i < eps.size(); ++i) eps_neg[i] = eps[i] / static_cast<float>(neg_rate);
    auto next_neg = eps_neg;
    SmallRng rng(seed);
    const float rep_factor = 2.0f * repulsion * b;
    const float att_factor = -2.0f * a * b;
    double samples = 0.0;
    for (size_t epoch = 0; epoch < n_epochs; ++epoch) {
        const float alpha =
            initial_alpha * (1.0f - static_cast<float>(epoch) / static_cast<float>(n_epochs));
        const float ef = static_cast<float>(epoch);
        for (size_t e = 0; e < edges.size(); ++e) {
            if (next[e] > ef) continue;
            samples += 1.0;
            const size_t head = edges[e].head, tail = edges[e].tail;
            if (head != tail) {
                if (dim == 2) {
                    const float dx = flat[head * 2] - flat[tail * 2];
                    const float dy = flat[head * 2 + 1] - flat[tail * 2 + 1];
                    const float d2 = dx * dx + dy * dy;
                    if (d2 > 0.0f) {
                        const float pb = powf(d2, b);
                        const float gc = att_factor * (pb / d2) / (a * pb + 1.0f);
                        const float gx = clip4(gc * dx), gy = clip4(gc * dy);
                        flat[head * 2] += gx * alpha;
                        flat[head * 2 + 1] += gy * alpha;
                        flat[tail * 2] -= gx * alpha;
                        flat[tail * 2 + 1] -= gy * alpha;
                    }
                } else {
                    float d2 = 0.0f;
                    for (size_t c = 0; c < dim; ++c) {
                        const float df = flat[head * dim + c] - flat[tail * dim + c];
                        d2 += df * df;
                    }
                    if (d2 > 0.0f) {
                        const float pb = powf(d2, b);
                        const float gc = att_factor * (pb / d2) / (a * pb + 1.0f);
                        for (size_t c = 0; c < dim; ++c) {
                            const float hv = flat[head * dim + c], tv = flat[tail * dim + c];
                            const float g = clip4(gc * (hv - tv));
                            flat[head * dim + c] = hv + g * alpha;
                            flat[tail * dim + c] = tv - g * alpha;
                        }
                    }
                }
            }
            next[e] += eps[e];
            const float en = eps_neg[e];
            if (!std::isfinite(en) || en <= 0.0f) continue;
            const size_t nneg = floor_to_usize((ef - next_neg[e]) / en);
            for (size_t s = 0; s < nneg; ++s) {
                const size_t neg = rng.gen_range(0, n_vertices);
                if (neg == head) continue;
                float d2 = 0.0f;
                if (dim == 2) {
                    const float dx = flat[head * 2] - flat[neg * 2];
                    const float dy = flat[head * 2 + 1] - flat[neg * 2 + 1];
                    d2 = dx * dx + dy * dy;
                } else {
                    for (size_t c = 0; c < dim; ++c) {
                        const float df = flat[head * dim + c] - flat[neg * dim + c];
                        d2 += df * df;
                    }
                }
                if (d2 > 0.0f) {
                    const float pb = powf(d2, b);
                    const float gc = rep_factor / ((0.001f + d2) * (a * pb + 1.0f));
                    if (gc > 0.0f) {
                        for (size_t c = 0; c < dim; ++c) {
                            const float hv = flat[head * dim + c], nv = flat[neg * dim + c];
                            const float g = clip4(gc * (hv - nv));
                            flat[head * dim + c] = hv + g * alpha;
                        }
                    }
                }
            }
            next_neg[e] += static_cast<float>(nneg) * en;
        }
    }
    return samples;
}

// ---------------------------------------------------------------- densMAP
// density_start_epoch (lib.rs:5052-5055).
size_t density_start_epoch(size_t n_epochs, float frac) {
    const size_t active =
        std::max<size_t>(static_cast<size_t>(std::ceil(static_cast<float>(n_epochs) * frac)), 1);
    return n_epochs > active ? n_epochs - active : 0;
}

// local_radii_from_knn (lib.rs:5057-5082): mean over non-self neighbours of
// ln(max(d, 0) + var_shift), FP32 sequential sum.
std::vector<float> local_radii(const Knn& knn, float var_shift) {
    const size_t n = knn.idx.size();
    std::vector<float> out(n);
    for (size_t r = 0; r < n; ++r) {
        float sum = 0.0f;
        size_t cnt = 0;
        for (size_t c = 0; c < knn.idx[r].size(); ++c) {
            const float dist = knn.dist[r][c];
            if (knn.idx[r][c] == r && std::fabs(dist) <= SMOOTH_K_TOLERANCE) continue;
            sum += logf(std::max(dist, 0.0f) + var_shift);
            ++cnt;
        }
        out[r] = cnt == 0 ? logf(var_shift) : sum / static_cast<float>(cnt);
    }
    return out;
}

inline float euclid(const float* x, const float* y, size_t dim) {
    return sqrtf(squared_distance(x, y, dim));
}

// embedding_radii_from_knn (lib.rs:5084-5108) on the flat embedding.
std::vector<float> embedding_radii(const std::vector<float>& flat, size_t dim, const Knn& knn,
                                   float var_shift) {
    const size_t n = knn.idx.size();
    std::vector<float> out(n);
    for (size_t r = 0; r < n; ++r) {
        float sum = 0.0f;
        size_t cnt = 0;
        for (size_t j : knn.idx[r]) {
            if (j == r) continue;
            sum += logf(std::max(euclid(&flat[r * dim], &flat[j * dim], dim), 0.0f) + var_shift);
            ++cnt;
        }
        out[r] = cnt == 0 ? logf(var_shift) : sum / static_cast<float>(cnt);
    }
    return out;
}

struct Density {
    std::vector<float> radii;
    size_t start_epoch;
    float lambda, var_shift;
};

// apply_density_gradient (lib.rs:5110-5134).
void density_step(std::vector<float>& flat, size_t dim, size_t head, size_t tail, float alpha,
                  const Density& dn) {
    if (head == tail) return;
    float* cur = &flat[head * dim];
    float* oth = &flat[tail * dim];
    const float dist = euclid(cur, oth, dim);
    const float target = std::max(expf((dn.radii[head] + dn.radii[tail]) * 0.5f), 1e-6f);
    const float coeff = 0.1f * dn.lambda * (dist - target) / (dist + dn.var_shift);
    for (size_t c = 0; c < dim; ++c) {
        const float dir = (cur[c] - oth[c]) / (dist + 1e-6f);
        const float g = clip4(coeff * dir);
        cur[c] -= g * alpha;
        oth[c] += g * alpha;
    }
}

// optimize_layout_training with a density term (lib.rs:5355-5440): the
// general-dimension loop, the attractive coefficient in its powf(d2, b - 1)
// form, then the density step for epochs >= start_epoch.
double optimize_layout_densmap(std::vector<float>& flat, size_t n_vertices, size_t dim,
                               const std::vector<Edge>& edges, size_t n_epochs, float a, float b,
                               float initial_alpha, size_t neg_rate, float repulsion,
                               uint64_t seed, const Density& dn) {
    if (edges.empty() || n_vertices == 0 || n_epochs == 0) return 0.0;
    std::vector<float> w(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) w[i] = edges[i].weight;
    const auto eps = epochs_per_sample(w, n_epochs);
    auto next = eps;
    std::vector<float> eps_neg(eps.size());
    for (size_t i = 0; i < eps.size(); ++i) eps_neg[i] = eps[i] / static_cast<float>(neg_rate);
    auto next_neg = eps_neg;
    SmallRng rng(seed);
    double samples = 0.0;
    for (size_t epoch = 0; epoch < n_epochs; ++epoch) {
        const float alpha =
            initial_alpha * (1.0f - static_cast<float>(epoch) / static_cast<float>(n_epochs));
        const float ef = static_cast<float>(epoch);
        for (size_t e = 0; e < edges.size(); ++e) {
            if (next[e] > ef) continue;
            samples += 1.0;
            const size_t head = edges[e].head, tail = edges[e].tail;
            if (head != tail) {
                const float d2 = squared_distance(&flat[head * dim], &flat[tail * dim], dim);
                float gc = 0.0f;
                if (d2 > 0.0f) {
                    const float pb = powf(d2, b);
                    gc = -2.0f * a * b * powf(d2, b - 1.0f) / (a * pb + 1.0f);
                }
                for (size_t c = 0; c < dim; ++c) {
                    const float hv = flat[head * dim + c], tv = flat[tail * dim + c];
                    const float g = clip4(gc * (hv - tv));
                    flat[head * dim + c] = hv + g * alpha;
                    flat[tail * dim + c] = tv - g * alpha;
                }
            }
            if (epoch >= dn.start_epoch) density_step(flat, dim, head, tail, alpha, dn);
            next[e] += eps[e];
            const float en = eps_neg[e];
            if (!std::isfinite(en) || en <= 0.0f) continue;
            const size_t nneg = floor_to_usize((ef - next_neg[e]) / en);
            for (size_t s = 0; s < nneg; ++s) {
                const size_t neg = rng.gen_range(0, n_vertices);
                if (neg == head) continue;
                const float d2 = squared_distance(&flat[head * dim], &flat[neg * dim], dim);
                float gc = 0.0f;
                if (d2 > 0.0f) {
                    const float pb = powf(d2, b);
                    gc = 2.0f * repulsion * b / ((0.001f + d2) * (a * pb + 1.0f));
                }
                if (gc > 0.0f)
                    for (size_t c = 0; c < dim; ++c) {
                        const float hv = flat[head * dim + c], nv = flat[neg * dim + c];
                        flat[head * dim + c] = hv + clip4(gc * (hv - nv)) * alpha;
                    }
            }
            next_neg[e] += static_cast<float>(nneg) * en;
        }
    }
    return samples;
}

// init_graph_transform (lib.rs:4793-4836).
Coords init_graph_transform(size_t nq, size_t dim, const std::vector<Edge>& edges,
                            const std::vector<float>& base) {
    std::vector<std::vector<std::pair<size_t, float>>> rows(nq);
    for (const auto& e : edges) rows[e.head].emplace_back(e.tail, e.weight);
    Coords out(nq, std::vector<float>(dim, 0.0f));
    for (size_t i = 0; i < nq; ++i) {
        if (rows[i].empty()) {
            std::fill(out[i].begin(), out[i].end(), std::numeric_limits<float>::quiet_NaN());
            continue;
        }
        bool copied = false;
        for (auto [c, w] : rows[i]) {
            if (std::fabs(w - 1.0f) < std::numeric_limits<float>::epsilon()) {
                for (size_t d = 0; d < dim; ++d) out[i][d] = base[c * dim + d];
                copied = true;
                break;
            }
        }
        if (copied) continue;
        float sum = 0.0f;
        for (auto [c, w] : rows[i]) sum += w;
        if (sum <= 0.0f) {
            std::fill(out[i].begin(), out[i].end(), std::numeric_limits<float>::quiet_NaN());
            continue;
        }
        for (auto [c, w] : rows[i]) {
            const float wn = w / sum;
            for (size_t d = 0; d < dim; ++d) out[i][d] += wn * base[c * dim + d];
        }
    }
    return out;
}

// query_head_seed (lib.rs:5028-5033).
uint64_t query_head_seed(uint64_t seed, uint64_t head) {
    uint64_t m = seed ^ (head * 0x9E3779B97F4A7C15ULL);
    m = (m ^ (m >> 30)) * 0xBF58476D1CE4E5B9ULL;
    m = (m ^ (m >> 27)) * 0x94D049BB133111EBULL;
    return m ^ (m >> 31);
}

// optimize_layout_transform (lib.rs:5444-5544): every query head is an
// independent problem with its own RNG stream.
void optimize_layout_transform(Coords& emb, const std::vector<float>& base, size_t n_base,
                               const std::vector<Edge>& edges, size_t n_epochs, float a, float b,
                               float initial_alpha, size_t neg_rate, float repulsion,
                               uint64_t seed) {
    if (edges.empty() || emb.empty() || n_epochs == 0) return;
    const size_t dim = emb[0].size();
    std::vector<float> w(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) w[i] = edges[i].weight;
    const auto eps = epochs_per_sample(w, n_epochs);
    std::vector<float> eps_neg(eps.size());
    for (size_t i = 0; i < eps.size(); ++i) eps_neg[i] = eps[i] / static_cast<float>(neg_rate);
    // grouped_edge_offsets (lib.rs:5009-5025)
    std::vector<size_t> off(emb.size() + 1, 0);
    {
        size_t ei = 0;
        for (size_t h = 0; h < emb.size(); ++h) {
            off[h] = ei;
            while (ei < edges.size() && edges[ei].head == h) ei++;
        }
        off[emb.size()] = ei;
        if (ei != edges.size()) return;
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t hh = 0; hh < static_cast<int64_t>(emb.size()); ++hh) {
        const size_t head = static_cast<size_t>(hh);
        auto& cur = emb[head];
        const size_t st = off[head], en = off[head + 1];
        std::vector<float> next(eps.begin() + st, eps.begin() + en);
        std::vector<float> next_neg(eps_neg.begin() + st, eps_neg.begin() + en);
        SmallRng rng(query_head_seed(seed, head));
        for (size_t epoch = 0; epoch < n_epochs; ++epoch) {
            const float alpha =
                initial_alpha * (1.0f - static_cast<float>(epoch) / static_cast<float>(n_epochs));
            const float ef = static_cast<float>(epoch);
            for (size_t li = 0, ei = st; ei < en; ++li, ++ei) {
                bool finite = true;
                for (float v : cur) finite &= std::isfinite(v);
                if (next[li] > ef || !finite) continue;
                const float* other = &base[edges[ei].tail * dim];
                float d2 = squared_distance(cur.data(), other, dim);
                float gc = 0.0f;
                if (d2 > 0.0f) {
                    const float pb = powf(d2, b);
                    gc = -2.0f * a * b * powf(d2, b - 1.0f) / (a * pb + 1.0f);
                }
                for (size_t d = 0; d < dim; ++d) {
                    const float g = clip4(gc * (cur[d] - other[d]));
                    cur[d] += g * alpha;
                }
                next[li] += eps[ei];
                const float en_ = eps_neg[ei];
                if (!std::isfinite(en_) || en_ <= 0.0f) continue;
                const size_t nneg = floor_to_usize((ef - next_neg[li]) / en_);
                for (size_t s = 0; s < nneg; ++s) {
                    const size_t neg = rng.gen_range(0, n_base);
                    const float* o2 = &base[neg * dim];
                    const float dd = squared_distance(cur.data(), o2, dim);
                    float g2 = 0.0f;
                    if (dd > 0.0f) {
                        const float pb = powf(dd, b);
                        g2 = 2.0f * repulsion * b / ((0.001f + dd) * (a * pb + 1.0f));
                    }
                    if (g2 > 0.0f)
                        for (size_t d = 0; d < dim; ++d) {
                            const float g = clip4(g2 * (cur[d] - o2[d]));
                            cur[d] += g * alpha;
                        }
                }
                next_neg[li] += static_cast<float>(nneg) * en_;
            }
        }
    }
}

std::vector<Edge> edges_from_arrays(const int32_t* h, const int32_t* t, const float* w,
                                    int64_t ne) {
    std::vector<Edge> e(static_cast<size_t>(ne));
    for (int64_t i = 0; i < ne; ++i)
        e[i] = {static_cast<size_t>(h[i]), static_cast<size_t>(t[i]), w[i]};
    return e;
}

Knn knn_from_arrays(const int64_t* idx, const float* dist, size_t n, size_t k) {
    Knn knn;
    knn.idx.resize(n);
    knn.dist.resize(n);
    for (size_t i = 0; i < n; ++i) {
        knn.idx[i].assign(idx + i * k, idx + (i + 1) * k);
        knn.dist[i].assign(dist + i * k, dist + (i + 1) * k);
    }
    return knn;
}

// ------------------------------------------------------------- sparse ---
// SparseCsrMatrix (rust_umap/src/sparse.rs:8-118): a CSR view with the
// squared norms (sum of v * v over the stored values, in stored order) and
// the L2 norms (their square roots) of every row.
struct CsrRows {
    int64_t n_rows = 0, n_cols = 0;
    const int64_t* indptr = nullptr;
    const int64_t* indices = nullptr;
    const float* data = nullptr;
    std::vector<float> sq, l2;
};

CsrRows csr_rows(const int64_t* indptr, const int64_t* indices, const float* data, int64_t n_rows,
                 int64_t n_cols) {
    CsrRows m;
    m.n_rows = n_rows;
    m.n_cols = n_cols;
    m.indptr = indptr;
    m.indices = indices;
    m.data = data;
    m.sq.assign(n_rows, 0.0f);
    m.l2.assign(n_rows, 0.0f);
    for (int64_t r = 0; r < n_rows; ++r) {
        float s = 0.0f;
        for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) s += data[e] * data[e];
        m.sq[r] = s;
        m.l2[r] = std::sqrt(s);
    }
    return m;
}

// sparse_dot (sparse.rs:220-239): products of the shared columns, summed in
// ascending column order.
float csr_dot(const CsrRows& a, int64_t ra, const CsrRows& b, int64_t rb) {
    int64_t i = a.indptr[ra], ie = a.indptr[ra + 1];
    int64_t j = b.indptr[rb], je = b.indptr[rb + 1];
    float dot = 0.0f;
    while (i < ie && j < je) {
        if (a.indices[i] < b.indices[j]) {
            ++i;
        } else if (a.indices[i] > b.indices[j]) {
            ++j;
        } else {
            dot += a.data[i] * b.data[j];
            ++i;
            ++j;
        }
    }
    return dot;
}

// euclidean_distance_from_dot (sparse.rs:241-244) and the cosine distance of
// sparse_slices_cosine_distance (sparse.rs:540-558).  A negative or zero
// radicand becomes +0.0.
float csr_distance(const CsrRows& a, int64_t ra, const CsrRows& b, int64_t rb, int metric) {
    if (metric == UMAPB_METRIC_COSINE) {
        const float la = a.l2[ra], lb = b.l2[rb];
        if (la == 0.0f && lb == 0.0f) return 0.0f;
        if (la == 0.0f || lb == 0.0f) return 1.0f;
        float c = csr_dot(a, ra, b, rb) / (la * lb);
        if (c < -1.0f) c = -1.0f;
        else if (c > 1.0f) c = 1.0f;
        return 1.0f - c;
    }
    float t = (a.sq[ra] + b.sq[rb]) - 2.0f * csr_dot(a, ra, b, rb);
    if (!(t > 0.0f)) t = 0.0f;
    return std::sqrt(t);
}

// exact_nearest_neighbors / exact_nearest_neighbors_sparse_query
// (sparse.rs:605-657): every query row against every reference row; in the
// self-join a row's distance to itself is 0.
Knn csr_knn(const CsrRows& q, const CsrRows& r, size_t k, int metric, bool self) {
    Knn out;
    out.idx.resize(q.n_rows);
    out.dist.resize(q.n_rows);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < q.n_rows; ++i) {
        auto& ri = out.idx[i];
        auto& rd = out.dist[i];
        ri.reserve(k + 1);
        rd.reserve(k + 1);
        for (int64_t j = 0; j < r.n_rows; ++j) {
            const float dist = (self && i == j) ? 0.0f : csr_distance(q, i, r, j, metric);
            push_top_k(ri, rd, static_cast<size_t>(j), dist, k);
        }
    }
    return out;
}

void knn_to_arrays(const Knn& knn, size_t k, int64_t* idx, float* dist) {
    for (size_t i = 0; i < knn.idx.size(); ++i)
        for (size_t c = 0; c < k; ++c) {
            idx[i * k + c] = static_cast<int64_t>(knn.idx[i][c]);
            dist[i * k + c] = knn.dist[i][c];
        }
}

}  // namespace

// ======================================================= C exports =====
extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_find_ab_params(float spread, float min_dist, float* a, float* b) {
    find_ab_params(spread, min_dist, a, b);
}

float orc_squared_distance(const float* x, const float* y, int64_t n) {
    return squared_distance(x, y, static_cast<size_t>(n));
}

float orc_cosine_distance(const float* x, const float* y, int64_t n) {
    return cosine_distance_with_norms(x, y, n, l2_norm(x, n), l2_norm(y, n));
}

// exact_nearest_neighbors (lib.rs:2911-2928): every row vs all rows.
void orc_exact_knn(const float* x, int64_t n, int64_t d, int64_t k, int32_t metric, int64_t* idx,
                   float* dist) {
    const Knn knn = exact_knn_query(x, n, x, n, d, k, metric);
    knn_to_arrays(knn, k, idx, dist);
}

// Exact kNN of a subset of rows of x against all rows of x (the same rows
// exact_nearest_neighbors returns for those row indices).
void orc_exact_knn_rows(const float* x, int64_t n, int64_t d, int64_t k, int32_t metric,
                        const int64_t* rows, int64_t n_rows, int64_t* idx, float* dist) {
    std::vector<float> q(static_cast<size_t>(n_rows * d));
    for (int64_t r = 0; r < n_rows; ++r)
        std::memcpy(&q[r * d], x + rows[r] * d, sizeof(float) * d);
    const Knn knn = exact_knn_query(q.data(), n_rows, x, n, d, k, metric);
    knn_to_arrays(knn, k, idx, dist);
}

// exact_nearest_neighbors_to_reference (lib.rs:3346-3399).
void orc_knn_query(const float* q, int64_t nq, const float* r, int64_t nr, int64_t d, int64_t k,
                   int32_t metric, int64_t* idx, float* dist) {
    const Knn knn = exact_knn_query(q, nq, r, nr, d, k, metric);
    knn_to_arrays(knn, k, idx, dist);
}

// exact_nearest_neighbors (sparse.rs:605-626) of a CSR matrix
// (indptr n_rows + 1, strictly increasing column indices per row).
void orc_csr_knn(const int64_t* indptr, const int64_t* indices, const float* data, int64_t n_rows,
                 int64_t n_cols, int64_t k, int32_t metric, int64_t* idx, float* dist) {
    const CsrRows m = csr_rows(indptr, indices, data, n_rows, n_cols);
    knn_to_arrays(csr_knn(m, m, static_cast<size_t>(k), metric, true), k, idx, dist);
}

// The rows `rows` of exact_nearest_neighbors (sparse.rs:605-626) of a CSR
// matrix: each listed row against every row, its own distance 0.
void orc_csr_knn_rows(const int64_t* indptr, const int64_t* indices, const float* data,
                      int64_t n_rows, int64_t n_cols, const int64_t* rows, int64_t n_sel,
                      int64_t k, int32_t metric, int64_t* idx, float* dist) {
    const CsrRows m = csr_rows(indptr, indices, data, n_rows, n_cols);
    Knn out;
    out.idx.resize(n_sel);
    out.dist.resize(n_sel);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t s = 0; s < n_sel; ++s) {
        const int64_t i = rows[s];
        for (int64_t j = 0; j < n_rows; ++j) {
            const float d = i == j ? 0.0f : csr_distance(m, i, m, j, metric);
            push_top_k(out.idx[s], out.dist[s], static_cast<size_t>(j), d, static_cast<size_t>(k));
        }
    }
    knn_to_arrays(out, static_cast<size_t>(k), idx, dist);
}

// exact_nearest_neighbors_sparse_query (sparse.rs:628-657): CSR queries
// against a CSR reference.
void orc_csr_knn_query(const int64_t* q_indptr, const int64_t* q_indices, const float* q_data,
                       int64_t nq, const int64_t* r_indptr, const int64_t* r_indices,
                       const float* r_data, int64_t nr, int64_t n_cols, int64_t k,
                       int32_t metric, int64_t* idx, float* dist) {
    const CsrRows q = csr_rows(q_indptr, q_indices, q_data, nq, n_cols);
    const CsrRows r = csr_rows(r_indptr, r_indices, r_data, nr, n_cols);
    knn_to_arrays(csr_knn(q, r, static_cast<size_t>(k), metric, false), k, idx, dist);
}

int64_t orc_nndescent(const float* x, int64_t n, int64_t d, int64_t k, int32_t metric,
                      int64_t cand, int64_t iters, uint64_t seed, int64_t* idx, float* dist) {
    size_t ran = 0;
    const Knn knn = nndescent(x, n, d, k, metric, cand, iters, seed, &ran);
    knn_to_arrays(knn, k, idx, dist);
    return static_cast<int64_t>(ran);
}

void orc_smooth_knn(const float* dists, int64_t n, int64_t kc, float k, float local_conn,
                    float bandwidth, int32_t include_self, float* sig, float* rho) {
    std::vector<std::vector<float>> rows(n);
    for (int64_t i = 0; i < n; ++i) rows[i].assign(dists + i * kc, dists + (i + 1) * kc);
    std::vector<float> s, r;
    smooth_knn_dist_t<float>(rows, k, local_conn, bandwidth, include_self != 0, s, r);
    std::memcpy(sig, s.data(), sizeof(float) * n);
    std::memcpy(rho, r.data(), sizeof(float) * n);
}

void orc_smooth_knn_f64(const float* dists, int64_t n, int64_t kc, double k, double local_conn,
                        double bandwidth, int32_t include_self, double* sig, double* rho) {
    std::vector<std::vector<float>> rows(n);
    for (int64_t i = 0; i < n; ++i) rows[i].assign(dists + i * kc, dists + (i + 1) * kc);
    std::vector<double> s, r;
    smooth_knn_dist_t<double>(rows, k, local_conn, bandwidth, include_self != 0, s, r);
    std::memcpy(sig, s.data(), sizeof(double) * n);
    std::memcpy(rho, r.data(), sizeof(double) * n);
}

// build_dense_fit_artifacts graph stages (lib.rs:1385-1431): self detection,
// smooth_knn_dist, membership, symmetrize and (n_epochs > 0) prune.
int64_t orc_fuzzy_graph(const int64_t* idx, const float* dist, int64_t n, int64_t k, float mix,
                        float local_conn, int64_t n_epochs, int32_t* heads, int32_t* tails,
                        float* weights, int64_t capacity, float* sig_out, float* rho_out) {
    const Knn knn = knn_from_arrays(idx, dist, n, k);
    std::vector<float> sig, rho;
    smooth_knn_dist_t<float>(knn.dist, static_cast<float>(k), local_conn, DEFAULT_BANDWIDTH,
                             knn_rows_include_self(knn), sig, rho);
    auto edges = symmetrize(membership(knn, sig, rho), mix);
    if (n_epochs > 0) prune_edges(edges, static_cast<size_t>(n_epochs));
    if (static_cast<int64_t>(edges.size()) > capacity) return -1;
    for (size_t e = 0; e < edges.size(); ++e) {
        heads[e] = static_cast<int32_t>(edges[e].head);
        tails[e] = static_cast<int32_t>(edges[e].tail);
        weights[e] = edges[e].weight;
    }
    if (sig_out) std::memcpy(sig_out, sig.data(), sizeof(float) * n);
    if (rho_out) std::memcpy(rho_out, rho.data(), sizeof(float) * n);
    return static_cast<int64_t>(edges.size());
}

// inverse_transform_rows (lib.rs:1800-1915) for a model given by its rows X
// (n x D), embedding E (n x L) and the fit's sigmas / rhos: exact kNN of the
// queries among E, weights 1 / (1 + a d^(2b)), init_inverse_points
// (lib.rs:4838-4935, with an LU of partial pivoting for the L x L system) and
// optimize_layout_inverse (lib.rs:5547-5645, one SmallRng over all edges in
// order).  n_epochs_param < 0 is None.
int32_t orc_inverse_transform(const float* X, int64_t n, int64_t D, const float* E, int64_t L,
                              const float* sig, const float* rho, const float* Z, int64_t nq,
                              int64_t n_neighbors, int64_t n_epochs_param, float a, float b,
                              float lr, int64_t neg_rate, float repulsion, uint64_t seed,
                              float* out) {
    if (nq == 0) return 0;
    const size_t k = static_cast<size_t>(std::max<int64_t>(1, std::min<int64_t>(n_neighbors, n)));
    const size_t n_epochs = n_epochs_param < 0 ? (nq <= 10000 ? 100 : 30)
                                               : static_cast<size_t>(std::max<int64_t>(n_epochs_param / 3, 1));
    const Knn knn = exact_knn_query(Z, nq, E, n, L, k, UMAPB_METRIC_EUCLIDEAN);
    std::vector<Edge> edges;
    std::vector<std::vector<float>> init_w(nq, std::vector<float>(k, 0.0f));
    std::vector<char> fixed(nq, 0);
    for (int64_t i = 0; i < nq; ++i) {
        float row_sum = 0.0f;
        for (size_t j = 0; j < k; ++j) {
            const float w = 1.0f / (1.0f + a * std::pow(knn.dist[i][j], 2.0f * b));
            if (w > 0.0f && std::isfinite(w)) {
                init_w[i][j] = w;
                row_sum += w;
                edges.push_back({static_cast<size_t>(i), knn.idx[i][j], w});
            }
        }
        if (row_sum > 0.0f)
            for (auto& w : init_w[i]) w /= row_sum;
        fixed[i] = knn.dist[i][0] <= 1e-6f;
    }
    std::vector<std::vector<float>> pts(nq, std::vector<float>(D, 0.0f));
    for (int64_t i = 0; i < nq; ++i) {
        auto& res = pts[i];
        if (fixed[i]) {
            std::copy(X + knn.idx[i][0] * D, X + knn.idx[i][0] * D + D, res.begin());
            continue;
        }
        std::vector<float> zbar(L, 0.0f), xbar(D, 0.0f);
        float wsum = 0.0f;
        for (size_t j = 0; j < k; ++j) {
            const float w = init_w[i][j];
            if (w <= 0.0f || !std::isfinite(w)) continue;
            wsum += w;
            const size_t id = knn.idx[i][j];
            for (int64_t c = 0; c < L; ++c) zbar[c] += w * E[id * L + c];
            for (int64_t d = 0; d < D; ++d) xbar[d] += w * X[id * D + d];
        }
        if (wsum <= 0.0f) {
            std::fill(res.begin(), res.end(), std::numeric_limits<float>::quiet_NaN());
            continue;
        }
        std::vector<float> g(L * L, 0.0f), rhs(L * D, 0.0f);
        size_t non_zero = 0;
        for (size_t j = 0; j < k; ++j) {
            const float w = init_w[i][j];
            if (w <= 0.0f || !std::isfinite(w)) continue;
            ++non_zero;
            const size_t id = knn.idx[i][j];
            for (int64_t aa = 0; aa < L; ++aa) {
                const float za = E[id * L + aa] - zbar[aa];
                for (int64_t bb = 0; bb < L; ++bb) g[aa * L + bb] += w * za * (E[id * L + bb] - zbar[bb]);
                for (int64_t d = 0; d < D; ++d) rhs[aa * D + d] += w * za * (X[id * D + d] - xbar[d]);
            }
        }
        for (int64_t c = 0; c < L; ++c) g[c * L + c] += 1e-3f;
        res = xbar;
        if (non_zero > static_cast<size_t>(L)) {
            // LU with partial pivoting; a zero pivot leaves x_bar
            std::vector<int64_t> perm(L);
            for (int64_t c = 0; c < L; ++c) perm[c] = c;
            bool ok = true;
            for (int64_t c = 0; c < L && ok; ++c) {
                int64_t piv = c;
                float best = std::fabs(g[c * L + c]);
                for (int64_t r = c + 1; r < L; ++r)
                    if (std::fabs(g[r * L + c]) > best) {
                        best = std::fabs(g[r * L + c]);
                        piv = r;
                    }
                if (best == 0.0f) {
                    ok = false;
                    break;
                }
                if (piv != c) {
                    for (int64_t cc = 0; cc < L; ++cc) std::swap(g[c * L + cc], g[piv * L + cc]);
                    std::swap(perm[c], perm[piv]);
                }
                for (int64_t r = c + 1; r < L; ++r) {
                    const float f = g[r * L + c] / g[c * L + c];
                    g[r * L + c] = f;
                    for (int64_t cc = c + 1; cc < L; ++cc) g[r * L + cc] -= f * g[c * L + cc];
                }
            }
            if (ok) {
                std::vector<float> pred(D);
                bool valid = true;
                std::vector<float> y(L), beta(L);
                for (int64_t d = 0; d < D && valid; ++d) {
                    for (int64_t r = 0; r < L; ++r) {
                        float v = rhs[perm[r] * D + d];
                        for (int64_t c = 0; c < r; ++c) v -= g[r * L + c] * y[c];
                        y[r] = v;
                    }
                    for (int64_t r = L - 1; r >= 0; --r) {
                        float v = y[r];
                        for (int64_t c = r + 1; c < L; ++c) v -= g[r * L + c] * beta[c];
                        beta[r] = v / g[r * L + r];
                    }
                    float v = xbar[d];
                    for (int64_t c = 0; c < L; ++c) v += (Z[i * L + c] - zbar[c]) * beta[c];
                    if (!std::isfinite(v)) valid = false;
                    pred[d] = v;
                }
                if (valid) res = pred;
            }
        }
    }
    // optimize_layout_inverse
    if (!edges.empty() && n_epochs > 0) {
        std::vector<float> w(edges.size());
        for (size_t e = 0; e < edges.size(); ++e) w[e] = edges[e].weight;
        const std::vector<float> eps = epochs_per_sample(w, n_epochs);
        std::vector<float> next = eps, eps_neg(eps.size()), next_neg;
        for (size_t e = 0; e < eps.size(); ++e) eps_neg[e] = eps[e] / static_cast<float>(neg_rate);
        next_neg = eps_neg;
        SmallRng rng(seed);
        const float alpha0 = lr / 4.0f;
        auto dist_denom = [&](const std::vector<float>& x, const float* y, float* dist) {
            float sq = 0.0f;
            for (int64_t d = 0; d < D; ++d) {
                const float df = x[d] - y[d];
                sq += df * df;
            }
            *dist = std::sqrt(sq);
            return 1e-6f + *dist;
        };
        for (size_t epoch = 0; epoch < n_epochs; ++epoch) {
            const float alpha = alpha0 * (1.0f - static_cast<float>(epoch) / static_cast<float>(n_epochs));
            for (size_t e = 0; e < edges.size(); ++e) {
                if (next[e] > static_cast<float>(epoch)) continue;
                const size_t head = edges[e].head, tail = edges[e].tail;
                auto& cur = pts[head];
                bool finite = true;
                for (float v : cur) finite = finite && std::isfinite(v);
                if (fixed[head] || !finite) continue;
                float dd;
                const float denom = dist_denom(cur, X + tail * D, &dd);
                const float gc = -(1.0f / (edges[e].weight * sig[tail] + 1e-6f));
                for (int64_t d = 0; d < D; ++d) {
                    const float gd = clip4(gc * ((cur[d] - X[tail * D + d]) / denom));
                    cur[d] += gd * alpha;
                }
                next[e] += eps[e];
                const float en = eps_neg[e];
                if (!std::isfinite(en) || en <= 0.0f) continue;
                const float f = std::floor((static_cast<float>(epoch) - next_neg[e]) / en);
                const size_t n_neg = f > 0.0f ? static_cast<size_t>(f) : 0;
                for (size_t s_ = 0; s_ < n_neg; ++s_) {
                    const size_t neg = rng.gen_range(0, static_cast<uint64_t>(n));
                    float dn;
                    const float den2 = dist_denom(cur, X + neg * D, &dn);
                    const float wh = std::exp(-std::max(dn - rho[neg], 1e-6f) / (sig[neg] + 1e-6f));
                    const float g2 = -repulsion * ((0.0f - wh) / ((1.0f - wh) * sig[neg] + 1e-6f));
                    for (int64_t d = 0; d < D; ++d) {
                        const float gd = clip4(g2 * ((cur[d] - X[neg * D + d]) / den2));
                        cur[d] += gd * alpha;
                    }
                }
                next_neg[e] += static_cast<float>(n_neg) * en;
            }
        }
    }
    for (int64_t i = 0; i < nq; ++i) std::copy(pts[i].begin(), pts[i].end(), out + i * D);
    return 0;
}

// The categorical target intersection (lib.rs:1426-1431) of an edge list,
// then prune_edges when n_epochs > 0.
int64_t orc_categorical_intersection(const int32_t* heads, const int32_t* tails,
                                     const float* weights, int64_t m, const int64_t* labels,
                                     int64_t n, float weight, int64_t n_epochs, int32_t* out_h,
                                     int32_t* out_t, float* out_w, int64_t capacity) {
    std::vector<Edge> edges(static_cast<size_t>(m));
    for (int64_t e = 0; e < m; ++e)
        edges[e] = {static_cast<size_t>(heads[e]), static_cast<size_t>(tails[e]), weights[e]};
    auto out = categorical_intersection(edges, labels, static_cast<size_t>(n), weight);
    if (n_epochs > 0) prune_edges(out, static_cast<size_t>(n_epochs));
    if (static_cast<int64_t>(out.size()) > capacity) return -1;
    for (size_t e = 0; e < out.size(); ++e) {
        out_h[e] = static_cast<int32_t>(out[e].head);
        out_t[e] = static_cast<int32_t>(out[e].tail);
        out_w[e] = out[e].weight;
    }
    return static_cast<int64_t>(out.size());
}

// spectral_init with the random-init fallback of initialize_embedding.
int32_t orc_spectral_init(const float* data, int64_t n, int64_t d, const int32_t* heads,
                          const int32_t* tails, const float* weights, int64_t ne, int64_t dim,
                          uint64_t seed, float* out, int64_t* n_components) {
    const auto edges = edges_from_arrays(heads, tails, weights, ne);
    int used = 0;
    size_t nc = 0;
    const Coords c = initialize_embedding(data, n, d, dim, edges, UMAPB_INIT_SPECTRAL, seed,
                                          &used, &nc);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j < dim; ++j) out[i * dim + j] = c[i][j];
    if (n_components) *n_components = static_cast<int64_t>(nc);
    return used;
}

void orc_random_init(int64_t n, int64_t dim, uint64_t seed, float low, float high, float* out) {
    const Coords c = random_init(n, dim, seed, low, high);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j < dim; ++j) out[i * dim + j] = c[i][j];
}

double orc_optimize_layout(float* emb, int64_t n, int64_t dim, const int32_t* heads,
                           const int32_t* tails, const float* weights, int64_t ne,
                           int64_t n_epochs, float a, float b, float lr, int64_t neg_rate,
                           float repulsion, uint64_t seed) {
    const auto edges = edges_from_arrays(heads, tails, weights, ne);
    std::vector<float> flat(emb, emb + n * dim);
    const double s = optimize_layout_training(flat, n, dim, edges, n_epochs, a, b, lr, neg_rate,
                                              repulsion, seed);
    std::memcpy(emb, flat.data(), sizeof(float) * n * dim);
    return s;
}

// Full dense fit_transform (UmapModel::fit_transform_dense, lib.rs:769-794,
// artifacts lib.rs:1367-1464).  Returns 0 on success, -1 for parameters the
// restatement does not cover.
int32_t orc_fit_transform_dens(const float* x, int64_t n, int64_t d, const umapb_params* p,
                               float* out, float* radii_orig, float* radii_emb);

int32_t orc_fit_transform(const float* x, int64_t n, int64_t d, const umapb_params* p,
                          float* out, double* edge_samples, int64_t* n_edges_out,
                          double* stage_sec) {
    if (p->densmap || p->output_dens) return -1;
    // stage_sec (nullable): kNN, graph (a/b, smooth_knn, union, prune), init, SGD
    auto clock = [] {
        return std::chrono::duration<double>(
                   std::chrono::steady_clock::now().time_since_epoch()).count();
    };
    double t0 = clock();
    const size_t k = static_cast<size_t>(p->n_neighbors);
    bool approx = false;  // should_use_approximate_knn (lib.rs:2285-2311)
    if (p->use_approximate_knn && n > p->approx_knn_threshold) {
        approx = true;
        if (p->approx_knn_threshold > 0 && n <= p->approx_knn_threshold * 4) approx = false;
    }
    Knn knn = approx ? nndescent(x, n, d, k, p->metric, p->approx_knn_candidates,
                                 p->approx_knn_iters, p->random_seed ^ 0xC0FEFEED1234ABCDULL,
                                 nullptr)
                     : exact_knn_query(x, n, x, n, d, k, p->metric);
    if (stage_sec) stage_sec[0] = clock() - t0;
    t0 = clock();
    const size_t n_epochs =
        p->n_epochs >= 0 ? static_cast<size_t>(p->n_epochs) : (n <= 10000 ? 500 : 200);
    float a, b;
    find_ab_params(p->spread, p->min_dist, &a, &b);
    std::vector<float> sig, rho;
    smooth_knn_dist_t<float>(knn.dist, static_cast<float>(k), p->local_connectivity,
                             DEFAULT_BANDWIDTH, knn_rows_include_self(knn), sig, rho);
    auto edges = symmetrize(membership(knn, sig, rho), p->set_op_mix_ratio);
    prune_edges(edges, n_epochs);
    if (n_edges_out) *n_edges_out = static_cast<int64_t>(edges.size());
    if (stage_sec) stage_sec[1] = clock() - t0;
    t0 = clock();
    const size_t dim = static_cast<size_t>(p->n_components);
    const Coords init =
        initialize_embedding(x, n, d, dim, edges, p->init, p->random_seed, nullptr, nullptr);
    if (stage_sec) stage_sec[2] = clock() - t0;
    t0 = clock();
    std::vector<float> flat(n * dim);
    for (int64_t i = 0; i < n; ++i)
        for (size_t j = 0; j < dim; ++j) flat[i * dim + j] = init[i][j];
    const double s = optimize_layout_training(
        flat, n, dim, edges, n_epochs, a, b, p->learning_rate,
        static_cast<size_t>(p->negative_sample_rate), p->repulsion_strength,
        p->random_seed ^ 0x9E3779B97F4A7C15ULL);
    if (edge_samples) *edge_samples = s;
    if (stage_sec) stage_sec[3] = clock() - t0;
    std::memcpy(out, flat.data(), sizeof(float) * n * dim);
    return 0;
}

// build_dense_fit_artifacts with densMAP / output_dens (lib.rs:1367-1464):
// the fit of orc_fit_transform plus the original radii (before the layout)
// and the embedding radii (after it); the density term joins the SGD when
// densmap is set and dens_lambda > 0.  radii_orig / radii_emb are n floats.
int32_t orc_fit_transform_dens(const float* x, int64_t n, int64_t d, const umapb_params* p,
                               float* out, float* radii_orig, float* radii_emb) {
    const size_t k = static_cast<size_t>(p->n_neighbors);
    bool approx = false;
    if (p->use_approximate_knn && n > p->approx_knn_threshold) {
        approx = true;
        if (p->approx_knn_threshold > 0 && n <= p->approx_knn_threshold * 4) approx = false;
    }
    Knn knn = approx ? nndescent(x, n, d, k, p->metric, p->approx_knn_candidates,
                                 p->approx_knn_iters, p->random_seed ^ 0xC0FEFEED1234ABCDULL,
                                 nullptr)
                     : exact_knn_query(x, n, x, n, d, k, p->metric);
    const size_t n_epochs =
        p->n_epochs >= 0 ? static_cast<size_t>(p->n_epochs) : (n <= 10000 ? 500 : 200);
    float a, b;
    find_ab_params(p->spread, p->min_dist, &a, &b);
    std::vector<float> sig, rho;
    smooth_knn_dist_t<float>(knn.dist, static_cast<float>(k), p->local_connectivity,
                             DEFAULT_BANDWIDTH, knn_rows_include_self(knn), sig, rho);
    const bool outputs = p->densmap || p->output_dens;
    std::vector<float> r_orig;
    if (outputs) r_orig = local_radii(knn, p->dens_var_shift);
    auto edges = symmetrize(membership(knn, sig, rho), p->set_op_mix_ratio);
    prune_edges(edges, n_epochs);
    const size_t dim = static_cast<size_t>(p->n_components);
    const Coords init =
        initialize_embedding(x, n, d, dim, edges, p->init, p->random_seed, nullptr, nullptr);
    std::vector<float> flat(n * dim);
    for (int64_t i = 0; i < n; ++i)
        for (size_t j = 0; j < dim; ++j) flat[i * dim + j] = init[i][j];
    const uint64_t sgd_seed = p->random_seed ^ 0x9E3779B97F4A7C15ULL;
    if (p->densmap && p->dens_lambda > 0.0f) {
        Density dn{r_orig, density_start_epoch(n_epochs, p->dens_frac), p->dens_lambda,
                   p->dens_var_shift};
        optimize_layout_densmap(flat, n, dim, edges, n_epochs, a, b, p->learning_rate,
                                static_cast<size_t>(p->negative_sample_rate),
                                p->repulsion_strength, sgd_seed, dn);
    } else {
        optimize_layout_training(flat, n, dim, edges, n_epochs, a, b, p->learning_rate,
                                 static_cast<size_t>(p->negative_sample_rate),
                                 p->repulsion_strength, sgd_seed);
    }
    std::memcpy(out, flat.data(), sizeof(float) * n * dim);
    if (outputs) {
        const auto r_emb = embedding_radii(flat, dim, knn, p->dens_var_shift);
        if (radii_orig) std::memcpy(radii_orig, r_orig.data(), sizeof(float) * n);
        if (radii_emb) std::memcpy(radii_emb, r_emb.data(), sizeof(float) * n);
    }
    return 0;
}

// local_radii_from_knn on a given kNN table (idx n x k int64, dist n x k).
void orc_local_radii(const int64_t* idx, const float* dist, int64_t n, int64_t k,
                     float var_shift, float* out) {
    Knn knn;
    knn.idx.resize(n);
    knn.dist.resize(n);
    for (int64_t r = 0; r < n; ++r) {
        knn.idx[r].assign(idx + r * k, idx + (r + 1) * k);
        knn.dist[r].assign(dist + r * k, dist + (r + 1) * k);
    }
    const auto v = local_radii(knn, var_shift);
    std::memcpy(out, v.data(), sizeof(float) * n);
}

// UmapModel::transform_rows + transform_from_knn (lib.rs:1604-1780) given
// the training matrix and its fitted embedding.
int32_t orc_transform(const float* train, int64_t n_train, const float* train_emb,
                      const float* q, int64_t nq, int64_t d, const umapb_params* p, float a,
                      float b, float* out) {
    if (nq == 0) return 0;
    const size_t k = std::min<size_t>(p->n_neighbors, n_train);
    const size_t n_epochs =
        p->n_epochs >= 0 ? std::max<size_t>(p->n_epochs, 1) : (nq <= 10000 ? 100 : 30);
    const Knn knn = exact_knn_query(q, nq, train, n_train, d, k, p->metric);
    const float lc = std::max(p->local_connectivity - 1.0f, 0.0f);
    std::vector<float> sig, rho;
    smooth_knn_dist_t<float>(knn.dist, static_cast<float>(k), lc, DEFAULT_BANDWIDTH, false, sig,
                             rho);
    auto edges = membership_bipartite(knn, sig, rho);
    prune_edges(edges, n_epochs);
    const size_t dim = static_cast<size_t>(p->n_components);
    std::vector<float> base(train_emb, train_emb + n_train * dim);
    Coords emb = init_graph_transform(nq, dim, edges, base);
    optimize_layout_transform(emb, base, n_train, edges, n_epochs, a, b, p->learning_rate / 4.0f,
                              static_cast<size_t>(p->negative_sample_rate), p->repulsion_strength,
                              p->random_seed ^ 0xA24BAED40B53C117ULL);
    for (int64_t i = 0; i < nq; ++i)
        for (size_t j = 0; j < dim; ++j) out[i * dim + j] = emb[i][j];
    return 0;
}

// The deterministic stages of transform_from_knn (lib.rs:1738-1763): query
// kNN, smooth_knn_dist with local_connectivity - 1, bipartite membership,
// prune_edges with the transform's epoch count and init_graph_transform.
// Returns the edge count, or -1 when `cap` is too small.
int64_t orc_transform_graph(const float* train, int64_t n_train, const float* train_emb,
                            const float* q, int64_t nq, int64_t d, const umapb_params* p,
                            float* sigmas, float* rhos, int32_t* heads, int32_t* tails,
                            float* weights, int64_t cap, float* init) {
    if (nq == 0) return 0;
    const size_t k = std::min<size_t>(p->n_neighbors, n_train);
    const size_t n_epochs =
        p->n_epochs >= 0 ? std::max<size_t>(p->n_epochs, 1) : (nq <= 10000 ? 100 : 30);
    const Knn knn = exact_knn_query(q, nq, train, n_train, d, k, p->metric);
    const float lc = std::max(p->local_connectivity - 1.0f, 0.0f);
    std::vector<float> sig, rho;
    smooth_knn_dist_t<float>(knn.dist, static_cast<float>(k), lc, DEFAULT_BANDWIDTH, false, sig,
                             rho);
    auto edges = membership_bipartite(knn, sig, rho);
    prune_edges(edges, n_epochs);
    if (static_cast<int64_t>(edges.size()) > cap) return -1;
    const size_t dim = static_cast<size_t>(p->n_components);
    std::vector<float> base(train_emb, train_emb + n_train * dim);
    Coords emb = init_graph_transform(nq, dim, edges, base);
    for (int64_t i = 0; i < nq; ++i) {
        sigmas[i] = sig[i];
        rhos[i] = rho[i];
        for (size_t j = 0; j < dim; ++j) init[i * dim + j] = emb[i][j];
    }
    for (size_t e = 0; e < edges.size(); ++e) {
        heads[e] = static_cast<int32_t>(edges[e].head);
        tails[e] = static_cast<int32_t>(edges[e].tail);
        weights[e] = edges[e].weight;
    }
    return static_cast<int64_t>(edges.size());
}

// optimize_layout_transform on explicit inputs (the thread-count determinism
// test of the reference, lib.rs:6193-6236, drives this function directly).
void orc_optimize_layout_transform(float* emb, int64_t nq, int64_t dim, const float* base,
                                   int64_t n_base, const int32_t* heads, const int32_t* tails,
                                   const float* weights, int64_t ne, int64_t n_epochs, float a,
                                   float b, float alpha, int64_t neg_rate, float repulsion,
                                   uint64_t seed) {
    const auto edges = edges_from_arrays(heads, tails, weights, ne);
    Coords e(nq, std::vector<float>(dim));
    for (int64_t i = 0; i < nq; ++i)
        for (int64_t j = 0; j < dim; ++j) e[i][j] = emb[i * dim + j];
    std::vector<float> bv(base, base + n_base * dim);
    optimize_layout_transform(e, bv, n_base, edges, n_epochs, a, b, alpha, neg_rate, repulsion,
                              seed);
    for (int64_t i = 0; i < nq; ++i)
        for (int64_t j = 0; j < dim; ++j) emb[i * dim + j] = e[i][j];
}

// normalized_laplacian_from_edges vs _from_affinity (pinned by the reference
// test at lib.rs:7457-7538): writes both n x n matrices.
int32_t orc_laplacians(int64_t n, const int32_t* heads, const int32_t* tails, const float* w,
                       int64_t ne, double* from_edges, double* from_affinity) {
    const auto edges = edges_from_arrays(heads, tails, w, ne);
    std::vector<double> aff(n * n, 0.0);
    for (const auto& e : edges) {
        if (e.head == e.tail) continue;
        const double v = static_cast<double>(std::max(e.weight, 0.0f));
        if (v > aff[e.head * n + e.tail]) aff[e.head * n + e.tail] = v;
    }
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = i + 1; j < n; ++j) {
            const double s = std::max(aff[i * n + j], aff[j * n + i]);
            aff[i * n + j] = s;
            aff[j * n + i] = s;
        }
    std::vector<double> L1, L2;
    if (!laplacian_from_edges(n, edges, L1)) return -1;
    if (!laplacian_from_affinity(aff, n, L2)) return -1;
    std::memcpy(from_edges, L1.data(), sizeof(double) * n * n);
    std::memcpy(from_affinity, L2.data(), sizeof(double) * n * n);
    return 0;
}

// SmallRng stream probe (first `count` next_u64 outputs) for RNG tests.
void orc_rng_u64(uint64_t seed, int64_t count, uint64_t* out) {
    SmallRng r(seed);
    for (int64_t i = 0; i < count; ++i) out[i] = r.next_u64();
}

}  // extern "C"
