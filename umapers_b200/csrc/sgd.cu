// sgd.cu - layout optimisation on the device.
//
// optimize_layout: the training SGD of rust_umap/src/lib.rs:5137-5321.  The
// reference walks the edges of one epoch sequentially with a single RNG
// stream; here one thread owns one edge per epoch (Hogwild): it keeps the
// reference's per-edge schedule (epoch_of_next_sample, epoch_of_next_negative
// sample, eps/neg_rate) exactly, moves its head point in registers through the
// attractive step and all of its negative samples, and publishes the head and
// tail moves with red.global.add, so concurrent edges never lose an update.
// Negative samples come from a counter-based stream keyed by (edge, epoch,
// sample) instead of the reference's shared SmallRng, so results do not depend
// on scheduling.  The embedding (n x dim FP32, 8 MB at 1M x 2) stays in L2.
//
// Small graphs (n_vertices x dim within kSmallLayoutFloats) run instead in
// one CTA that holds the embedding in shared memory for all epochs: the
// edges are coloured greedily in graph order so that no two edges of a colour
// share a vertex, and each epoch walks the colours in order, a colour's
// edges in parallel (Gauss-Seidel by colour).  Heads and tails are then
// updated without atomics, negatives read the epoch's starting positions,
// and the result is the same on every run.
//
// transform_layout: init_graph_transform (lib.rs:4793-4836) followed by
// optimize_layout_transform (lib.rs:5444-5544).  Queries never interact, so
// one thread runs one query's whole schedule sequentially, as the reference's
// per-query closure does.
#include <cub/cub.cuh>

#include <cfloat>
#include <cmath>

#include <vector>

#include "kernels.cuh"

namespace umapb {
namespace {

__device__ inline float clip4(float v) { return fminf(fmaxf(v, -4.0f), 4.0f); }  // lib.rs:4962

// floor(v).max(0.0) as usize, saturating (lib.rs:5204-5206)
__device__ inline uint32_t floor_count(float v) {
    const float f = floorf(v);
    if (!(f > 0.0f)) return 0u;
    if (f >= 4294967295.0f) return 0xffffffffu;
    return static_cast<uint32_t>(f);
}

// x^y for finite x > 0 through the base-2 logarithm, at a fraction of
// powf's instruction count.  The relative error is about |y log2 x| * 2^-23
// (log2f and exp2f are within 2 ulp): for the exponents used here (b and
// b - 1, |y| <= 2) under 5e-6 at squared distances in [1e-6, 1e6] and under
// 4e-5 anywhere in float range, far below the spread between Hogwild update
// orders.
__device__ __forceinline__ float pow_pos(float x, float y) {
    return exp2f(__fmul_rn(y, log2f(x)));
}

// x^y for finite x > 0 and y = b > 0 with CUDA's fast __powf intrinsic (the
// hardware base-2 logarithm and exponential), for the Hogwild epochs of large
// graphs, whose update order is not reproducible anyway.  Its relative error
// is about 2^-22 plus |y log2 x| * 2^-24: under 2e-6 at squared distances in
// [1e-6, 1e6].  Subnormal x gives 0 (x^b is then below 1e-28 for the b of
// any min_dist / spread in use).
__device__ __forceinline__ float pow_fast(float x, float y) { return __powf(x, y); }

// `row_max`/`heads` (nullable): the largest weight of each edge's head row
// replaces max_w (row-local transform graphs).
__global__ void epochs_per_sample_kernel(const float* __restrict__ w, int64_t m, float max_w,
                                         float n_epochs_f, float neg_rate_f,
                                         float* __restrict__ eps, float* __restrict__ next,
                                         float* __restrict__ next_neg,
                                         const float* __restrict__ row_max = nullptr,
                                         const int32_t* __restrict__ heads = nullptr) {
    // make_epochs_per_sample (lib.rs:4937-4960)
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    if (row_max != nullptr) max_w = fmaxf(row_max[heads[e]], 1e-12f);
    const float ns = __fmul_rn(n_epochs_f, __fdiv_rn(w[e], max_w));
    const float v = ns > 0.0f ? __fdiv_rn(n_epochs_f, ns) : INFINITY;
    eps[e] = v;
    if (next) next[e] = v;
    if (next_neg) next_neg[e] = __fdiv_rn(v, neg_rate_f);
}

// Sort keys of the edge order: the window of 2^shift consecutive edges
// (graph order, i.e. by head) in the high word, the sampling period in the
// low word.  Periods are positive floats or +inf, whose bit patterns order
// as unsigned integers.  Windows hold 65536 edges at most and are cut
// smaller on small graphs, so that a graph always spans at least 256 of them
// (down to 512 edges): the coarse head order survives the sort.
constexpr int kSortWindowMaxShift = 16;
constexpr int kSortWindowMinShift = 9;
constexpr int64_t kSortMinWindows = 256;

int sort_window_shift(int64_t m) {
    int shift = kSortWindowMinShift;
    while (shift < kSortWindowMaxShift && (static_cast<int64_t>(1) << (shift + 1)) * kSortMinWindows <= m)
        ++shift;
    return shift;
}

__global__ void period_keys_kernel(const float* __restrict__ eps, int64_t m, int shift,
                                   uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    keys[e] = (static_cast<uint64_t>(e >> shift) << 32) | __float_as_uint(eps[e]);
    ids[e] = static_cast<int32_t>(e);
}

// Position e of the sorted order takes edge order[e].
__global__ void gather_edges_kernel(const int32_t* __restrict__ order,
                                    const int32_t* __restrict__ heads,
                                    const int32_t* __restrict__ tails,
                                    const float* __restrict__ eps_in, float neg_rate_f, int64_t m,
                                    int32_t* __restrict__ heads_out,
                                    int32_t* __restrict__ tails_out, float* __restrict__ eps,
                                    float* __restrict__ next, float* __restrict__ next_neg) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int32_t o = order[e];
    heads_out[e] = heads[o];
    tails_out[e] = tails[o];
    const float v = eps_in[o];
    eps[e] = v;
    next[e] = v;
    next_neg[e] = __fdiv_rn(v, neg_rate_f);
}

struct SgdArgs {
    float* emb;
    const int32_t* heads;
    const int32_t* tails;
    const float* eps;
    float* next;
    float* next_neg;
    int64_t n_edges;
    uint32_t n_vertices;
    int dim;
    float epoch_f;
    float alpha;
    float a, b;
    float att_factor;  // -2ab
    float rep_factor;  // 2 * repulsion * b
    float neg_rate_f;
    uint64_t seed;
    uint64_t epoch;
    // densMAP (sgd_epoch_dens only)
    const float* radii;       // local_radii_from_knn of the input rows
    float dens_lambda, dens_var_shift;
    int dens_on;              // epoch >= density_start_epoch
};

// The attractive samples of all epochs, replayed from each edge's schedule:
// an edge fires in an epoch when its next-sample epoch is not above it, and
// its next-sample epoch then advances by its period, in the same FP32
// arithmetic as the epoch kernels.  The schedule does not depend on the
// layout, so the count is exact, and the epochs themselves count nothing.
__global__ void count_samples_kernel(const float* __restrict__ eps, int64_t m, int64_t n_epochs,
                                     unsigned long long* __restrict__ total) {
    unsigned long long c = 0;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < m;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float v = eps[e];
        float nxt = v;
        for (int64_t ep = 0; ep < n_epochs; ++ep) {
            if (!(nxt > static_cast<float>(ep))) {
                ++c;
                nxt = __fadd_rn(nxt, v);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(total, c);
}

// Negative samples drawn and loaded together in the 2-D epoch (even: two
// samples share one random word).
constexpr int kNegBatch = 4;
static_assert(kNegBatch % 2 == 0, "samples are drawn in pairs");

// One epoch for dim == 2 (the reference's flat fast path, lib.rs:5172-5244).
__global__ void __launch_bounds__(256) sgd_epoch_2d(SgdArgs p) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e < p.n_edges) {
        const float nxt = p.next[e];
        if (!(nxt > p.epoch_f)) {
            const int32_t head = p.heads[e];
            const int32_t tail = p.tails[e];
            float2* emb = reinterpret_cast<float2*>(p.emb);
            const float2 h0 = emb[head];
            float hx = h0.x, hy = h0.y;
            if (head != tail) {
                const float2 t = emb[tail];
                const float dx = __fsub_rn(hx, t.x), dy = __fsub_rn(hy, t.y);
                const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                if (d2 > 0.0f) {
                    const float pb = pow_fast(d2, p.b);
                    const float gc = __fdiv_rn(__fmul_rn(p.att_factor, __fdiv_rn(pb, d2)),
                                               __fadd_rn(__fmul_rn(p.a, pb), 1.0f));
                    const float gx = clip4(__fmul_rn(gc, dx)), gy = clip4(__fmul_rn(gc, dy));
                    const float mx = __fmul_rn(gx, p.alpha), my = __fmul_rn(gy, p.alpha);
                    hx = __fadd_rn(hx, mx);
                    hy = __fadd_rn(hy, my);
                    // one vector atomic moves both coordinates (each added atomically)
                    atomicAdd(reinterpret_cast<float2*>(p.emb) + tail, make_float2(-mx, -my));
                }
            }
            const float eps = p.eps[e];
            p.next[e] = __fadd_rn(nxt, eps);
            const float en = __fdiv_rn(eps, p.neg_rate_f);
            if (isfinite(en) && en > 0.0f) {
                const float nn = p.next_neg[e];
                const uint32_t n_neg = floor_count(__fdiv_rn(__fsub_rn(p.epoch_f, nn), en));
                // The negatives' positions do not depend on the head's moves:
                // kNegBatch are drawn and loaded at once, then applied in order.
                // Sample s takes the high (even s) or low (odd s) 32 bits of
                // the word keyed by (edge, epoch, s / 2).
                const uint64_t stream = mix64(p.seed ^ mix64(static_cast<uint64_t>(e)));
                for (uint32_t s0 = 0; s0 < n_neg; s0 += kNegBatch) {
                    float2 o[kNegBatch];
                    bool use[kNegBatch];
                    uint64_t wd[kNegBatch / 2];
#pragma unroll
                    for (int j = 0; j < kNegBatch / 2; ++j)
                        wd[j] = s0 + 2 * j < n_neg
                                    ? mix64(stream ^ ((p.epoch << 32) | ((s0 >> 1) + j)))
                                    : 0;
#pragma unroll
                    for (int j = 0; j < kNegBatch; ++j) {
                        const uint32_t s = s0 + j;
                        uint32_t neg = static_cast<uint32_t>(head);
                        if (s < n_neg) {
                            const uint64_t w = wd[j >> 1];
                            neg = rng_below32(static_cast<uint32_t>(j & 1 ? w : w >> 32),
                                              p.n_vertices);
                        }
                        use[j] = neg != static_cast<uint32_t>(head);
                        o[j] = use[j] ? emb[neg] : make_float2(0.0f, 0.0f);
                    }
#pragma unroll
                    for (int j = 0; j < kNegBatch; ++j) {
                        if (!use[j]) continue;
                        const float dx = __fsub_rn(hx, o[j].x), dy = __fsub_rn(hy, o[j].y);
                        const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                        if (d2 > 0.0f) {
                            const float pb = pow_fast(d2, p.b);
                            const float gc = __fdiv_rn(
                                p.rep_factor,
                                __fmul_rn(__fadd_rn(0.001f, d2), __fadd_rn(__fmul_rn(p.a, pb), 1.0f)));
                            if (gc > 0.0f) {
                                hx = __fadd_rn(hx, __fmul_rn(clip4(__fmul_rn(gc, dx)), p.alpha));
                                hy = __fadd_rn(hy, __fmul_rn(clip4(__fmul_rn(gc, dy)), p.alpha));
                            }
                        }
                    }
                }
                p.next_neg[e] = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), en));
            }
            if (hx != h0.x || hy != h0.y)
                atomicAdd(reinterpret_cast<float2*>(p.emb) + head,
                          make_float2(__fsub_rn(hx, h0.x), __fsub_rn(hy, h0.y)));
        }
    }
}

// One epoch for any dim (lib.rs:5248-5318).  The head moves in a per-thread
// copy of at most kMaxDim coordinates.
constexpr int kMaxDim = 16;

// One epoch of the densMAP layout (optimize_layout_training with a density
// state, lib.rs:5355-5440): the attractive coefficient in its
// -2ab d2^(b-1) / (a d2^b + 1) form, then, from density_start_epoch on,
// apply_density_gradient (lib.rs:5110-5134) on the same edge, then the
// negative samples.  Head in registers, tail moves published with atomics.
__global__ void __launch_bounds__(256) sgd_epoch_dens(SgdArgs p) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e < p.n_edges) {
        const float nxt = p.next[e];
        if (!(nxt > p.epoch_f)) {
            const int dim = p.dim;
            const int32_t head = p.heads[e];
            const int32_t tail = p.tails[e];
            float h0[kMaxDim], h[kMaxDim];
            for (int c = 0; c < dim; ++c) h0[c] = h[c] = p.emb[static_cast<int64_t>(head) * dim + c];
            if (head != tail) {
                float* t = p.emb + static_cast<int64_t>(tail) * dim;
                float d2 = 0.0f;
                for (int c = 0; c < dim; ++c) {
                    const float df = __fsub_rn(h[c], t[c]);
                    d2 = __fadd_rn(d2, __fmul_rn(df, df));
                }
                float gc = 0.0f;
                if (d2 > 0.0f) {
                    const float pb = powf(d2, p.b);
                    gc = __fdiv_rn(__fmul_rn(__fmul_rn(-2.0f * p.a, p.b), powf(d2, p.b - 1.0f)),
                                   __fadd_rn(__fmul_rn(p.a, pb), 1.0f));
                }
                for (int c = 0; c < dim; ++c) {
                    const float g = clip4(__fmul_rn(gc, __fsub_rn(h[c], t[c])));
                    const float mv = __fmul_rn(g, p.alpha);
                    h[c] = __fadd_rn(h[c], mv);
                    if (mv != 0.0f) atomicAdd(&t[c], -mv);
                }
                if (p.dens_on) {
                    float sq = 0.0f;
                    for (int c = 0; c < dim; ++c) {
                        const float df = __fsub_rn(h[c], t[c]);
                        sq = __fadd_rn(sq, __fmul_rn(df, df));
                    }
                    const float dist = __fsqrt_rn(sq);
                    const float target =
                        fmaxf(expf(__fmul_rn(__fadd_rn(p.radii[head], p.radii[tail]), 0.5f)), 1e-6f);
                    const float coeff =
                        __fdiv_rn(__fmul_rn(__fmul_rn(0.1f, p.dens_lambda), __fsub_rn(dist, target)),
                                  __fadd_rn(dist, p.dens_var_shift));
                    for (int c = 0; c < dim; ++c) {
                        const float dir =
                            __fdiv_rn(__fsub_rn(h[c], t[c]), __fadd_rn(dist, 1e-6f));
                        const float mv = __fmul_rn(clip4(__fmul_rn(coeff, dir)), p.alpha);
                        h[c] = __fsub_rn(h[c], mv);
                        if (mv != 0.0f) atomicAdd(&t[c], mv);
                    }
                }
            }
            const float eps = p.eps[e];
            p.next[e] = __fadd_rn(nxt, eps);
            const float en = __fdiv_rn(eps, p.neg_rate_f);
            if (isfinite(en) && en > 0.0f) {
                const float nn = p.next_neg[e];
                const uint32_t n_neg = floor_count(__fdiv_rn(__fsub_rn(p.epoch_f, nn), en));
                for (uint32_t s = 0; s < n_neg; ++s) {
                    const uint64_t word = rng_word(p.seed, static_cast<uint64_t>(e),
                                                   (p.epoch << 32) | s);
                    const uint32_t neg = rng_below(word, p.n_vertices);
                    if (neg == static_cast<uint32_t>(head)) continue;
                    const float* o = p.emb + static_cast<int64_t>(neg) * dim;
                    float d2 = 0.0f;
                    for (int c = 0; c < dim; ++c) {
                        const float df = __fsub_rn(h[c], o[c]);
                        d2 = __fadd_rn(d2, __fmul_rn(df, df));
                    }
                    if (d2 > 0.0f) {
                        const float pb = powf(d2, p.b);
                        const float gc =
                            __fdiv_rn(p.rep_factor, __fmul_rn(__fadd_rn(0.001f, d2),
                                                              __fadd_rn(__fmul_rn(p.a, pb), 1.0f)));
                        if (gc > 0.0f)
                            for (int c = 0; c < dim; ++c)
                                h[c] = __fadd_rn(
                                    h[c], __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(h[c], o[c]))),
                                                    p.alpha));
                    }
                }
                p.next_neg[e] = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), en));
            }
            for (int c = 0; c < dim; ++c)
                if (h[c] != h0[c])
                    atomicAdd(&p.emb[static_cast<int64_t>(head) * dim + c], __fsub_rn(h[c], h0[c]));
        }
    }
}

// local_radii_from_knn (lib.rs:5057-5082): one thread per row, FP32
// sequential sum of ln(max(d, 0) + var_shift) over non-self neighbours.
__global__ void local_radii_kernel(const int32_t* __restrict__ idx, const float* __restrict__ dist,
                                   int64_t n, int k, float var_shift, float* __restrict__ out) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float sum = 0.0f;
    int cnt = 0;
    for (int c = 0; c < k; ++c) {
        const float d = dist[r * k + c];
        if (idx[r * k + c] == r && fabsf(d) <= 1e-5f) continue;  // SMOOTH_K_TOLERANCE
        sum = __fadd_rn(sum, logf(__fadd_rn(fmaxf(d, 0.0f), var_shift)));
        ++cnt;
    }
    out[r] = cnt == 0 ? logf(var_shift) : __fdiv_rn(sum, static_cast<float>(cnt));
}

// embedding_radii_from_knn (lib.rs:5084-5108) on the fitted embedding.
__global__ void embedding_radii_kernel(const float* __restrict__ emb, int dim,
                                       const int32_t* __restrict__ idx, int64_t n, int k,
                                       float var_shift, float* __restrict__ out) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float sum = 0.0f;
    int cnt = 0;
    for (int c = 0; c < k; ++c) {
        const int64_t j = idx[r * k + c];
        if (j == r) continue;
        float sq = 0.0f;
        for (int t = 0; t < dim; ++t) {
            const float df = __fsub_rn(emb[r * dim + t], emb[j * dim + t]);
            sq = __fadd_rn(sq, __fmul_rn(df, df));
        }
        sum = __fadd_rn(sum, logf(__fadd_rn(fmaxf(__fsqrt_rn(sq), 0.0f), var_shift)));
        ++cnt;
    }
    out[r] = cnt == 0 ? logf(var_shift) : __fdiv_rn(sum, static_cast<float>(cnt));
}

__global__ void __launch_bounds__(256) sgd_epoch_nd(SgdArgs p) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e < p.n_edges) {
        const float nxt = p.next[e];
        if (!(nxt > p.epoch_f)) {
            const int dim = p.dim;
            const int32_t head = p.heads[e];
            const int32_t tail = p.tails[e];
            float h0[kMaxDim], h[kMaxDim];
            for (int c = 0; c < dim; ++c) h0[c] = h[c] = p.emb[static_cast<int64_t>(head) * dim + c];
            if (head != tail) {
                const float* t = p.emb + static_cast<int64_t>(tail) * dim;
                float d2 = 0.0f;
                for (int c = 0; c < dim; ++c) {
                    const float df = __fsub_rn(h[c], t[c]);
                    d2 = __fadd_rn(d2, __fmul_rn(df, df));
                }
                if (d2 > 0.0f) {
                    const float pb = powf(d2, p.b);
                    const float gc = __fdiv_rn(__fmul_rn(p.att_factor, __fdiv_rn(pb, d2)),
                                               __fadd_rn(__fmul_rn(p.a, pb), 1.0f));
                    for (int c = 0; c < dim; ++c) {
                        const float tv = t[c];
                        const float g = clip4(__fmul_rn(gc, __fsub_rn(h[c], tv)));
                        const float mv = __fmul_rn(g, p.alpha);
                        h[c] = __fadd_rn(h[c], mv);
                        atomicAdd(&p.emb[static_cast<int64_t>(tail) * dim + c], -mv);
                    }
                }
            }
            const float eps = p.eps[e];
            p.next[e] = __fadd_rn(nxt, eps);
            const float en = __fdiv_rn(eps, p.neg_rate_f);
            if (isfinite(en) && en > 0.0f) {
                const float nn = p.next_neg[e];
                const uint32_t n_neg = floor_count(__fdiv_rn(__fsub_rn(p.epoch_f, nn), en));
                for (uint32_t s = 0; s < n_neg; ++s) {
                    const uint64_t word = rng_word(p.seed, static_cast<uint64_t>(e),
                                                   (p.epoch << 32) | s);
                    const uint32_t neg = rng_below(word, p.n_vertices);
                    if (neg == static_cast<uint32_t>(head)) continue;
                    const float* o = p.emb + static_cast<int64_t>(neg) * dim;
                    float d2 = 0.0f;
                    for (int c = 0; c < dim; ++c) {
                        const float df = __fsub_rn(h[c], o[c]);
                        d2 = __fadd_rn(d2, __fmul_rn(df, df));
                    }
                    if (d2 > 0.0f) {
                        const float pb = powf(d2, p.b);
                        const float gc =
                            __fdiv_rn(p.rep_factor, __fmul_rn(__fadd_rn(0.001f, d2),
                                                              __fadd_rn(__fmul_rn(p.a, pb), 1.0f)));
                        if (gc > 0.0f)
                            for (int c = 0; c < dim; ++c)
                                h[c] = __fadd_rn(
                                    h[c], __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(h[c], o[c]))),
                                                    p.alpha));
                    }
                }
                p.next_neg[e] = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), en));
            }
            for (int c = 0; c < dim; ++c)
                if (h[c] != h0[c])
                    atomicAdd(&p.emb[static_cast<int64_t>(head) * dim + c], __fsub_rn(h[c], h0[c]));
        }
    }
}

// ------------------------------------------------------ small graphs ----
// Graphs with n_vertices * dim up to this many floats take the one-CTA
// coloured layout (two copies in shared memory: 128 KiB).
constexpr int64_t kSmallLayoutFloats = 16384;
constexpr int kSmallThreads = 1024;

struct SmallArgs {
    float* emb;               // n x dim, global (read at start, written at end)
    const int32_t* heads;     // edges ordered by (colour, graph order)
    const int32_t* tails;
    const float* eps;
    float* next;
    float* next_neg;
    const int32_t* color_ptr; // n_colors + 1 offsets
    int n_colors;
    uint32_t n_vertices;
    int dim;
    int64_t n_epochs;
    float lr, a, b, att_factor, rep_factor, neg_rate_f;
    const int64_t* edge_id;   // graph-order id of each edge (keys its negative stream)
    uint64_t seed;
    unsigned long long* samples;  // attractive samples over all epochs
};

// The reference's per-edge arithmetic (lib.rs:5172-5318) on shared-memory
// positions: `cur` is the live embedding, `snap` its state at the start of
// the epoch (read by the negative samples).
__global__ void __launch_bounds__(kSmallThreads, 1) sgd_small_kernel(SmallArgs p) {
    extern __shared__ float sm[];
    const int dim = p.dim;
    const int64_t nf = static_cast<int64_t>(p.n_vertices) * dim;
    float* cur = sm;
    float* snap = sm + nf;
    for (int64_t i = threadIdx.x; i < nf; i += blockDim.x) cur[i] = p.emb[i];
    unsigned long long sampled = 0;
    const float nef = static_cast<float>(p.n_epochs);
    for (int64_t epoch = 0; epoch < p.n_epochs; ++epoch) {
        __syncthreads();
        for (int64_t i = threadIdx.x; i < nf; i += blockDim.x) snap[i] = cur[i];
        __syncthreads();
        const float alpha = p.lr * (1.0f - static_cast<float>(epoch) / nef);
        const float ef = static_cast<float>(epoch);
        for (int c = 0; c < p.n_colors; ++c) {
            for (int32_t e = p.color_ptr[c] + threadIdx.x; e < p.color_ptr[c + 1];
                 e += blockDim.x) {
                const float nxt = p.next[e];
                if (nxt > ef) continue;
                ++sampled;
                const int32_t head = p.heads[e], tail = p.tails[e];
                float h[kMaxDim];
                for (int d = 0; d < dim; ++d) h[d] = cur[head * dim + d];
                if (head != tail) {
                    float d2 = 0.0f;
                    for (int d = 0; d < dim; ++d) {
                        const float df = __fsub_rn(h[d], cur[tail * dim + d]);
                        d2 = __fadd_rn(d2, __fmul_rn(df, df));
                    }
                    if (d2 > 0.0f) {
                        const float pb = pow_pos(d2, p.b);
                        const float gc = __fdiv_rn(__fmul_rn(p.att_factor, __fdiv_rn(pb, d2)),
                                                   __fadd_rn(__fmul_rn(p.a, pb), 1.0f));
                        for (int d = 0; d < dim; ++d) {
                            const float g = clip4(__fmul_rn(gc, __fsub_rn(h[d], cur[tail * dim + d])));
                            const float mv = __fmul_rn(g, alpha);
                            h[d] = __fadd_rn(h[d], mv);
                            cur[tail * dim + d] = __fsub_rn(cur[tail * dim + d], mv);
                        }
                    }
                }
                const float eps = p.eps[e];
                p.next[e] = __fadd_rn(nxt, eps);
                const float en = __fdiv_rn(eps, p.neg_rate_f);
                if (isfinite(en) && en > 0.0f) {
                    const float nn = p.next_neg[e];
                    const uint32_t n_neg = floor_count(__fdiv_rn(__fsub_rn(ef, nn), en));
                    const uint64_t eid = static_cast<uint64_t>(p.edge_id[e]);
                    for (uint32_t sn = 0; sn < n_neg; ++sn) {
                        const uint64_t word =
                            rng_word(p.seed, eid, (static_cast<uint64_t>(epoch) << 32) | sn);
                        const uint32_t neg = rng_below(word, p.n_vertices);
                        if (neg == static_cast<uint32_t>(head)) continue;
                        const float* o = snap + static_cast<int64_t>(neg) * dim;
                        float d2 = 0.0f;
                        for (int d = 0; d < dim; ++d) {
                            const float df = __fsub_rn(h[d], o[d]);
                            d2 = __fadd_rn(d2, __fmul_rn(df, df));
                        }
                        if (d2 > 0.0f) {
                            const float pb = pow_pos(d2, p.b);
                            const float gc = __fdiv_rn(
                                p.rep_factor,
                                __fmul_rn(__fadd_rn(0.001f, d2), __fadd_rn(__fmul_rn(p.a, pb), 1.0f)));
                            if (gc > 0.0f)
                                for (int d = 0; d < dim; ++d)
                                    h[d] = __fadd_rn(
                                        h[d], __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(h[d], o[d]))),
                                                        alpha));
                        }
                    }
                    p.next_neg[e] = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), en));
                }
                for (int d = 0; d < dim; ++d) cur[head * dim + d] = h[d];
            }
            __syncthreads();
        }
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < nf; i += blockDim.x) p.emb[i] = cur[i];
    if (p.samples && sampled) atomicAdd(p.samples, sampled);
}

// Greedy edge colouring in graph order: each edge takes the smallest colour
// not yet used at its head or its tail.  Returns the colour of every edge.
std::vector<int32_t> color_edges(const std::vector<int32_t>& heads,
                                 const std::vector<int32_t>& tails, int64_t n, int* n_colors) {
    const int64_t m = static_cast<int64_t>(heads.size());
    std::vector<std::vector<uint64_t>> used(n);
    std::vector<int32_t> color(m);
    int top = 0;
    auto is_used = [&](int64_t v, int c) {
        const auto& u = used[v];
        const size_t w = static_cast<size_t>(c) >> 6;
        return w < u.size() && ((u[w] >> (c & 63)) & 1u);
    };
    auto mark = [&](int64_t v, int c) {
        auto& u = used[v];
        const size_t w = static_cast<size_t>(c) >> 6;
        if (u.size() <= w) u.resize(w + 1, 0);
        u[w] |= uint64_t{1} << (c & 63);
    };
    for (int64_t e = 0; e < m; ++e) {
        const int64_t h = heads[e], t = tails[e];
        int c = 0;
        while (is_used(h, c) || is_used(t, c)) ++c;
        color[e] = c;
        mark(h, c);
        mark(t, c);
        top = std::max(top, c + 1);
    }
    *n_colors = top;
    return color;
}

// The one-CTA coloured layout of a small graph; returns the sample count.
double optimize_layout_small(float* emb, int64_t n_vertices, int dim, const Graph& g,
                             int64_t n_epochs, float a, float b, float lr, int64_t neg_rate,
                             float repulsion, uint64_t seed, float* kernel_ms, cudaStream_t s) {
    const int64_t m = g.n_edges;
    std::vector<int32_t> hh(m), th(m);
    UMAPB_CUDA(cudaMemcpyAsync(hh.data(), g.heads.get(), m * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(th.data(), g.tails.get(), m * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    int n_colors = 0;
    const std::vector<int32_t> color = color_edges(hh, th, n_vertices, &n_colors);
    std::vector<int32_t> ptr(n_colors + 1, 0);
    for (int32_t c : color) ++ptr[c + 1];
    for (int c = 0; c < n_colors; ++c) ptr[c + 1] += ptr[c];
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1), oh(m), ot(m);
    std::vector<int64_t> oid(m);
    for (int64_t e = 0; e < m; ++e) {
        const int32_t at = fill[color[e]]++;
        oh[at] = hh[e];
        ot[at] = th[e];
        oid[at] = e;
    }
    const float mx = std::max(max_weight(g.weights.get(), m, s), 1e-12f);
    const float nef = static_cast<float>(n_epochs);
    const float nrf = static_cast<float>(neg_rate);
    // edge periods in graph order (make_epochs_per_sample, lib.rs:4937-4960),
    // then permuted into colour order on the host
    DevBuf<float> eps_raw(m, s);
    epochs_per_sample_kernel<<<static_cast<unsigned>(ceil_div(m, 256)), 256, 0, s>>>(
        g.weights.get(), m, mx, nef, nrf, eps_raw.get(), nullptr, nullptr);
    UMAPB_LAUNCH_CHECK();
    std::vector<float> er(m), eo(m), no(m);
    UMAPB_CUDA(cudaMemcpyAsync(er.data(), eps_raw.get(), m * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    for (int64_t e = 0; e < m; ++e) {
        eo[e] = er[oid[e]];
        no[e] = eo[e] / nrf;  // the same FP32 division as gather_edges_kernel
    }
    DevBuf<int32_t> dh(m, s), dt(m, s), dptr(n_colors + 1, s);
    DevBuf<int64_t> did(m, s);
    DevBuf<float> deps(m, s), dnext(m, s), dneg(m, s);
    DevBuf<unsigned long long> samples(1, s);
    UMAPB_CUDA(cudaMemcpyAsync(dh.get(), oh.data(), m * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(dt.get(), ot.data(), m * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(did.get(), oid.data(), m * 8, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(dptr.get(), ptr.data(), (n_colors + 1) * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(deps.get(), eo.data(), m * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(dnext.get(), eo.data(), m * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(dneg.get(), no.data(), m * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemsetAsync(samples.get(), 0, 8, s));
    SmallArgs p{};
    p.emb = emb;
    p.heads = dh.get();
    p.tails = dt.get();
    p.eps = deps.get();
    p.next = dnext.get();
    p.next_neg = dneg.get();
    p.color_ptr = dptr.get();
    p.n_colors = n_colors;
    p.n_vertices = static_cast<uint32_t>(n_vertices);
    p.dim = dim;
    p.n_epochs = n_epochs;
    p.lr = lr;
    p.a = a;
    p.b = b;
    p.att_factor = -2.0f * a * b;
    p.rep_factor = 2.0f * repulsion * b;
    p.neg_rate_f = nrf;
    p.edge_id = did.get();
    p.seed = seed;
    p.samples = samples.get();
    const size_t smem = static_cast<size_t>(2 * n_vertices * dim) * sizeof(float);
    UMAPB_CUDA(cudaFuncSetAttribute(sgd_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernel_ms) {
        UMAPB_CUDA(cudaEventCreate(&e0));
        UMAPB_CUDA(cudaEventCreate(&e1));
        UMAPB_CUDA(cudaEventRecord(e0, s));
    }
    sgd_small_kernel<<<1, kSmallThreads, smem, s>>>(p);
    UMAPB_LAUNCH_CHECK();
    if (kernel_ms) {
        UMAPB_CUDA(cudaEventRecord(e1, s));
        UMAPB_CUDA(cudaEventSynchronize(e1));
        UMAPB_CUDA(cudaEventElapsedTime(kernel_ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    unsigned long long h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, samples.get(), 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return static_cast<double>(h);
}

// ------------------------------------------------------------ transform --
struct TransformArgs {
    float* out;
    const float* base;
    const int32_t* row_ptr;
    const int32_t* tails;
    const float* weights;
    const float* eps;
    float* next;
    float* next_neg;
    int64_t nq;
    uint32_t n_base;
    int dim;
    int64_t n_epochs;
    float a, b, lr, rep, neg_rate_f;
    uint64_t seed;
    const int32_t* qid;  // (nullable) row of each query in the whole request
    int64_t qid_offset;  // added to qid (or to the query index)
};

// The query's row in the whole request keys its random stream, so a query
// transformed alone, with a batch, or as a gated row of a surrogate request
// draws the same negatives.
__device__ __forceinline__ uint64_t query_seed(const TransformArgs& p, int64_t q) {
    const int64_t key = (p.qid != nullptr ? static_cast<int64_t>(p.qid[q]) : q) + p.qid_offset;
    return mix64(p.seed ^ mix64(static_cast<uint64_t>(key)));
}

__device__ inline bool row_finite(const float* v, int dim) {
    for (int c = 0; c < dim; ++c)
        if (!isfinite(v[c])) return false;
    return true;
}

// The 2-D schedule of one query, the same arithmetic in the same order as
// the general loop below.  Every position it reads is a fixed training
// point (the edge's tail and the negatives drawn for it), so an edge's
// positions are loaded together before the dependent updates: one memory
// latency per edge instead of one per sample.
constexpr int kNegPrefetch = 8;

__device__ __forceinline__ void transform_schedule_2d(const TransformArgs& p, int64_t q,
                                                      int32_t st, int32_t en, uint64_t qseed,
                                                      float* cur) {
    const float2* base = reinterpret_cast<const float2*>(p.base);
    const float att = __fmul_rn(__fmul_rn(-2.0f, p.a), p.b);
    const float rep = __fmul_rn(__fmul_rn(2.0f, p.rep), p.b);
    float cx = cur[0], cy = cur[1];
    for (int64_t epoch = 0; epoch < p.n_epochs && st < en; ++epoch) {
        const float alpha = __fmul_rn(
            p.lr, __fsub_rn(1.0f, __fdiv_rn(static_cast<float>(epoch),
                                            static_cast<float>(p.n_epochs))));
        const float ef = static_cast<float>(epoch);
        for (int32_t e = st; e < en; ++e) {
            const float nx = p.next[e];
            if (nx > ef || !(isfinite(cx) && isfinite(cy))) continue;
            const float eps = p.eps[e];
            const float eneg = __fdiv_rn(eps, p.neg_rate_f);
            const bool neg_ok = isfinite(eneg) && eneg > 0.0f;
            const float nn = p.next_neg[e];
            const uint32_t n_neg = neg_ok ? floor_count(__fdiv_rn(__fsub_rn(ef, nn), eneg)) : 0u;
            // loads first: the tail and the first kNegPrefetch negatives
            const float2 ot = base[p.tails[e]];
            float2 ng[kNegPrefetch];
#pragma unroll
            for (int s = 0; s < kNegPrefetch; ++s) {
                if (static_cast<uint32_t>(s) < n_neg) {
                    const uint64_t word = rng_word(qseed, static_cast<uint64_t>(e - st),
                                                   (static_cast<uint64_t>(epoch) << 32) | s);
                    ng[s] = base[rng_below(word, p.n_base)];
                }
            }
            {
                const float dx = __fsub_rn(cx, ot.x), dy = __fsub_rn(cy, ot.y);
                const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                float gc = 0.0f;
                if (d2 > 0.0f) {
                    const float pb = powf(d2, p.b);
                    gc = __fdiv_rn(__fmul_rn(att, powf(d2, p.b - 1.0f)),
                                   __fadd_rn(__fmul_rn(p.a, pb), 1.0f));
                }
                cx = __fadd_rn(cx, __fmul_rn(clip4(__fmul_rn(gc, dx)), alpha));
                cy = __fadd_rn(cy, __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(cy, ot.y))), alpha));
            }
            p.next[e] = __fadd_rn(nx, eps);
            if (!neg_ok) continue;
            for (uint32_t s = 0; s < n_neg; ++s) {
                float2 o;
                if (s < static_cast<uint32_t>(kNegPrefetch)) {
                    o = ng[0];
#pragma unroll
                    for (int t = 1; t < kNegPrefetch; ++t)
                        if (s == static_cast<uint32_t>(t)) o = ng[t];
                } else {
                    const uint64_t word = rng_word(qseed, static_cast<uint64_t>(e - st),
                                                   (static_cast<uint64_t>(epoch) << 32) | s);
                    o = base[rng_below(word, p.n_base)];
                }
                const float dx = __fsub_rn(cx, o.x), dy = __fsub_rn(cy, o.y);
                const float dd = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                float g2 = 0.0f;
                if (dd > 0.0f) {
                    const float pb = powf(dd, p.b);
                    g2 = __fdiv_rn(rep, __fmul_rn(__fadd_rn(0.001f, dd),
                                                  __fadd_rn(__fmul_rn(p.a, pb), 1.0f)));
                }
                if (g2 > 0.0f) {
                    cx = __fadd_rn(cx, __fmul_rn(clip4(__fmul_rn(g2, dx)), alpha));
                    cy = __fadd_rn(cy, __fmul_rn(clip4(__fmul_rn(g2, __fsub_rn(cy, o.y))), alpha));
                }
            }
            p.next_neg[e] = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), eneg));
        }
    }
    cur[0] = cx;
    cur[1] = cy;
}

// A 2-D query with at most kStageEdges edges keeps its whole edge state in
// shared memory: the tail positions (fixed training points) and the
// per-edge schedule (eps, epoch of next sample, epoch of next negative
// sample), loaded once before the first epoch.  The schedule loop then
// touches global memory only for the negative samples.  Slot [j][tid]
// belongs to thread tid alone, so no barrier is needed.
constexpr int kTransformThreads = 128;
constexpr int kStageEdges = 16;

struct TransformStage {
    float next[kStageEdges][kTransformThreads];
    float next_neg[kStageEdges][kTransformThreads];
    float eps[kStageEdges][kTransformThreads];
    float2 tail[kStageEdges][kTransformThreads];
};

// init_graph_transform (lib.rs:4793-4836) for a staged 2-D query, the same
// arithmetic in the same order as the general path in transform_kernel.
__device__ __forceinline__ void stage_query_2d(const TransformArgs& p, int32_t st, int cnt,
                                               TransformStage& sm, int tid, float* cur) {
    const float2* base = reinterpret_cast<const float2*>(p.base);
    int32_t tl[kStageEdges];
    float w[kStageEdges];
#pragma unroll
    for (int j = 0; j < kStageEdges; ++j) {
        if (j < cnt) {
            tl[j] = p.tails[st + j];
            w[j] = p.weights[st + j];
            sm.eps[j][tid] = p.eps[st + j];
            sm.next[j][tid] = p.next[st + j];
            sm.next_neg[j][tid] = p.next_neg[st + j];
        }
    }
#pragma unroll
    for (int j = 0; j < kStageEdges; ++j)
        if (j < cnt) sm.tail[j][tid] = base[tl[j]];
    if (cnt == 0) {
        cur[0] = cur[1] = NAN;
        return;
    }
    int copy_j = -1;
#pragma unroll
    for (int j = 0; j < kStageEdges; ++j)
        if (j < cnt && copy_j < 0 && fabsf(__fsub_rn(w[j], 1.0f)) < FLT_EPSILON) copy_j = j;
    if (copy_j >= 0) {
        const float2 t = sm.tail[copy_j][tid];
        cur[0] = t.x;
        cur[1] = t.y;
        return;
    }
    float sum = 0.0f;
#pragma unroll
    for (int j = 0; j < kStageEdges; ++j)
        if (j < cnt) sum = __fadd_rn(sum, w[j]);
    if (sum <= 0.0f) {
        cur[0] = cur[1] = NAN;
        return;
    }
    cur[0] = cur[1] = 0.0f;
#pragma unroll
    for (int j = 0; j < kStageEdges; ++j) {
        if (j < cnt) {
            const float wj = __fdiv_rn(w[j], sum);
            const float2 t = sm.tail[j][tid];
            cur[0] = __fadd_rn(cur[0], __fmul_rn(wj, t.x));
            cur[1] = __fadd_rn(cur[1], __fmul_rn(wj, t.y));
        }
    }
}

// transform_schedule_2d over the staged edge state; edge j of the query is
// graph edge st + j, which keys its negative-sample stream.  Each epoch
// first collects the query's due edges in a bit mask, then serves them in
// edge order: the lanes of a warp step through their own due edges together,
// so a warp runs as many edge updates as its busiest query has due, not as
// many as all 32 queries have together.
__device__ __forceinline__ void transform_schedule_2d_staged(const TransformArgs& p, int32_t st,
                                                             int cnt, uint64_t qseed,
                                                             TransformStage& sm, int tid,
                                                             float* cur) {
    const float2* base = reinterpret_cast<const float2*>(p.base);
    const float att = __fmul_rn(__fmul_rn(-2.0f, p.a), p.b);
    const float rep = __fmul_rn(__fmul_rn(2.0f, p.rep), p.b);
    float cx = cur[0], cy = cur[1];
    if (!(isfinite(cx) && isfinite(cy))) return;  // every sample would be skipped
    for (int64_t epoch = 0; epoch < p.n_epochs; ++epoch) {
        const float alpha = __fmul_rn(
            p.lr, __fsub_rn(1.0f, __fdiv_rn(static_cast<float>(epoch),
                                            static_cast<float>(p.n_epochs))));
        const float ef = static_cast<float>(epoch);
        uint32_t due = 0;
#pragma unroll
        for (int j = 0; j < kStageEdges; ++j)
            if (j < cnt && !(sm.next[j][tid] > ef)) due |= 1u << j;
        while (due) {
            const int j = __ffs(due) - 1;
            due &= due - 1;
            if (!(isfinite(cx) && isfinite(cy))) continue;
            const float nx = sm.next[j][tid];
            const int64_t e = st + j;
            const float eps = sm.eps[j][tid];
            const float eneg = __fdiv_rn(eps, p.neg_rate_f);
            const bool neg_ok = isfinite(eneg) && eneg > 0.0f;
            const float nn = sm.next_neg[j][tid];
            const uint32_t n_neg = neg_ok ? floor_count(__fdiv_rn(__fsub_rn(ef, nn), eneg)) : 0u;
            float2 ng[kNegPrefetch];
#pragma unroll
            for (int s = 0; s < kNegPrefetch; ++s) {
                if (static_cast<uint32_t>(s) < n_neg) {
                    const uint64_t word = rng_word(qseed, static_cast<uint64_t>(e - st),
                                                   (static_cast<uint64_t>(epoch) << 32) | s);
                    ng[s] = base[rng_below(word, p.n_base)];
                }
            }
            const float2 ot = sm.tail[j][tid];
            {
                const float dx = __fsub_rn(cx, ot.x), dy = __fsub_rn(cy, ot.y);
                const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                float gc = 0.0f;
                if (d2 > 0.0f) {
                    const float l2 = log2f(d2);
                    const float pb = exp2f(__fmul_rn(p.b, l2));
                    gc = __fdiv_rn(__fmul_rn(att, exp2f(__fmul_rn(p.b - 1.0f, l2))),
                                   __fadd_rn(__fmul_rn(p.a, pb), 1.0f));
                }
                cx = __fadd_rn(cx, __fmul_rn(clip4(__fmul_rn(gc, dx)), alpha));
                cy = __fadd_rn(cy, __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(cy, ot.y))), alpha));
            }
            sm.next[j][tid] = __fadd_rn(nx, eps);
            if (!neg_ok) continue;
            for (uint32_t s = 0; s < n_neg; ++s) {
                float2 o;
                if (s < static_cast<uint32_t>(kNegPrefetch)) {
                    o = ng[0];
#pragma unroll
                    for (int t = 1; t < kNegPrefetch; ++t)
                        if (s == static_cast<uint32_t>(t)) o = ng[t];
                } else {
                    const uint64_t word = rng_word(qseed, static_cast<uint64_t>(e - st),
                                                   (static_cast<uint64_t>(epoch) << 32) | s);
                    o = base[rng_below(word, p.n_base)];
                }
                const float dx = __fsub_rn(cx, o.x), dy = __fsub_rn(cy, o.y);
                const float dd = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                float g2 = 0.0f;
                if (dd > 0.0f) {
                    const float pb = pow_pos(dd, p.b);
                    g2 = __fdiv_rn(rep, __fmul_rn(__fadd_rn(0.001f, dd),
                                                  __fadd_rn(__fmul_rn(p.a, pb), 1.0f)));
                }
                if (g2 > 0.0f) {
                    cx = __fadd_rn(cx, __fmul_rn(clip4(__fmul_rn(g2, dx)), alpha));
                    cy = __fadd_rn(cy, __fmul_rn(clip4(__fmul_rn(g2, __fsub_rn(cy, o.y))), alpha));
                }
            }
            sm.next_neg[j][tid] = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), eneg));
        }
    }
    cur[0] = cx;
    cur[1] = cy;
}

__global__ void __launch_bounds__(kTransformThreads) transform_kernel(TransformArgs p) {
    __shared__ TransformStage sm;
    const int tid = threadIdx.x;
    const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid;
    if (q >= p.nq) return;
    const int dim = p.dim;
    const int32_t st = p.row_ptr[q], en = p.row_ptr[q + 1];
    if (dim == 2 && en - st <= kStageEdges) {
        float c2[2];
        stage_query_2d(p, st, en - st, sm, tid, c2);
        const uint64_t qseed = query_seed(p, q);
        transform_schedule_2d_staged(p, st, en - st, qseed, sm, tid, c2);
        p.out[q * 2] = c2[0];
        p.out[q * 2 + 1] = c2[1];
        return;
    }
    float cur[kMaxDim];
    // init_graph_transform (lib.rs:4793-4836)
    if (st == en) {
        for (int c = 0; c < dim; ++c) cur[c] = NAN;
    } else {
        int32_t copy_from = -1;
        for (int32_t e = st; e < en; ++e)
            if (fabsf(__fsub_rn(p.weights[e], 1.0f)) < FLT_EPSILON) {
                copy_from = p.tails[e];
                break;
            }
        if (copy_from >= 0) {
            for (int c = 0; c < dim; ++c) cur[c] = p.base[static_cast<int64_t>(copy_from) * dim + c];
        } else {
            float sum = 0.0f;
            for (int32_t e = st; e < en; ++e) sum = __fadd_rn(sum, p.weights[e]);
            if (sum <= 0.0f) {
                for (int c = 0; c < dim; ++c) cur[c] = NAN;
            } else {
                for (int c = 0; c < dim; ++c) cur[c] = 0.0f;
                for (int32_t e = st; e < en; ++e) {
                    const float w = __fdiv_rn(p.weights[e], sum);
                    const float* bt = p.base + static_cast<int64_t>(p.tails[e]) * dim;
                    for (int c = 0; c < dim; ++c) cur[c] = __fadd_rn(cur[c], __fmul_rn(w, bt[c]));
                }
            }
        }
    }
    // optimize_layout_transform (lib.rs:5444-5544)
    const uint64_t qseed = query_seed(p, q);
    if (dim == 2) {
        transform_schedule_2d(p, q, st, en, qseed, cur);
        p.out[q * 2] = cur[0];
        p.out[q * 2 + 1] = cur[1];
        return;
    }
    for (int64_t epoch = 0; epoch < p.n_epochs && st < en; ++epoch) {
        const float alpha = __fmul_rn(
            p.lr, __fsub_rn(1.0f, __fdiv_rn(static_cast<float>(epoch),
                                            static_cast<float>(p.n_epochs))));
        const float ef = static_cast<float>(epoch);
        for (int32_t e = st; e < en; ++e) {
            if (p.next[e] > ef || !row_finite(cur, dim)) continue;
            const float* other = p.base + static_cast<int64_t>(p.tails[e]) * dim;
            float d2 = 0.0f;
            for (int c = 0; c < dim; ++c) {
                const float df = __fsub_rn(cur[c], other[c]);
                d2 = __fadd_rn(d2, __fmul_rn(df, df));
            }
            float gc = 0.0f;
            if (d2 > 0.0f) {
                const float pb = powf(d2, p.b);
                gc = __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(-2.0f, p.a), p.b), powf(d2, p.b - 1.0f)),
                               __fadd_rn(__fmul_rn(p.a, pb), 1.0f));
            }
            for (int c = 0; c < dim; ++c)
                cur[c] = __fadd_rn(cur[c], __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(cur[c], other[c]))),
                                                     alpha));
            p.next[e] = __fadd_rn(p.next[e], p.eps[e]);
            const float eneg = __fdiv_rn(p.eps[e], p.neg_rate_f);
            if (!isfinite(eneg) || eneg <= 0.0f) continue;
            const float nn = p.next_neg[e];
            const uint32_t n_neg = floor_count(__fdiv_rn(__fsub_rn(ef, nn), eneg));
            for (uint32_t s = 0; s < n_neg; ++s) {
                const uint64_t word = rng_word(qseed, static_cast<uint64_t>(e - st),
                                               (static_cast<uint64_t>(epoch) << 32) | s);
                const uint32_t neg = rng_below(word, p.n_base);
                const float* o = p.base + static_cast<int64_t>(neg) * dim;
                float dd = 0.0f;
                for (int c = 0; c < dim; ++c) {
                    const float df = __fsub_rn(cur[c], o[c]);
                    dd = __fadd_rn(dd, __fmul_rn(df, df));
                }
                float g2 = 0.0f;
                if (dd > 0.0f) {
                    const float pb = powf(dd, p.b);
                    g2 = __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, p.rep), p.b),
                                   __fmul_rn(__fadd_rn(0.001f, dd), __fadd_rn(__fmul_rn(p.a, pb), 1.0f)));
                }
                if (g2 > 0.0f)
                    for (int c = 0; c < dim; ++c)
                        cur[c] = __fadd_rn(
                            cur[c], __fmul_rn(clip4(__fmul_rn(g2, __fsub_rn(cur[c], o[c]))), alpha));
            }
            p.next_neg[e] = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), eneg));
        }
    }
    for (int c = 0; c < dim; ++c) p.out[q * dim + c] = cur[c];
}

// ------------------------------------------------------ inverse transform --
// inverse_transform_rows (rust_umap/src/lib.rs:1800-1915): every embedded
// query q gets k neighbours among the fitted embedding's rows, edge weights
// 1 / (1 + a d^(2b)), an initial point in data space (init_inverse_points,
// lib.rs:4838-4935), then per-query SGD against the fitted rows
// (optimize_layout_inverse, lib.rs:5547-5645).  One warp per query; lanes
// split the data dimensions.
constexpr int kInvMaxLow = 16;  // n_components
constexpr int kInvMaxK = 32;    // neighbours per query

struct InverseArgs {
    const float* zq;      // nq x L embedded queries
    const int32_t* idx;   // nq x k neighbours in the fitted embedding
    const float* dist;    // nq x k
    const float* emb;     // n x L fitted embedding
    const float* X;       // n x D fitted rows
    const float* sig;     // n: the fit's sigmas
    const float* rho;     // n: the fit's rhos
    float* out;           // nq x D
    float* w;             // nq x k edge weights, 0 where the reference adds no edge
    uint8_t* fixed;       // nq: first neighbour within 1e-6
    int64_t nq, n;
    int L, D, k;
    float a, b;
    // optimize_layout_inverse
    float max_w;          // largest edge weight of the whole inverse graph
    int64_t n_epochs;
    float alpha0, neg_rate_f, rep;
    uint64_t seed;
};

// Partial-pivoting LU of the L x L matrix g (row-major, in place) with the
// row permutation in perm; false when a pivot is 0 (nalgebra's solve then
// returns None).
__device__ bool lu_factor(float* g, int L, int* perm) {
    for (int i = 0; i < L; ++i) perm[i] = i;
    for (int i = 0; i < L; ++i) {
        int piv = i;
        float best = fabsf(g[i * L + i]);
        for (int r = i + 1; r < L; ++r)
            if (fabsf(g[r * L + i]) > best) {
                best = fabsf(g[r * L + i]);
                piv = r;
            }
        if (best == 0.0f) return false;
        if (piv != i) {
            for (int c = 0; c < L; ++c) {
                const float t = g[i * L + c];
                g[i * L + c] = g[piv * L + c];
                g[piv * L + c] = t;
            }
            const int t = perm[i];
            perm[i] = perm[piv];
            perm[piv] = t;
        }
        const float inv = g[i * L + i];
        for (int r = i + 1; r < L; ++r) {
            const float f = __fdiv_rn(g[r * L + i], inv);
            g[r * L + i] = f;
            for (int c = i + 1; c < L; ++c)
                g[r * L + c] = __fsub_rn(g[r * L + c], __fmul_rn(f, g[i * L + c]));
        }
    }
    return true;
}

// Solves LU x = P rhs for one right-hand side (x overwrites rhs).
__device__ void lu_solve(const float* g, int L, const int* perm, float* rhs) {
    float y[kInvMaxLow];
    for (int i = 0; i < L; ++i) {
        float v = rhs[perm[i]];
        for (int c = 0; c < i; ++c) v = __fsub_rn(v, __fmul_rn(g[i * L + c], y[c]));
        y[i] = v;
    }
    for (int i = L - 1; i >= 0; --i) {
        float v = y[i];
        for (int c = i + 1; c < L; ++c) v = __fsub_rn(v, __fmul_rn(g[i * L + c], rhs[c]));
        rhs[i] = __fdiv_rn(v, g[i * L + i]);
    }
}

__global__ void __launch_bounds__(256) inverse_init_kernel(InverseArgs p) {
    const int64_t q = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= p.nq) return;
    const int L = p.L, D = p.D, k = p.k;
    const int32_t* nb = p.idx + q * k;
    float* out = p.out + q * D;
    // edge weights in neighbour order (lib.rs:1871-1893)
    float wj = 0.0f;
    if (lane < k) {
        const float d = p.dist[q * k + lane];
        const float v = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(p.a, powf(d, __fmul_rn(2.0f, p.b)))));
        wj = (v > 0.0f && isfinite(v)) ? v : 0.0f;
        p.w[q * k + lane] = wj;
    }
    float row_sum = 0.0f;
    for (int j = 0; j < k; ++j) row_sum = __fadd_rn(row_sum, __shfl_sync(0xffffffffu, wj, j));
    const float nw = row_sum > 0.0f ? __fdiv_rn(wj, row_sum) : wj;  // normalised init weight
    const bool fixed = p.dist[q * k] <= 1e-6f;
    if (lane == 0) p.fixed[q] = fixed ? 1 : 0;
    if (fixed) {
        const float* src = p.X + static_cast<int64_t>(nb[0]) * D;
        for (int d = lane; d < D; d += 32) out[d] = src[d];
        return;
    }
    // weighted means of the neighbours' embedding and data rows (lib.rs:4859-4875)
    float zbar[kInvMaxLow];
    for (int c = 0; c < L; ++c) zbar[c] = 0.0f;
    float wsum = 0.0f;
    int non_zero = 0;
    for (int j = 0; j < k; ++j) {
        const float w = __shfl_sync(0xffffffffu, nw, j);
        if (!(w > 0.0f) || !isfinite(w)) continue;
        wsum = __fadd_rn(wsum, w);
        ++non_zero;
        const float* e = p.emb + static_cast<int64_t>(nb[j]) * L;
        for (int c = 0; c < L; ++c) zbar[c] = __fadd_rn(zbar[c], __fmul_rn(w, e[c]));
    }
    if (wsum <= 0.0f) {
        for (int d = lane; d < D; d += 32) out[d] = NAN;
        return;
    }
    // gram = sum w z_a z_b, plus 1e-3 on the diagonal (lib.rs:4881-4902)
    float g[kInvMaxLow * kInvMaxLow];
    for (int c = 0; c < L * L; ++c) g[c] = 0.0f;
    for (int j = 0; j < k; ++j) {
        const float w = __shfl_sync(0xffffffffu, nw, j);
        if (!(w > 0.0f) || !isfinite(w)) continue;
        const float* e = p.emb + static_cast<int64_t>(nb[j]) * L;
        for (int a = 0; a < L; ++a) {
            const float za = __fsub_rn(e[a], zbar[a]);
            for (int b = 0; b < L; ++b)
                g[a * L + b] = __fadd_rn(g[a * L + b], __fmul_rn(__fmul_rn(w, za), __fsub_rn(e[b], zbar[b])));
        }
    }
    for (int c = 0; c < L; ++c) g[c * L + c] = __fadd_rn(g[c * L + c], 1e-3f);
    int perm[kInvMaxLow];
    const bool solve = non_zero > L && lu_factor(g, L, perm);
    const float* zq = p.zq + q * L;
    // per data dimension: x_bar, the rhs column, beta = gram^-1 rhs, the
    // prediction x_bar + (z - z_bar) beta (lib.rs:4870-4931)
    bool ok = true;
    for (int d0 = 0; d0 < D; d0 += 32) {
        const int d = d0 + lane;
        const bool in = d < D;
        float xbar = 0.0f;
        for (int j = 0; j < k; ++j) {
            const float w = __shfl_sync(0xffffffffu, nw, j);
            if (!(w > 0.0f) || !isfinite(w) || !in) continue;
            xbar = __fadd_rn(xbar, __fmul_rn(w, p.X[static_cast<int64_t>(nb[j]) * D + d]));
        }
        float pred = xbar;
        float rhs[kInvMaxLow];
        for (int a = 0; a < L; ++a) rhs[a] = 0.0f;
        for (int j = 0; j < k; ++j) {
            // every lane takes part in the shuffle; only lanes with a column add
            const float w = __shfl_sync(0xffffffffu, nw, j);
            if (!(w > 0.0f) || !isfinite(w) || !in || !solve) continue;
            const float* e = p.emb + static_cast<int64_t>(nb[j]) * L;
            const float xd = __fsub_rn(p.X[static_cast<int64_t>(nb[j]) * D + d], xbar);
            for (int a = 0; a < L; ++a)
                rhs[a] = __fadd_rn(rhs[a], __fmul_rn(__fmul_rn(w, __fsub_rn(e[a], zbar[a])), xd));
        }
        if (solve && in) {
            lu_solve(g, L, perm, rhs);
            float v = xbar;
            for (int a = 0; a < L; ++a) v = __fadd_rn(v, __fmul_rn(__fsub_rn(zq[a], zbar[a]), rhs[a]));
            if (!isfinite(v)) ok = false;
            pred = v;
        }
        if (in) out[d] = pred;
    }
    // a non-finite prediction anywhere keeps x_bar for the whole row
    if (solve && __any_sync(0xffffffffu, !ok)) {
        for (int d0 = 0; d0 < D; d0 += 32) {
            const int d = d0 + lane;
            float xbar = 0.0f;
            for (int j = 0; j < k; ++j) {
                const float w = __shfl_sync(0xffffffffu, nw, j);
                if (!(w > 0.0f) || !isfinite(w) || d >= D) continue;
                xbar = __fadd_rn(xbar, __fmul_rn(w, p.X[static_cast<int64_t>(nb[j]) * D + d]));
            }
            if (d < D) out[d] = xbar;
        }
    }
}

// Euclidean distance between a query row and a fitted row, reduced across
// the warp: (distance, 1e-6 + distance) as euclidean_distance_with_grad_denom
// (lib.rs:5035-5043).
__device__ __forceinline__ float warp_dist(const float* x, const float* y, int D, int lane) {
    float sq = 0.0f;
    for (int d = lane; d < D; d += 32) {
        const float df = __fsub_rn(x[d], y[d]);
        sq = __fadd_rn(sq, __fmul_rn(df, df));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq = __fadd_rn(sq, __shfl_xor_sync(0xffffffffu, sq, o));
    return sqrtf(sq);
}

__global__ void __launch_bounds__(256) inverse_sgd_kernel(InverseArgs p) {
    const int64_t q = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= p.nq || p.fixed[q]) return;
    const int D = p.D, k = p.k;
    const int32_t* nb = p.idx + q * k;
    float* cur = p.out + q * D;
    // per-edge schedule, lane j for neighbour j (make_epochs_per_sample over
    // the whole inverse graph, lib.rs:4937-4960)
    const float wl = lane < k ? p.w[q * k + lane] : 0.0f;
    const float nef = static_cast<float>(p.n_epochs);
    float eps = INFINITY;
    if (wl > 0.0f) {
        const float ns = __fmul_rn(nef, __fdiv_rn(wl, p.max_w));
        eps = ns > 0.0f ? __fdiv_rn(nef, ns) : INFINITY;
    }
    float next = eps;
    const float eps_neg = __fdiv_rn(eps, p.neg_rate_f);
    float next_neg = eps_neg;
    const uint64_t qseed = mix64(p.seed ^ mix64(static_cast<uint64_t>(q)));
    for (int64_t epoch = 0; epoch < p.n_epochs; ++epoch) {
        const float alpha = __fmul_rn(p.alpha0, __fsub_rn(1.0f, __fdiv_rn(static_cast<float>(epoch), nef)));
        const float ef = static_cast<float>(epoch);
        for (int j = 0; j < k; ++j) {
            const float wj = __shfl_sync(0xffffffffu, wl, j);
            if (!(wj > 0.0f)) continue;  // no edge for this neighbour
            if (__shfl_sync(0xffffffffu, next, j) > ef) continue;
            bool fin = true;
            for (int d = lane; d < D; d += 32) fin = fin && isfinite(cur[d]);
            if (!__all_sync(0xffffffffu, fin)) continue;
            const int32_t tail = nb[j];
            const float* other = p.X + static_cast<int64_t>(tail) * D;
            const float denom = __fadd_rn(1e-6f, warp_dist(cur, other, D, lane));
            const float gc = -__fdiv_rn(1.0f, __fadd_rn(__fmul_rn(wj, p.sig[tail]), 1e-6f));
            for (int d = lane; d < D; d += 32) {
                const float gd = clip4(__fmul_rn(gc, __fdiv_rn(__fsub_rn(cur[d], other[d]), denom)));
                cur[d] = __fadd_rn(cur[d], __fmul_rn(gd, alpha));
            }
            __syncwarp();
            if (lane == j) next = __fadd_rn(next, eps);
            const float en = __shfl_sync(0xffffffffu, eps_neg, j);
            if (!isfinite(en) || en <= 0.0f) continue;
            const float nn = __shfl_sync(0xffffffffu, next_neg, j);
            const uint32_t n_neg = floor_count(__fdiv_rn(__fsub_rn(ef, nn), en));
            for (uint32_t s = 0; s < n_neg; ++s) {
                const uint64_t word = rng_word(qseed, static_cast<uint64_t>(j),
                                               (static_cast<uint64_t>(epoch) << 32) | s);
                const uint32_t neg = rng_below(word, static_cast<uint32_t>(p.n));
                const float* o = p.X + static_cast<int64_t>(neg) * D;
                const float dn = warp_dist(cur, o, D, lane);
                const float sn = p.sig[neg];
                const float wh = expf(__fdiv_rn(-fmaxf(__fsub_rn(dn, p.rho[neg]), 1e-6f),
                                                __fadd_rn(sn, 1e-6f)));
                const float g2 = __fmul_rn(-p.rep, __fdiv_rn(__fsub_rn(0.0f, wh),
                                                              __fadd_rn(__fmul_rn(__fsub_rn(1.0f, wh), sn), 1e-6f)));
                const float den2 = __fadd_rn(1e-6f, dn);
                for (int d = lane; d < D; d += 32) {
                    const float gd = clip4(__fmul_rn(g2, __fdiv_rn(__fsub_rn(cur[d], o[d]), den2)));
                    cur[d] = __fadd_rn(cur[d], __fmul_rn(gd, alpha));
                }
                __syncwarp();
            }
            if (lane == j) next_neg = __fadd_rn(nn, __fmul_rn(static_cast<float>(n_neg), en));
        }
    }
}

}  // namespace

void local_radii(const int32_t* idx, const float* dist, int64_t n, int k, float var_shift,
                 float* out, cudaStream_t s) {
    if (n == 0) return;
    local_radii_kernel<<<static_cast<unsigned>(ceil_div(n, 256)), 256, 0, s>>>(idx, dist, n, k,
                                                                             var_shift, out);
    UMAPB_LAUNCH_CHECK();
}

void embedding_radii(const float* emb, int dim, const int32_t* idx, int64_t n, int k,
                     float var_shift, float* out, cudaStream_t s) {
    if (n == 0) return;
    embedding_radii_kernel<<<static_cast<unsigned>(ceil_div(n, 256)), 256, 0, s>>>(
        emb, dim, idx, n, k, var_shift, out);
    UMAPB_LAUNCH_CHECK();
}

int64_t density_start_epoch(int64_t n_epochs, float frac) {
    // lib.rs:5052-5055, the product taken in f32
    const int64_t active = std::max<int64_t>(
        static_cast<int64_t>(std::ceil(static_cast<float>(n_epochs) * frac)), 1);
    return n_epochs > active ? n_epochs - active : 0;
}

double optimize_layout(float* emb, int64_t n_vertices, int dim, const Graph& g, int64_t n_epochs,
                       float a, float b, float lr, int64_t neg_rate, float repulsion,
                       uint64_t seed, bool count_samples, float* kernel_ms, cudaStream_t s,
                       const DensityParams* dens) {
    const int64_t m = g.n_edges;
    if (m == 0 || n_vertices == 0 || n_epochs == 0) return 0.0;
    if (dim > kMaxDim) invalid("n_components above 16 is not supported by the GPU layout kernel");
    if (!dens && n_vertices * dim <= kSmallLayoutFloats && m <= 0x7FFFFFFFll)
        return optimize_layout_small(emb, n_vertices, dim, g, n_epochs, a, b, lr, neg_rate,
                                     repulsion, seed, kernel_ms, s);
    const float mx = std::max(max_weight(g.weights.get(), m, s), 1e-12f);
    DevBuf<int32_t> sorted_heads, sorted_tails;
    if (m > 0x7FFFFFFFll) invalid("optimize_layout: too many edges");
    DevBuf<float> eps(m, s), next(m, s), next_neg(m, s);
    const float nef = static_cast<float>(n_epochs);
    const float nrf = static_cast<float>(neg_rate);
    const unsigned grid = static_cast<unsigned>(ceil_div(m, 256));
    {
        // Edge periods (make_epochs_per_sample, lib.rs:4937-4960).  Within
        // each window of consecutive edges (graph order, by head) the
        // edges are ordered by period: edges with close periods fire in the
        // same epochs, so the lanes of a warp mostly fire together, while the
        // sweep over heads keeps the graph order across the epoch.  Each
        // edge's schedule and arithmetic are the reference's; only the order
        // of concurrent edges changes, as in any Hogwild order.
        DevBuf<float> eps_raw(m, s);
        epochs_per_sample_kernel<<<grid, 256, 0, s>>>(g.weights.get(), m, mx, nef, nrf,
                                                      eps_raw.get(), nullptr, nullptr);
        UMAPB_LAUNCH_CHECK();
        DevBuf<uint64_t> keys(m, s), keys_sorted(m, s);
        DevBuf<int32_t> ids(m, s), order(m, s);
        const int shift = sort_window_shift(m);
        period_keys_kernel<<<grid, 256, 0, s>>>(eps_raw.get(), m, shift, keys.get(), ids.get());
        UMAPB_LAUNCH_CHECK();
        int window_bits = 1;
        while ((static_cast<int64_t>(1) << window_bits) <= (m >> shift)) ++window_bits;
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.get(), keys_sorted.get(), ids.get(),
                                        order.get(), static_cast<int>(m), 0, 32 + window_bits, s);
        DevBuf<uint8_t> tmp(bytes, s);
        cub::DeviceRadixSort::SortPairs(tmp.get(), bytes, keys.get(), keys_sorted.get(),
                                        ids.get(), order.get(), static_cast<int>(m), 0,
                                        32 + window_bits, s);
        UMAPB_CUDA(cudaGetLastError());
        sorted_heads.alloc(m, s);
        sorted_tails.alloc(m, s);
        gather_edges_kernel<<<grid, 256, 0, s>>>(order.get(), g.heads.get(), g.tails.get(),
                                                 eps_raw.get(), nrf, m, sorted_heads.get(),
                                                 sorted_tails.get(), eps.get(), next.get(),
                                                 next_neg.get());
        UMAPB_LAUNCH_CHECK();
    }
    SgdArgs p{};
    p.emb = emb;
    p.heads = sorted_heads.get();
    p.tails = sorted_tails.get();
    p.eps = eps.get();
    p.next = next.get();
    p.next_neg = next_neg.get();
    p.n_edges = m;
    p.n_vertices = static_cast<uint32_t>(n_vertices);
    p.dim = dim;
    p.a = a;
    p.b = b;
    p.att_factor = -2.0f * a * b;
    p.rep_factor = 2.0f * repulsion * b;
    p.neg_rate_f = nrf;
    p.seed = seed;
    if (dens) {
        p.radii = dens->radii;
        p.dens_lambda = dens->lambda;
        p.dens_var_shift = dens->var_shift;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernel_ms) {
        UMAPB_CUDA(cudaEventCreate(&e0));
        UMAPB_CUDA(cudaEventCreate(&e1));
        UMAPB_CUDA(cudaEventRecord(e0, s));
    }
    for (int64_t epoch = 0; epoch < n_epochs; ++epoch) {
        // alpha = initial_alpha * (1 - epoch / n_epochs) in FP32 (lib.rs:5174)
        p.alpha = lr * (1.0f - static_cast<float>(epoch) / nef);
        p.epoch_f = static_cast<float>(epoch);
        p.epoch = static_cast<uint64_t>(epoch);
        if (dens) {
            p.dens_on = epoch >= dens->start_epoch ? 1 : 0;
            sgd_epoch_dens<<<grid, 256, 0, s>>>(p);
        } else if (dim == 2) {
            sgd_epoch_2d<<<grid, 256, 0, s>>>(p);
        } else {
            sgd_epoch_nd<<<grid, 256, 0, s>>>(p);
        }
        UMAPB_LAUNCH_CHECK();
    }
    if (kernel_ms) {
        UMAPB_CUDA(cudaEventRecord(e1, s));
        UMAPB_CUDA(cudaEventSynchronize(e1));
        UMAPB_CUDA(cudaEventElapsedTime(kernel_ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (!count_samples) return 0.0;
    DevBuf<unsigned long long> total(1, s);
    UMAPB_CUDA(cudaMemsetAsync(total.get(), 0, 8, s));
    count_samples_kernel<<<std::min<unsigned>(grid, 148u * 8u), 256, 0, s>>>(eps.get(), m, n_epochs,
                                                                         total.get());
    UMAPB_LAUNCH_CHECK();
    unsigned long long h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, total.get(), 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return static_cast<double>(h);
}

void transform_layout(float* out, int64_t nq, int dim, const float* base, int64_t n_base,
                      const Graph& g, int64_t n_epochs, float a, float b, float lr,
                      int64_t neg_rate, float repulsion, uint64_t seed, cudaStream_t s,
                      const int32_t* qid, int64_t qid_offset) {
    if (nq == 0) return;
    if (dim > kMaxDim) invalid("n_components above 16 is not supported by the GPU layout kernel");
    const int64_t m = g.n_edges;
    DevBuf<float> eps(std::max<int64_t>(m, 1), s), next(std::max<int64_t>(m, 1), s),
        next_neg(std::max<int64_t>(m, 1), s);
    const float nef = static_cast<float>(n_epochs);
    const float nrf = static_cast<float>(neg_rate);
    if (m > 0) {
        const bool local = g.row_max.get() != nullptr;
        const float mx = local ? 1.0f : std::max(max_weight(g.weights.get(), m, s), 1e-12f);
        epochs_per_sample_kernel<<<static_cast<unsigned>(ceil_div(m, 256)), 256, 0, s>>>(
            g.weights.get(), m, mx, nef, nrf, eps.get(), next.get(), next_neg.get(),
            local ? g.row_max.get() : nullptr, local ? g.heads.get() : nullptr);
        UMAPB_LAUNCH_CHECK();
    }
    TransformArgs p{};
    p.out = out;
    p.base = base;
    p.row_ptr = g.row_ptr.get();
    p.tails = g.tails.get();
    p.weights = g.weights.get();
    p.eps = eps.get();
    p.next = next.get();
    p.next_neg = next_neg.get();
    p.nq = nq;
    p.n_base = static_cast<uint32_t>(n_base);
    p.dim = dim;
    p.n_epochs = n_epochs;
    p.a = a;
    p.b = b;
    p.lr = lr;
    p.rep = repulsion;
    p.neg_rate_f = nrf;
    p.seed = seed;
    p.qid = qid;
    p.qid_offset = qid_offset;
    transform_kernel<<<static_cast<unsigned>(ceil_div(nq, static_cast<int64_t>(kTransformThreads))),
                       kTransformThreads, 0, s>>>(p);
    UMAPB_LAUNCH_CHECK();
}

void inverse_layout(const float* zq, int64_t nq, int L, const int32_t* idx, const float* dist,
                    int k, const float* emb, const float* X, int64_t n, int D, const float* sig,
                    const float* rho, float a, float b, int64_t n_epochs, float lr,
                    int64_t neg_rate, float repulsion, uint64_t seed, float* out,
                    cudaStream_t s) {
    if (nq == 0) return;
    if (L > kInvMaxLow) invalid("inverse_transform supports n_components <= 16 on the GPU path");
    if (k > kInvMaxK) invalid("inverse_transform supports n_neighbors <= 32 on the GPU path");
    DevBuf<float> w(nq * k, s);
    DevBuf<uint8_t> fixed(nq, s);
    InverseArgs p{};
    p.zq = zq;
    p.idx = idx;
    p.dist = dist;
    p.emb = emb;
    p.X = X;
    p.sig = sig;
    p.rho = rho;
    p.out = out;
    p.w = w.get();
    p.fixed = fixed.get();
    p.nq = nq;
    p.n = n;
    p.L = L;
    p.D = D;
    p.k = k;
    p.a = a;
    p.b = b;
    const unsigned grid = static_cast<unsigned>(ceil_div(nq * 32, 256));
    inverse_init_kernel<<<grid, 256, 0, s>>>(p);
    UMAPB_LAUNCH_CHECK();
    // optimize_layout_inverse returns at once for an empty graph or 0 epochs
    const float mx = max_weight(w.get(), nq * k, s);
    if (n_epochs == 0 || !(mx > 0.0f)) return;
    p.max_w = mx;
    p.n_epochs = n_epochs;
    p.alpha0 = lr / 4.0f;
    p.neg_rate_f = static_cast<float>(neg_rate);
    p.rep = repulsion;
    p.seed = seed;
    inverse_sgd_kernel<<<grid, 256, 0, s>>>(p);
    UMAPB_LAUNCH_CHECK();
}

}  // namespace umapb
