// spectral.cu - spectral initialisation (rust_umap/src/lib.rs:3841-4791).
//
// The reference runs, per connected component, block subspace iteration on
// the shifted operator I + D^-1/2 W D^-1/2: 256 iterations, s = (dim+1)*6
// columns, modified Gram-Schmidt applied twice in FP64, then a Rayleigh-Ritz
// step (lib.rs:4227-4326).  Here all components of the graph that take the
// iterative path run at once: the sparse product is one pull-style SpMM over
// the CSR graph (components never share edges, so the operator is block
// diagonal), the block is kept in FP32 (N x s, L2 resident at 1M rows), and
// orthonormalisation is CholQR2 per component: the s x s Gram matrix is
// reduced in FP64, factored in FP64 on the device, and its inverse factor is
// applied in FP64.  CholQR and MGS produce the same orthonormal basis in exact
// arithmetic (the unique QR factor with positive diagonal); the MGS failure
// test (column norm^2 <= 1e-12 after projection, lib.rs:4188) is the
// Cholesky pivot test.  The block is orthonormalised after every fourth
// product instead of every product: the span of (I + A)^4 X does not depend
// on whether X was re-orthonormalised in between (exactly so in exact
// arithmetic), and over four products of an operator with spectrum in [0, 2]
// the columns' condition grows by at most 2^4 on the bulk of the spectrum,
// far inside what an FP64 Gram matrix of FP32 columns resolves.  256 is a
// multiple of 4, so the last product is followed by an orthonormalisation as
// in the reference.  The Ritz matrices are solved on the host.
//
// Small pieces follow the reference on the host: the dense Laplacian path
// (lib.rs:4007-4069, 3917-3957) for components below 128 nodes or connected
// inputs with <= 8 features and <= 2048 rows, random init for components
// with fewer than 2*dim nodes, and the meta layout of component centroids
// (lib.rs:4519-4554).  Random numbers (initial block, noise, random layouts)
// come from counter-based streams, not the reference's SmallRng sequence.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "kernels.cuh"

namespace umapb {
namespace {

constexpr int kIters = 256;             // SPECTRAL_ITERATIVE_MAX_ITERS (lib.rs:31)
constexpr int kOrthoEvery = 4;          // products between orthonormalisations
constexpr int kOversampling = 6;        // lib.rs:32
constexpr int64_t kComponentIterThreshold = 128;  // lib.rs:30
constexpr int64_t kDenseFallbackMax = 4096;       // lib.rs:33
constexpr double kOrthoEps = 1e-12;     // lib.rs:34
constexpr float kInitMaxCoord = 10.0f;  // lib.rs:22
constexpr float kInitNoise = 1e-4f;     // lib.rs:23
constexpr int kMaxS = 32;               // s <= 32 -> n_components <= 4

inline unsigned grid_for(int64_t n, int t = 256) {
    return static_cast<unsigned>(ceil_div(std::max<int64_t>(n, 1), t));
}

// ---------------------------------------------------- components (device)
__device__ inline int32_t find_root(const int32_t* parent, int32_t x) {
    int32_t p = parent[x];
    while (p != x) {
        x = p;
        p = parent[x];
    }
    return x;
}

__global__ void cc_init(int32_t* parent, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) parent[i] = static_cast<int32_t>(i);
}

__global__ void cc_hook(const int32_t* __restrict__ heads, const int32_t* __restrict__ tails,
                        int64_t m, int32_t* parent, int* changed) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int32_t u = heads[e], v = tails[e];
    if (u >= v) return;  // each undirected pair once
    const int32_t ru = find_root(parent, u), rv = find_root(parent, v);
    if (ru == rv) return;
    const int32_t hi = ru > rv ? ru : rv, lo = ru > rv ? rv : ru;
    atomicMin(&parent[hi], lo);
    *changed = 1;
}

__global__ void cc_compress(int32_t* parent, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) parent[i] = find_root(parent, static_cast<int32_t>(i));
}

__global__ void cc_is_root(const int32_t* parent, int64_t n, int32_t* flag) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = parent[i] == i ? 1 : 0;
}

__global__ void cc_label(const int32_t* parent, const int32_t* rank, int64_t n, int32_t* label) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) label[i] = rank[parent[i]];
}

__global__ void iota_kernel(int32_t* v, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) v[i] = static_cast<int32_t>(i);
}

// --------------------------------------------------- subspace iteration --
__global__ void degree_kernel(const int32_t* __restrict__ row_ptr, const float* __restrict__ w,
                              int64_t n, double* __restrict__ deg, float* __restrict__ dinv) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int32_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) s += static_cast<double>(w[e]);
    deg[i] = s;
    dinv[i] = s > 0.0 ? static_cast<float>(1.0 / sqrt(s)) : 0.0f;
}

__global__ void norm_weight_kernel(const int32_t* __restrict__ heads,
                                   const int32_t* __restrict__ tails, const float* __restrict__ w,
                                   const double* __restrict__ deg, int64_t m,
                                   float* __restrict__ nw) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const double di = deg[heads[e]], dj = deg[tails[e]];
    const double ii = di > 0.0 ? 1.0 / sqrt(di) : 0.0, ij = dj > 0.0 ? 1.0 / sqrt(dj) : 0.0;
    nw[e] = static_cast<float>(static_cast<double>(w[e]) * ii * ij);
}

// The iterative components' rows are processed in "position" order: the
// nodes of slot 0, then slot 1, ... (slots = components on the iterative
// path).  Blocks X and Y are stored in that order, so every pass except the
// SpMM gathers streams contiguous memory.

__global__ void pos_kernel(const int32_t* __restrict__ nodes, int64_t cnt, int32_t* __restrict__ pos) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p < cnt) pos[nodes[p]] = static_cast<int32_t>(p);
}

__global__ void prow_len_kernel(const int32_t* __restrict__ nodes, int64_t cnt,
                                const int32_t* __restrict__ row_ptr, int32_t* __restrict__ len) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p < cnt) {
        const int32_t v = nodes[p];
        len[p] = row_ptr[v + 1] - row_ptr[v];
    }
}

// CSR of the shifted operator in position order (tails mapped to positions).
__global__ void pcsr_kernel(const int32_t* __restrict__ nodes, int64_t cnt,
                            const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ tails,
                            const float* __restrict__ nw, const int32_t* __restrict__ pos,
                            const int32_t* __restrict__ prow_ptr, int32_t* __restrict__ ptails,
                            float* __restrict__ pnw) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= cnt) return;
    const int32_t v = nodes[p];
    int32_t o = prow_ptr[p];
    for (int32_t e = row_ptr[v]; e < row_ptr[v + 1]; ++e, ++o) {
        ptails[o] = pos[tails[e]];
        pnw[o] = nw[e];
    }
}

// Initial block: column 0 = sqrt(degree), the others U(-1, 1) (lib.rs:4254-4261).
__global__ void init_block_kernel(const int32_t* __restrict__ nodes, int64_t cnt,
                                  const int32_t* __restrict__ slot_of_pos,
                                  const uint64_t* __restrict__ slot_seed,
                                  const double* __restrict__ deg, int s, int sp,
                                  float* __restrict__ X) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    const int32_t i = nodes[t];
    const uint64_t seed = slot_seed[slot_of_pos[t]] ^ 0x7A5B3D91CE42A117ULL;
    float* row = X + t * sp;
    row[0] = static_cast<float>(sqrt(deg[i]));
    for (int c = 1; c < sp; ++c) {
        float v = 0.0f;
        if (c < s) v = static_cast<float>(-1.0 + 2.0 * rng_unit_f64(rng_word(seed, i, c)));
        row[c] = v;
    }
}

// Y = X + A_hat X in position order.  SP / 4 lanes share a row, one float4
// of it each, so every neighbour's row is gathered by one coalesced access;
// each lane sums its components over the row's edges in edge order.
template <int SP>
__host__ __device__ constexpr int spmm_rows_per_warp() { return 32 / (SP / 4); }

template <int SP>
__global__ void __launch_bounds__(256)
    spmm_kernel(int64_t cnt, const int32_t* __restrict__ prow_ptr,
                const int32_t* __restrict__ ptails, const float* __restrict__ pnw,
                const float* __restrict__ X, float* __restrict__ Y) {
    constexpr int V = SP / 4;
    constexpr int RW = spmm_rows_per_warp<SP>();
    const int lane = threadIdx.x & 31;
    const int sub = lane / V, v = lane - sub * V;
    const int64_t t =
        ((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * RW + sub;
    if (sub >= RW || t >= cnt) return;
    float4 acc = reinterpret_cast<const float4*>(X + t * SP)[v];
    const int32_t st = prow_ptr[t], en = prow_ptr[t + 1];
#pragma unroll 4
    for (int32_t e = st; e < en; ++e) {
        const float wv = __ldg(pnw + e);
        const float4 q =
            __ldg(reinterpret_cast<const float4*>(X + static_cast<int64_t>(__ldg(ptails + e)) * SP) + v);
        acc.x = fmaf(wv, q.x, acc.x);
        acc.y = fmaf(wv, q.y, acc.y);
        acc.z = fmaf(wv, q.z, acc.z);
        acc.w = fmaf(wv, q.w, acc.w);
    }
    reinterpret_cast<float4*>(Y + t * SP)[v] = acc;
}

struct Chunk {
    int32_t slot;
    int32_t start;  // position range [start, end)
    int32_t end;
};

// Upper triangle of A^T B per slot over contiguous position ranges, FP64.
// S is a multiple of 3 ((dim + 1) * 6), so the upper triangle is covered by
// NT = T (T + 1) / 2 tiles of 3 x 3 entries (T = S / 3); thread t owns tile
// t % NT for the rows t / NT, t / NT + G, ... of each staged slab (G row
// groups).  Slabs of R rows are staged in shared memory as FP64, the next
// slab's FP32 rows wait in registers meanwhile; at the end the G partial
// tiles are summed in shared memory and added to G atomically.
template <int S, int SP>
struct GramShape {
    static_assert(S % 3 == 0, "the block width is a multiple of 3");
    static constexpr int T = S / 3;
    static constexpr int NT = T * (T + 1) / 2;
    static constexpr int G = 256 / NT;
    static constexpr int R = SP <= 20 ? 128 : 64;  // rows per slab
    static constexpr int V4 = R * SP / 4;          // float4 per slab and operand
    static constexpr int PF = (V4 + 255) / 256;    // float4 per thread and operand
    static constexpr int kStage = 2 * R * SP;      // doubles
    static constexpr int kReduce = G * NT * 9;     // doubles
    static constexpr int kSmem = kStage > kReduce ? kStage : kReduce;
    static_assert(kSmem * 8 <= 48 * 1024, "static shared memory");
};

template <int S, int SP>
__global__ void __launch_bounds__(256)
    gram_kernel(const Chunk* __restrict__ chunks, const float* __restrict__ A,
                const float* __restrict__ B, double* __restrict__ G) {
    using Sh = GramShape<S, SP>;
    __shared__ double sm[Sh::kSmem];
    // A^T A (every orthonormalisation) stages one operand; A^T B (the Ritz
    // step) two
    const bool same = A == B;
    double* As = sm;
    double* Bs = same ? sm : sm + Sh::R * SP;
    const Chunk ch = chunks[blockIdx.x];
    const int tid = threadIdx.x;
    const bool worker = tid < Sh::G * Sh::NT;
    const int tile = tid % Sh::NT, grp = tid / Sh::NT;
    int tp = 0, tq = tile;  // tile (tp, tq), tp <= tq
    while (tq >= Sh::T - tp) {
        tq -= Sh::T - tp;
        ++tp;
    }
    tq += tp;
    double acc[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) acc[i][j] = 0.0;

    float4 pa[Sh::PF], pb[Sh::PF];
    auto prefetch = [&](int r0) {
        const int rows = min(Sh::R, ch.end - r0);
        const float4* a4 = reinterpret_cast<const float4*>(A + static_cast<int64_t>(r0) * SP);
        const float4* b4 = reinterpret_cast<const float4*>(B + static_cast<int64_t>(r0) * SP);
#pragma unroll
        for (int k = 0; k < Sh::PF; ++k) {
            const int e = tid + k * 256;
            if (e < rows * SP / 4) {
                pa[k] = a4[e];
                if (!same) pb[k] = b4[e];
            }
        }
    };
    if (ch.start < ch.end) prefetch(ch.start);
    for (int r0 = ch.start; r0 < ch.end; r0 += Sh::R) {
        const int rows = min(Sh::R, ch.end - r0);
        __syncthreads();  // the previous slab's products are done
#pragma unroll
        for (int k = 0; k < Sh::PF; ++k) {
            const int e = tid + k * 256;
            if (e < rows * SP / 4) {
                As[4 * e] = pa[k].x;
                As[4 * e + 1] = pa[k].y;
                As[4 * e + 2] = pa[k].z;
                As[4 * e + 3] = pa[k].w;
                if (!same) {
                    Bs[4 * e] = pb[k].x;
                    Bs[4 * e + 1] = pb[k].y;
                    Bs[4 * e + 2] = pb[k].z;
                    Bs[4 * e + 3] = pb[k].w;
                }
            }
        }
        __syncthreads();
        if (r0 + Sh::R < ch.end) prefetch(r0 + Sh::R);
        if (worker) {
            for (int r = grp; r < rows; r += Sh::G) {
                const double* ar = As + r * SP + 3 * tp;
                const double* br = Bs + r * SP + 3 * tq;
                const double a0 = ar[0], a1 = ar[1], a2 = ar[2];
                const double b0 = br[0], b1 = br[1], b2 = br[2];
                acc[0][0] = fma(a0, b0, acc[0][0]);
                acc[0][1] = fma(a0, b1, acc[0][1]);
                acc[0][2] = fma(a0, b2, acc[0][2]);
                acc[1][0] = fma(a1, b0, acc[1][0]);
                acc[1][1] = fma(a1, b1, acc[1][1]);
                acc[1][2] = fma(a1, b2, acc[1][2]);
                acc[2][0] = fma(a2, b0, acc[2][0]);
                acc[2][1] = fma(a2, b1, acc[2][1]);
                acc[2][2] = fma(a2, b2, acc[2][2]);
            }
        }
    }
    __syncthreads();  // the staging buffer becomes the reduction buffer
    if (worker) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) sm[(grp * Sh::NT + tile) * 9 + i * 3 + j] = acc[i][j];
    }
    __syncthreads();
    for (int o = tid; o < Sh::NT * 9; o += 256) {
        const int t = o / 9, ij = o - t * 9, i = ij / 3, j = ij - i * 3;
        int p = 0, q = t;
        while (q >= Sh::T - p) {
            q -= Sh::T - p;
            ++p;
        }
        q += p;
        const int ea = 3 * p + i, eb = 3 * q + j;
        if (ea > eb) continue;  // lower part of a diagonal tile
        double v = 0.0;
        for (int g = 0; g < Sh::G; ++g) v += sm[(g * Sh::NT + t) * 9 + ij];
        atomicAdd(&G[static_cast<int64_t>(ch.slot) * S * S + ea * S + eb], v);
    }
}

// G = L L^T per slot, one warp: lane i keeps row i; right-looking updates
// with the pivot column shared by shuffles.  A pivot <= 1e-12 is the MGS
// failure of the reference (column norm^2 after projection).
template <int S>
__global__ void chol_kernel(const double* __restrict__ G, double* __restrict__ Lout,
                            double* __restrict__ dinv, int* __restrict__ fail) {
    const int slot = blockIdx.x;
    const int lane = threadIdx.x;
    const double* g = G + static_cast<int64_t>(slot) * S * S;
    double row[S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        double v = 0.0;
        if (lane < S) v = lane <= k ? g[lane * S + k] : g[k * S + lane];
        row[k] = v;
    }
    bool ok = true;
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const double pivot = __shfl_sync(0xffffffffu, row[j], j);
        if (!(pivot > kOrthoEps) || !isfinite(pivot)) {
            ok = false;
            break;
        }
        const double ljj = sqrt(pivot);
        const double lij = lane == j ? ljj : row[j] / ljj;
        if (lane >= j) row[j] = lij;
#pragma unroll
        for (int k = j + 1; k < S; ++k) {
            const double lkj = __shfl_sync(0xffffffffu, lij, k);
            if (lane > j) row[k] -= lij * lkj;
        }
    }
    if (!ok) {
        if (lane == 0) fail[slot] = 1;
        if (lane < S) {
#pragma unroll
            for (int k = 0; k < S; ++k) Lout[static_cast<int64_t>(slot) * S * S + lane * S + k] = lane == k;
            dinv[slot * S + lane] = 1.0;
        }
        return;
    }
    if (lane < S) {
#pragma unroll
        for (int k = 0; k < S; ++k)
            Lout[static_cast<int64_t>(slot) * S * S + lane * S + k] = k <= lane ? row[k] : 0.0;
        dinv[slot * S + lane] = 1.0 / row[lane];
    }
}

// X = Y L^-T by forward substitution per row, FP64.  A block takes 256
// consecutive rows: they are staged in shared memory with coalesced loads,
// solved in place, and written back with coalesced stores (a row stride of
// SP floats, a multiple of 4, keeps the 16-byte shared accesses of a
// quarter-warp on distinct banks).  Each thread solves rows t and t + 128;
// when both lie in the same slot (the common case: slots are contiguous
// position ranges of at least 128 rows) every load of L serves both rows.
constexpr int kApplyRows = 256;
constexpr int kApplyThreads = 128;

template <int S, int SP, int NR>
__device__ __forceinline__ void solve_rows(float* const (&row)[NR], const double* __restrict__ Ls,
                                           const double* __restrict__ di) {
    double x[NR][S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
        double v[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) v[q] = static_cast<double>(row[q][c]);
#pragma unroll
        for (int a = 0; a < c; ++a) {
            const double l = __ldg(Ls + c * S + a);
#pragma unroll
            for (int q = 0; q < NR; ++q) v[q] -= x[q][a] * l;
        }
        const double d = __ldg(di + c);
#pragma unroll
        for (int q = 0; q < NR; ++q) x[q][c] = v[q] * d;
    }
#pragma unroll
    for (int q = 0; q < NR; ++q) {
        float4* r4 = reinterpret_cast<float4*>(row[q]);
#pragma unroll
        for (int v = 0; v < SP / 4; ++v) {
            float o[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                o[k] = 4 * v + k < S ? static_cast<float>(x[q][4 * v + k]) : 0.0f;
            r4[v] = make_float4(o[0], o[1], o[2], o[3]);
        }
    }
}

template <int S, int SP>
__global__ void __launch_bounds__(kApplyThreads)
    apply_kernel(int64_t cnt, const int32_t* __restrict__ slot_of_pos,
                 const double* __restrict__ L, const double* __restrict__ dinv,
                 const float* __restrict__ Y, float* __restrict__ X) {
    __shared__ __align__(16) float rows[kApplyRows * SP];
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kApplyRows;
    const int nrows = static_cast<int>(min(static_cast<int64_t>(kApplyRows), cnt - r0));
    const float4* y4 = reinterpret_cast<const float4*>(Y + r0 * SP);
    float4* s4 = reinterpret_cast<float4*>(rows);
    for (int e = threadIdx.x; e < nrows * SP / 4; e += kApplyThreads) s4[e] = y4[e];
    __syncthreads();
    const int ta = threadIdx.x, tb = threadIdx.x + kApplyThreads;
    const int sa = ta < nrows ? slot_of_pos[r0 + ta] : -1;
    const int sb = tb < nrows ? slot_of_pos[r0 + tb] : -1;
    auto Lof = [&](int slot) { return L + static_cast<int64_t>(slot) * S * S; };
    if (sa >= 0 && sa == sb) {
        float* const both[2] = {rows + ta * SP, rows + tb * SP};
        solve_rows<S, SP, 2>(both, Lof(sa), dinv + sa * S);
    } else {
        if (sa >= 0) {
            float* const one[1] = {rows + ta * SP};
            solve_rows<S, SP, 1>(one, Lof(sa), dinv + sa * S);
        }
        if (sb >= 0) {
            float* const one[1] = {rows + tb * SP};
            solve_rows<S, SP, 1>(one, Lof(sb), dinv + sb * S);
        }
    }
    __syncthreads();
    float4* x4 = reinterpret_cast<float4*>(X + r0 * SP);
    for (int e = threadIdx.x; e < nrows * SP / 4; e += kApplyThreads) x4[e] = s4[e];
}

// coords = X V (V: s x dim per slot), FP64; and per-slot max |coord|.
__global__ void project_kernel(const int32_t* __restrict__ nodes, int64_t cnt,
                               const int32_t* __restrict__ slot_of_pos,
                               const double* __restrict__ V, int s, int sp, int dim,
                               const float* __restrict__ X, float* __restrict__ out,
                               unsigned* __restrict__ max_abs_bits) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    const int64_t i = nodes[t];
    const int slot = slot_of_pos[t];
    const double* v = V + static_cast<int64_t>(slot) * s * dim;
    float mx = 0.0f;
    for (int oc = 0; oc < dim; ++oc) {
        double acc = 0.0;
        for (int b = 0; b < s; ++b) acc += static_cast<double>(X[t * sp + b]) * v[b * dim + oc];
        const float f = static_cast<float>(acc);
        out[i * dim + oc] = f;
        mx = fmaxf(mx, fabsf(f));
    }
    atomicMax(&max_abs_bits[slot], __float_as_uint(mx));
}

// coord = coord * expansion + N(0, noise) + anchor (noisy_scale_coords,
// lib.rs:4766-4791, and the per-component placement of lib.rs:4713-4752).
__global__ void finish_kernel(const int32_t* __restrict__ nodes, int64_t cnt,
                              const int32_t* __restrict__ slot_of_node,
                              const float* __restrict__ expansion,
                              const float* __restrict__ anchors, const uint64_t* __restrict__ nseed,
                              int dim, float noise, float* __restrict__ out) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    const int64_t i = nodes[t];
    const int slot = slot_of_node[t];
    for (int c = 0; c < dim; ++c) {
        const uint64_t w1 = rng_word(nseed[slot], static_cast<uint64_t>(i), 2 * c);
        const uint64_t w2 = rng_word(nseed[slot], static_cast<uint64_t>(i), 2 * c + 1);
        double u1 = rng_unit_f64(w1);
        if (u1 < 1e-300) u1 = 1e-300;
        const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * rng_unit_f64(w2));
        const float v = out[i * dim + c] * expansion[slot] + static_cast<float>(noise * z);
        out[i * dim + c] = v + anchors[slot * dim + c];
    }
}

__global__ void random_init_kernel(int64_t n, int dim, uint64_t seed, float low, float high,
                                   float* out) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * dim) return;
    const float u = rng_unit_f32(rng_word(seed, static_cast<uint64_t>(t / dim), t % dim));
    out[t] = low + u * (high - low);
}

__global__ void scatter_rows_kernel(const int32_t* __restrict__ nodes, int64_t cnt, int dim,
                                    const float* __restrict__ vals, float* __restrict__ out) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= cnt * dim) return;
    out[static_cast<int64_t>(nodes[t / dim]) * dim + t % dim] = vals[t];
}

// centroid sums per component (FP64) over the component-sorted node list
__global__ void centroid_kernel(const Chunk* __restrict__ chunks, const int32_t* __restrict__ nodes,
                                const float* __restrict__ X, int d, double* __restrict__ cent) {
    const Chunk ch = chunks[blockIdx.x];
    for (int f = threadIdx.x; f < d; f += blockDim.x) {
        double acc = 0.0;
        for (int r = ch.start; r < ch.end; ++r)
            acc += static_cast<double>(X[static_cast<int64_t>(nodes[r]) * d + f]);
        atomicAdd(&cent[static_cast<int64_t>(ch.slot) * d + f], acc);
    }
}

// the same sums from CSR rows (component_centroids_sparse, lib.rs:4487-4505)
__global__ void centroid_csr_kernel(const Chunk* __restrict__ chunks,
                                    const int32_t* __restrict__ nodes,
                                    const int64_t* __restrict__ indptr,
                                    const int32_t* __restrict__ indices,
                                    const float* __restrict__ values, int d,
                                    double* __restrict__ cent) {
    const Chunk ch = chunks[blockIdx.x];
    for (int r = ch.start + static_cast<int>(threadIdx.x); r < ch.end; r += blockDim.x) {
        const int64_t v = nodes[r];
        for (int64_t e = indptr[v]; e < indptr[v + 1]; ++e)
            atomicAdd(&cent[static_cast<int64_t>(ch.slot) * d + indices[e]],
                      static_cast<double>(values[e]));
    }
}

// ------------------------------------------------------------ host side --
using HostCoords = std::vector<float>;  // row-major n x dim

bool finite_all(const std::vector<float>& v) {
    for (float x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

// normalized_laplacian_from_edges + spectral_embedding_from_laplacian
// (lib.rs:4007-4069, 3917-3957) for a small component given its local edges.
bool dense_spectral(int64_t n, int dim, const std::vector<std::array<int64_t, 2>>& pairs,
                    const std::vector<float>& w, HostCoords& out) {
    if (n <= dim + 1 || pairs.empty()) return false;
    std::vector<double> L(n * n, 0.0), deg(n, 0.0);
    for (int64_t i = 0; i < n; ++i) L[i * n + i] = 1.0;
    std::vector<std::pair<int64_t, int64_t>> und;
    for (size_t e = 0; e < pairs.size(); ++e) {
        const int64_t h = pairs[e][0], t = pairs[e][1];
        if (h == t) continue;
        const double wv = static_cast<double>(std::max(w[e], 0.0f));
        if (wv <= 0.0) continue;
        const int64_t i = std::min(h, t), j = std::max(h, t);
        const double prev = L[i * n + j];
        if (wv > prev) {
            if (prev == 0.0) und.emplace_back(i, j);
            const double delta = wv - prev;
            L[i * n + j] = wv;
            L[j * n + i] = wv;
            deg[i] += delta;
            deg[j] += delta;
        }
    }
    bool any = false;
    for (double v : deg) any |= v > 0.0;
    if (!any) return false;
    std::vector<double> inv(n);
    for (int64_t i = 0; i < n; ++i) inv[i] = deg[i] > 0 ? 1.0 / std::sqrt(deg[i]) : 0.0;
    for (auto [i, j] : und) {
        const double v = L[i * n + j] * inv[i] * inv[j];
        L[i * n + j] = -v;
        L[j * n + i] = -v;
    }
    for (int64_t i = 0; i < n; ++i) L[i * n + i] = 1.0;
    std::vector<double> ev, V;
    symmetric_eigen(L, static_cast<int>(n), ev, V);
    if (n <= dim + 1) return false;
    out.assign(n * dim, 0.0f);
    for (int c = 0; c < dim; ++c)
        for (int64_t r = 0; r < n; ++r) out[r * dim + c] = static_cast<float>(V[r * n + c + 1]);
    return finite_all(out);
}

void host_random(int64_t n, int dim, uint64_t seed, float low, float high, HostCoords& out) {
    out.resize(n * dim);
    for (int64_t t = 0; t < n * dim; ++t) {
        const float u = rng_unit_f32(rng_word(seed, static_cast<uint64_t>(t / dim), t % dim));
        out[t] = low + u * (high - low);
    }
}

double host_normal(uint64_t seed, uint64_t a, uint64_t b) {
    double u1 = rng_unit_f64(rng_word(seed, a, 2 * b));
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) *
           std::cos(6.283185307179586 * rng_unit_f64(rng_word(seed, a, 2 * b + 1)));
}

// meta_component_layout_from_centroids (lib.rs:4519-4554)
bool meta_layout(const std::vector<double>& cents, int64_t m, int d, int dim, uint64_t seed,
                 HostCoords& out) {
    if (m == 0) return false;
    if (m == 1) {
        out.assign(dim, 0.0f);
        return true;
    }
    if (m <= 2 * dim) {
        const int64_t k = (m + 1) / 2;
        out.assign(m * dim, 0.0f);
        for (int64_t i = 0; i < m; ++i) out[i * dim + (i % k)] = i < k ? 1.0f : -1.0f;
        return true;
    }
    std::vector<double> aff(m * m, 0.0), deg(m, 0.0);
    for (int64_t i = 0; i < m; ++i) {
        aff[i * m + i] = 1.0;
        for (int64_t j = i + 1; j < m; ++j) {
            double d2 = 0.0;
            for (int f = 0; f < d; ++f) {
                const double dd = cents[i * d + f] - cents[j * d + f];
                d2 += dd * dd;
            }
            const double wv = std::exp(-d2);
            aff[i * m + j] = wv;
            aff[j * m + i] = wv;
        }
    }
    for (int64_t i = 0; i < m; ++i)
        for (int64_t j = 0; j < m; ++j) deg[i] += aff[i * m + j];
    std::vector<double> inv(m), L(m * m, 0.0);
    for (int64_t i = 0; i < m; ++i) inv[i] = deg[i] > 0 ? 1.0 / std::sqrt(deg[i]) : 0.0;
    for (int64_t i = 0; i < m; ++i) L[i * m + i] = 1.0;
    for (int64_t i = 0; i < m; ++i) {
        if (deg[i] <= 0) continue;
        for (int64_t j = 0; j < m; ++j) {
            if (deg[j] <= 0) continue;
            if (aff[i * m + j] > 0.0) L[i * m + j] -= aff[i * m + j] * inv[i] * inv[j];
        }
    }
    std::vector<double> ev, V;
    symmetric_eigen(L, static_cast<int>(m), ev, V);
    if (m <= dim + 1) return false;
    out.assign(m * dim, 0.0f);
    for (int c = 0; c < dim; ++c)
        for (int64_t r = 0; r < m; ++r) out[r * dim + c] = static_cast<float>(V[r * m + c + 1]);
    // noisy_scale_coords(seed ^ 0xC85E7D6ADA318F21, 10, 1e-4)
    float mx = 0.0f;
    for (float v : out) mx = std::max(mx, std::fabs(v));
    const float expansion = mx > 0.0f ? kInitMaxCoord / mx : 1.0f;
    const uint64_t ns = seed ^ 0xC85E7D6ADA318F21ULL;
    for (int64_t r = 0; r < m; ++r)
        for (int c = 0; c < dim; ++c)
            out[r * dim + c] = out[r * dim + c] * expansion +
                               static_cast<float>(kInitNoise * host_normal(ns, r, c));
    return finite_all(out);
}

// Block subspace iteration for every iterative component at once; writes
// the scaled, noised and anchored coordinates of their nodes into `out`.
// Returns false where the reference would return None (an orthonormalisation
// failure or a non-finite result).
template <int S, int SP>
bool run_iterative(const std::vector<int64_t>& it_comps, const std::vector<int64_t>& cstart,
                   const std::vector<int32_t>& order_h, const std::vector<uint64_t>& cseed,
                   const std::vector<float>& data_range, const std::vector<float>& anchors,
                   bool multi, uint64_t seed, int dim, int64_t n, const Graph& g, float* out,
                   cudaStream_t s) {
    const int64_t m = g.n_edges;
    const int64_t n_slots = static_cast<int64_t>(it_comps.size());
    std::vector<int32_t> nodes_h, slot_h;
    std::vector<Chunk> chunks;
    std::vector<uint64_t> slot_seed(n_slots), noise_seed(n_slots);
    std::vector<float> expand_target(n_slots), slot_anchor(n_slots * dim);
    for (int64_t sl = 0; sl < n_slots; ++sl) {
        const int64_t c = it_comps[sl];
        const int32_t base = static_cast<int32_t>(nodes_h.size());
        for (int64_t q = cstart[c]; q < cstart[c + 1]; ++q) {
            nodes_h.push_back(order_h[q]);
            slot_h.push_back(static_cast<int32_t>(sl));
        }
        const int32_t end = static_cast<int32_t>(nodes_h.size());
        for (int32_t st = base; st < end; st += 1024)
            chunks.push_back({static_cast<int32_t>(sl), st, std::min(end, st + 1024)});
        slot_seed[sl] = cseed[c];
        noise_seed[sl] = multi ? seed ^ (static_cast<uint64_t>(c + 1) * 0x94D049BBULL)
                               : seed ^ 0x5DEECE66DULL;
        expand_target[sl] = multi ? data_range[c] : kInitMaxCoord;
        for (int k = 0; k < dim; ++k) slot_anchor[sl * dim + k] = multi ? anchors[c * dim + k] : 0.0f;
    }
    const int64_t cnt = static_cast<int64_t>(nodes_h.size());
    DevBuf<int32_t> nodes(cnt, s), slots(cnt, s), pos(n, s), plen(cnt + 1, s), prow(cnt + 1, s);
    DevBuf<Chunk> dch(chunks.size(), s);
    DevBuf<uint64_t> dseed(n_slots, s), dnseed(n_slots, s);
    UMAPB_CUDA(cudaMemcpyAsync(nodes.get(), nodes_h.data(), cnt * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(slots.get(), slot_h.data(), cnt * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(dch.get(), chunks.data(), chunks.size() * sizeof(Chunk),
                               cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(dseed.get(), slot_seed.data(), n_slots * 8, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(dnseed.get(), noise_seed.data(), n_slots * 8, cudaMemcpyHostToDevice, s));

    // degrees and normalised weights in node space
    DevBuf<double> deg(n, s);
    DevBuf<float> dinvn(n, s), nw(std::max<int64_t>(m, 1), s);
    degree_kernel<<<grid_for(n), 256, 0, s>>>(g.row_ptr.get(), g.weights.get(), n, deg.get(),
                                              dinvn.get());
    UMAPB_LAUNCH_CHECK();
    norm_weight_kernel<<<grid_for(m), 256, 0, s>>>(g.heads.get(), g.tails.get(), g.weights.get(),
                                                   deg.get(), m, nw.get());
    UMAPB_LAUNCH_CHECK();
    // position-ordered CSR
    pos_kernel<<<grid_for(cnt), 256, 0, s>>>(nodes.get(), cnt, pos.get());
    UMAPB_LAUNCH_CHECK();
    prow_len_kernel<<<grid_for(cnt), 256, 0, s>>>(nodes.get(), cnt, g.row_ptr.get(), plen.get());
    UMAPB_LAUNCH_CHECK();
    UMAPB_CUDA(cudaMemsetAsync(plen.get() + cnt, 0, 4, s));
    {
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, plen.get(), prow.get(), cnt + 1, s));
        DevBuf<unsigned char> tmp(tb, s);
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, plen.get(), prow.get(), cnt + 1, s));
    }
    int32_t m_it = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&m_it, prow.get() + cnt, 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    DevBuf<int32_t> ptails(std::max<int32_t>(m_it, 1), s);
    DevBuf<float> pnw(std::max<int32_t>(m_it, 1), s);
    pcsr_kernel<<<grid_for(cnt), 256, 0, s>>>(nodes.get(), cnt, g.row_ptr.get(), g.tails.get(),
                                              nw.get(), pos.get(), prow.get(), ptails.get(), pnw.get());
    UMAPB_LAUNCH_CHECK();

    DevBuf<float> Xb(cnt * SP, s), Yb(cnt * SP, s);
    DevBuf<double> G(n_slots * S * S, s), L(n_slots * S * S, s), dg(n_slots * S, s);
    DevBuf<int> fail(n_slots, s);
    UMAPB_CUDA(cudaMemsetAsync(fail.get(), 0, n_slots * 4, s));
    init_block_kernel<<<grid_for(cnt), 256, 0, s>>>(nodes.get(), cnt, slots.get(), dseed.get(),
                                                    deg.get(), S, SP, Xb.get());
    UMAPB_LAUNCH_CHECK();
    const unsigned nch = static_cast<unsigned>(chunks.size());
    const unsigned gr = grid_for(cnt);
    const unsigned ga = grid_for(cnt, kApplyRows);
    // CholQR2: src -> dst -> src; the orthonormal block ends in src
    auto cholqr = [&](float* src, float* dst) {
        for (int pass = 0; pass < 2; ++pass) {
            float* a = pass == 0 ? src : dst;
            float* b = pass == 0 ? dst : src;
            UMAPB_CUDA(cudaMemsetAsync(G.get(), 0, n_slots * S * S * 8, s));
            gram_kernel<S, SP><<<nch, 256, 0, s>>>(dch.get(), a, a, G.get());
            UMAPB_LAUNCH_CHECK();
            chol_kernel<S><<<static_cast<unsigned>(n_slots), 32, 0, s>>>(G.get(), L.get(), dg.get(),
                                                                        fail.get());
            UMAPB_LAUNCH_CHECK();
            apply_kernel<S, SP><<<ga, kApplyThreads, 0, s>>>(cnt, slots.get(), L.get(), dg.get(), a, b);
            UMAPB_LAUNCH_CHECK();
        }
    };
    const unsigned gr_spmm = static_cast<unsigned>(
        ceil_div(ceil_div(cnt, static_cast<int64_t>(spmm_rows_per_warp<SP>())) * 32, 256));
    auto spmm = [&](const float* x, float* y) {
        spmm_kernel<SP><<<gr_spmm, 256, 0, s>>>(cnt, prow.get(), ptails.get(), pnw.get(), x, y);
        UMAPB_LAUNCH_CHECK();
    };
    static_assert(kIters % kOrthoEvery == 0, "the last product must be orthonormalised");
    cholqr(Xb.get(), Yb.get());
    for (int it = 0; it < kIters; ++it) {
        spmm(Xb.get(), Yb.get());  // Y = (I + A) X
        std::swap(Xb, Yb);
        if ((it + 1) % kOrthoEvery == 0) cholqr(Xb.get(), Yb.get());  // orthonormal in X
    }
    spmm(Xb.get(), Yb.get());
    UMAPB_CUDA(cudaMemsetAsync(G.get(), 0, n_slots * S * S * 8, s));
    gram_kernel<S, SP><<<nch, 256, 0, s>>>(dch.get(), Xb.get(), Yb.get(), G.get());
    UMAPB_LAUNCH_CHECK();
    std::vector<double> G_h(n_slots * S * S);
    std::vector<int> fail_h(n_slots);
    UMAPB_CUDA(cudaMemcpyAsync(G_h.data(), G.get(), G_h.size() * 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(fail_h.data(), fail.get(), n_slots * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    for (int64_t sl = 0; sl < n_slots; ++sl)
        if (fail_h[sl]) return false;  // orthonormalize_columns failed (lib.rs:4262-4273)
    // Rayleigh-Ritz: eigenvectors by descending eigenvalue, skipping the first
    std::vector<double> Vsel(n_slots * S * dim);
    for (int64_t sl = 0; sl < n_slots; ++sl) {
        std::vector<double> R(S * S);
        const double* gs = G_h.data() + sl * S * S;
        for (int i = 0; i < S; ++i)
            for (int j = i; j < S; ++j) {
                R[i * S + j] = gs[i * S + j];
                R[j * S + i] = gs[i * S + j];
            }
        std::vector<double> ev, V;
        symmetric_eigen(R, S, ev, V);
        std::vector<int> ord(S);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return ev[a] > ev[b]; });
        for (int oc = 0; oc < dim; ++oc)
            for (int b = 0; b < S; ++b) Vsel[(sl * S + b) * dim + oc] = V[b * S + ord[oc + 1]];
    }
    DevBuf<double> dV(Vsel.size(), s);
    DevBuf<unsigned> maxbits(n_slots, s);
    UMAPB_CUDA(cudaMemcpyAsync(dV.get(), Vsel.data(), Vsel.size() * 8, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemsetAsync(maxbits.get(), 0, n_slots * 4, s));
    project_kernel<<<gr, 256, 0, s>>>(nodes.get(), cnt, slots.get(), dV.get(), S, SP, dim, Xb.get(),
                                      out, maxbits.get());
    UMAPB_LAUNCH_CHECK();
    std::vector<unsigned> mb(n_slots);
    UMAPB_CUDA(cudaMemcpyAsync(mb.data(), maxbits.get(), n_slots * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    std::vector<float> expansion(n_slots);
    for (int64_t sl = 0; sl < n_slots; ++sl) {
        float mx;
        std::memcpy(&mx, &mb[sl], 4);
        if (!std::isfinite(mx)) return false;
        expansion[sl] = mx > 0.0f ? expand_target[sl] / mx : 1.0f;
    }
    DevBuf<float> dexp(n_slots, s), danch(n_slots * dim, s);
    UMAPB_CUDA(cudaMemcpyAsync(dexp.get(), expansion.data(), n_slots * 4, cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(danch.get(), slot_anchor.data(), n_slots * dim * 4,
                               cudaMemcpyHostToDevice, s));
    finish_kernel<<<gr, 256, 0, s>>>(nodes.get(), cnt, slots.get(), dexp.get(), danch.get(),
                                     dnseed.get(), dim, kInitNoise, out);
    UMAPB_LAUNCH_CHECK();
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return true;
}

}  // namespace

void random_init(int64_t n, int dim, uint64_t seed, float low, float high, float* out,
                 cudaStream_t s) {
    if (n == 0) return;
    random_init_kernel<<<grid_for(n * dim), 256, 0, s>>>(n, dim, seed, low, high, out);
    UMAPB_LAUNCH_CHECK();
}

SpectralResult spectral_init(const float* X, int64_t n, int d, const Graph& g, int dim,
                             uint64_t seed, float* out, cudaStream_t s, const CsrDevice* csr) {
    SpectralResult res;
    const int64_t m = g.n_edges;
    if (n <= dim + 1 || m == 0) return res;
    const int sdim = std::max((dim + 1) * kOversampling, dim + 1);
    if (sdim > kMaxS) invalid("spectral init supports n_components <= 4 on the GPU path");

    // ---- connected components (union-find with atomicMin hooking)
    DevBuf<int32_t> parent(n, s);
    cc_init<<<grid_for(n), 256, 0, s>>>(parent.get(), n);
    UMAPB_LAUNCH_CHECK();
    DevBuf<int> changed(1, s);
    for (int round = 0; round < 64; ++round) {
        UMAPB_CUDA(cudaMemsetAsync(changed.get(), 0, 4, s));
        cc_hook<<<grid_for(m), 256, 0, s>>>(g.heads.get(), g.tails.get(), m, parent.get(),
                                            changed.get());
        UMAPB_LAUNCH_CHECK();
        cc_compress<<<grid_for(n), 256, 0, s>>>(parent.get(), n);
        UMAPB_LAUNCH_CHECK();
        int h = 0;
        UMAPB_CUDA(cudaMemcpyAsync(&h, changed.get(), 4, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
        if (!h) break;
    }
    DevBuf<int32_t> isroot(n, s), rank(n, s), label(n, s), order(n, s), lab_sorted(n, s),
        iota(n, s);
    cc_is_root<<<grid_for(n), 256, 0, s>>>(parent.get(), n, isroot.get());
    UMAPB_LAUNCH_CHECK();
    {
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, isroot.get(), rank.get(), n, s));
        DevBuf<unsigned char> tmp(tb, s);
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, isroot.get(), rank.get(), n, s));
    }
    int32_t last_rank = 0, last_root = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&last_rank, rank.get() + n - 1, 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(&last_root, isroot.get() + n - 1, 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    const int64_t n_comp = static_cast<int64_t>(last_rank) + last_root;
    res.n_components = n_comp;
    cc_label<<<grid_for(n), 256, 0, s>>>(parent.get(), rank.get(), n, label.get());
    UMAPB_LAUNCH_CHECK();
    iota_kernel<<<grid_for(n), 256, 0, s>>>(iota.get(), n);
    UMAPB_LAUNCH_CHECK();
    {
        int bits = 1;
        while ((int64_t(1) << bits) < n_comp + 1) ++bits;
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, label.get(), lab_sorted.get(),
                                                   iota.get(), order.get(), n, 0, bits, s));
        DevBuf<unsigned char> tmp(tb, s);
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, label.get(), lab_sorted.get(),
                                                   iota.get(), order.get(), n, 0, bits, s));
    }
    // component sizes on the host from the sorted labels
    std::vector<int32_t> lab_h(n), order_h;
    UMAPB_CUDA(cudaMemcpyAsync(lab_h.data(), lab_sorted.get(), n * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> cstart(n_comp + 1, 0);
    for (int64_t i = 0; i < n; ++i) cstart[lab_h[i] + 1]++;
    for (int64_t c = 0; c < n_comp; ++c) cstart[c + 1] += cstart[c];

    // ---- decide the path of every component
    enum Kind { kIter, kDense, kRandom };
    std::vector<Kind> kind(n_comp);
    std::vector<uint64_t> cseed(n_comp);
    const bool multi = n_comp > 1;
    for (int64_t c = 0; c < n_comp; ++c) {
        const int64_t sz = cstart[c + 1] - cstart[c];
        if (!multi) {
            const int64_t thr = d <= 8 ? 2049 : 0;  // spectral_iterative_connected_threshold
            kind[c] = (sz >= thr && sz > sdim) ? kIter : kDense;
            cseed[c] = seed;
        } else {
            if (sz < 2 * dim || sz <= dim + 1)
                kind[c] = kRandom;
            else
                kind[c] = (sz >= kComponentIterThreshold && sz > sdim) ? kIter : kDense;
            cseed[c] = seed ^ (static_cast<uint64_t>(c + 1) * 0xBF58476D1CE4E5B9ULL);
        }
    }
    if (!multi && kind[0] == kDense && n > kDenseFallbackMax && n >= (d <= 8 ? 2049 : 0))
        return res;

    // ---- meta layout (anchors) and per-component ranges
    std::vector<float> anchors(n_comp * dim, 0.0f), data_range(n_comp, 1.0f);
    if (multi) {
        std::vector<double> cents;
        if (n_comp > 2 * dim) {
            std::vector<Chunk> chunks;
            for (int64_t c = 0; c < n_comp; ++c)
                for (int64_t st = cstart[c]; st < cstart[c + 1]; st += 4096)
                    chunks.push_back({static_cast<int32_t>(c), static_cast<int32_t>(st),
                                      static_cast<int32_t>(std::min(cstart[c + 1], st + 4096))});
            DevBuf<Chunk> dch(chunks.size(), s);
            DevBuf<double> dcent(n_comp * d, s);
            UMAPB_CUDA(cudaMemcpyAsync(dch.get(), chunks.data(), chunks.size() * sizeof(Chunk),
                                       cudaMemcpyHostToDevice, s));
            UMAPB_CUDA(cudaMemsetAsync(dcent.get(), 0, n_comp * d * 8, s));
            if (csr)
                centroid_csr_kernel<<<static_cast<unsigned>(chunks.size()), 128, 0, s>>>(
                    dch.get(), order.get(), csr->indptr.get(), csr->indices.get(),
                    csr->values.get(), d, dcent.get());
            else
                centroid_kernel<<<static_cast<unsigned>(chunks.size()), 128, 0, s>>>(
                    dch.get(), order.get(), X, d, dcent.get());
            UMAPB_LAUNCH_CHECK();
            cents.resize(n_comp * d);
            UMAPB_CUDA(cudaMemcpyAsync(cents.data(), dcent.get(), n_comp * d * 8,
                                       cudaMemcpyDeviceToHost, s));
            UMAPB_CUDA(cudaStreamSynchronize(s));
            for (int64_t c = 0; c < n_comp; ++c) {
                const double sc = 1.0 / static_cast<double>(cstart[c + 1] - cstart[c]);
                for (int f = 0; f < d; ++f) cents[c * d + f] *= sc;
            }
        }
        HostCoords layout;
        if (!meta_layout(cents, n_comp, d, dim, seed ^ 0xA13F52A92D4CB801ULL, layout)) return res;
        anchors = layout;
        for (int64_t c = 0; c < n_comp; ++c) {
            float r = INFINITY;
            for (int64_t o = 0; o < n_comp; ++o) {
                if (o == c) continue;
                float d2 = 0.0f;
                for (int k = 0; k < dim; ++k) {
                    const float df = anchors[c * dim + k] - anchors[o * dim + k];
                    d2 += df * df;
                }
                const float dist = std::sqrt(d2);
                if (dist > 0.0f) r = std::min(r, dist / 2.0f);
            }
            if (!std::isfinite(r) || r <= 0.0f) r = 1.0f;
            data_range[c] = r;
        }
    }

    // ---- host components (dense spectral / random)
    bool need_host_graph = false;
    for (int64_t c = 0; c < n_comp; ++c) need_host_graph |= kind[c] == kDense;
    std::vector<int32_t> rp_h, tl_h;
    std::vector<float> w_h;
    if (need_host_graph) {
        rp_h.resize(n + 1);
        tl_h.resize(m);
        w_h.resize(m);
        order_h.resize(n);
        UMAPB_CUDA(cudaMemcpyAsync(rp_h.data(), g.row_ptr.get(), (n + 1) * 4, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaMemcpyAsync(tl_h.data(), g.tails.get(), m * 4, cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaMemcpyAsync(w_h.data(), g.weights.get(), m * 4, cudaMemcpyDeviceToHost, s));
    }
    if (order_h.empty()) order_h.resize(n);
    UMAPB_CUDA(cudaMemcpyAsync(order_h.data(), order.get(), n * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));

    std::vector<int32_t> host_nodes;
    std::vector<float> host_vals;
    std::vector<int64_t> local_of(need_host_graph ? n : 0, -1);
    for (int64_t c = 0; c < n_comp; ++c) {
        if (kind[c] == kIter) continue;
        const int64_t sz = cstart[c + 1] - cstart[c];
        HostCoords local;
        if (kind[c] == kRandom) {
            host_random(sz, dim, seed ^ (static_cast<uint64_t>(c + 1) * 0x9E3779B9ULL),
                        -data_range[c], data_range[c], local);
        } else {
            for (int64_t li = 0; li < sz; ++li) local_of[order_h[cstart[c] + li]] = li;
            std::vector<std::array<int64_t, 2>> pairs;
            std::vector<float> pw;
            for (int64_t li = 0; li < sz; ++li) {
                const int64_t node = order_h[cstart[c] + li];
                for (int32_t e = rp_h[node]; e < rp_h[node + 1]; ++e) {
                    pairs.push_back({li, local_of[tl_h[e]]});
                    pw.push_back(w_h[e]);
                }
            }
            if (!dense_spectral(sz, dim, pairs, pw, local)) return res;
            float mx = 0.0f;
            for (float v : local) mx = std::max(mx, std::fabs(v));
            const float target = multi ? data_range[c] : kInitMaxCoord;
            const float expansion = mx > 0.0f ? target / mx : 1.0f;
            const uint64_t ns = multi ? seed ^ (static_cast<uint64_t>(c + 1) * 0x94D049BBULL)
                                      : seed ^ 0x5DEECE66DULL;
            for (int64_t li = 0; li < sz; ++li)
                for (int k = 0; k < dim; ++k)
                    local[li * dim + k] = local[li * dim + k] * expansion +
                                          static_cast<float>(kInitNoise * host_normal(ns, li, k));
        }
        for (int64_t li = 0; li < sz; ++li) {
            host_nodes.push_back(order_h[cstart[c] + li]);
            for (int k = 0; k < dim; ++k)
                host_vals.push_back(local[li * dim + k] + (multi ? anchors[c * dim + k] : 0.0f));
        }
    }
    if (!host_nodes.empty()) {
        const int64_t cnt = static_cast<int64_t>(host_nodes.size());
        DevBuf<int32_t> hn(cnt, s);
        DevBuf<float> hv(cnt * dim, s);
        UMAPB_CUDA(cudaMemcpyAsync(hn.get(), host_nodes.data(), cnt * 4, cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(hv.get(), host_vals.data(), cnt * dim * 4, cudaMemcpyHostToDevice, s));
        scatter_rows_kernel<<<grid_for(cnt * dim), 256, 0, s>>>(hn.get(), cnt, dim, hv.get(), out);
        UMAPB_LAUNCH_CHECK();
        UMAPB_CUDA(cudaStreamSynchronize(s));
    }

    // ---- iterative components on the device
    std::vector<int64_t> it_comps;
    for (int64_t c = 0; c < n_comp; ++c)
        if (kind[c] == kIter) it_comps.push_back(c);
    if (!it_comps.empty()) {
        bool ok = false;
        switch (sdim) {
            case 12: ok = run_iterative<12, 12>(it_comps, cstart, order_h, cseed, data_range, anchors,
                                               multi, seed, dim, n, g, out, s); break;
            case 18: ok = run_iterative<18, 20>(it_comps, cstart, order_h, cseed, data_range, anchors,
                                               multi, seed, dim, n, g, out, s); break;
            case 24: ok = run_iterative<24, 24>(it_comps, cstart, order_h, cseed, data_range, anchors,
                                               multi, seed, dim, n, g, out, s); break;
            case 30: ok = run_iterative<30, 32>(it_comps, cstart, order_h, cseed, data_range, anchors,
                                               multi, seed, dim, n, g, out, s); break;
            default: invalid("unsupported spectral block width");
        }
        if (!ok) return res;
    }
    res.used_spectral = true;
    return res;
}

}  // namespace umapb
