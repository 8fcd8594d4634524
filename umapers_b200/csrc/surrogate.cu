// surrogate.cu - learned transform surrogate: a BF16 MLP trained on the GPU
// to map rows straight to the fitted embedding, with a per-row gate that
// sends rows it cannot vouch for to the plain transform.
//
// The reference has no such component; its transform is
// UmapModel::transform_dense (rust_umap/src/lib.rs:1593-1685), and its
// separate ParametricUmapModel (rust_umap/src/parametric.rs:89-534) sets the
// precedent of distilling a fitted embedding into a network over
// standardised inputs (parametric.rs:634-707, same mean / scale rule).
//
// Network: x (n_features, standardised, zero-padded to dp = round_up(., 128))
//   Z1 = X W1^T + b1, A1 = bf16(gelu(Z1))          hidden
//   Z2 = A1 W2^T + b2, A2 = bf16(gelu(Z2))         hidden
//   Y  = shift + scale * (A2 W3^T + b3)            n_out (FP32)
// where shift / scale are the fitted embedding's per-axis mean and std.
// The two hidden layers and every weight gradient run on tcgen05 tensor
// cores (gemm_tc.cu) with FP32 accumulation; the n_out-wide head, the loss
// and the reductions run on CUDA cores in FP32.  Master weights and Adam
// moments are FP32; BF16 copies of W1, W2 and W2^T feed the GEMMs.
//
// Loss per batch of B rows (the gradient is the UMAP SGD form):
//   mse_w * |y_i - e_i|^2
//   + edge_w * sum_j w_ij * log(1 + a d_ij^(2b))             (fuzzy edges of i)
//   + edge_w * sum_s rep_w * (-log(1 - q))                   (negative samples)
// with d the distance from y_i to the fitted position of the other end,
// q = 1 / (1 + a d^(2b)), rep_w = neg_scale * sum_j w_ij / n_neg, and per
// pair gradient coefficients 2ab d^(2b-2) / (1 + a d^(2b)) (attractive,
// rust_umap/src/lib.rs:5170, 5193-5194) and
// -2b / ((0.001 + d^2)(1 + a d^(2b))) (repulsive), each coordinate clipped to
// [-4, 4] as in clip (rust_umap/src/lib.rs:4962-4964); everything over B.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <vector>

#include "kernels.cuh"

namespace umapb {

namespace {

constexpr float kScaleEps = 1e-6f;  // parametric.rs:6
constexpr float kBeta1 = 0.9f, kBeta2 = 0.999f, kAdamEps = 1e-8f;
constexpr int64_t kInferChunk = 1 << 20;  // rows per inference pass
constexpr double kCellPrior = 10.0;        // pseudo-rows of the gate's cell smoothing

__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ float clip4(float v) { return fminf(fmaxf(v, -4.0f), 4.0f); }

int grid_for(int64_t n, int block = 256) { return static_cast<int>(ceil_div(n, block)); }

// ------------------------------------------------------------ kernels ---

// Per-block column sums and sums of squares (FP64) over a range of rows.
__global__ void col_stats_kernel(const float* __restrict__ X, int64_t n, int d,
                                 int64_t rows_per_block, double* __restrict__ part) {
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * rows_per_block;
    const int64_t r1 = min(n, r0 + rows_per_block);
    for (int f = threadIdx.x; f < d; f += blockDim.x) {
        double s = 0.0, ss = 0.0;
        for (int64_t r = r0; r < r1; ++r) {
            const double v = X[r * d + f];
            s += v;
            ss += v * v;
        }
        part[static_cast<int64_t>(blockIdx.x) * 2 * d + f] = s;
        part[static_cast<int64_t>(blockIdx.x) * 2 * d + d + f] = ss;
    }
}

// out[r][f] = bf16((X[src][f] - mean[f]) / scale[f]) for f < d, 0 up to dp;
// src = ids ? ids[r] : r.  Optional transposed copy out_t[f][r] (ld ld_t).
// One block stages a 32 x 32 tile so both layouts are written coalesced.
__global__ void standardize_kernel(const float* __restrict__ X, int d,
                                   const int32_t* __restrict__ ids, int64_t rows,
                                   const float* __restrict__ mean,
                                   const float* __restrict__ scale, int dp,
                                   __nv_bfloat16* __restrict__ out,
                                   __nv_bfloat16* __restrict__ out_t, int64_t ld_t) {
    __shared__ float tile[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 32;
    const int f = blockIdx.x * 32 + tx;
    for (int i = ty; i < 32; i += 8) {
        const int64_t r = r0 + i;
        float v = 0.0f;
        if (r < rows) {
            const int64_t src = ids ? ids[r] : r;
            if (f < d) v = (X[src * d + f] - mean[f]) / scale[f];
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            out[r * dp + f] = h;
            v = __bfloat162float(h);
        }
        tile[i][tx] = v;
    }
    if (!out_t) return;
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
        const int fo = blockIdx.x * 32 + i;
        const int64_t r = r0 + tx;
        if (r < rows) out_t[fo * ld_t + r] = __float2bfloat16_rn(tile[tx][i]);
    }
}

// standardize_kernel's row-major output alone, one thread per 8 output
// columns of a row: 16-byte loads of a 16-byte aligned X (d % 4 == 0) and
// one 16-byte store, the same arithmetic per element.
__global__ void standardize_rows_kernel(const float* __restrict__ X, int d,
                                        const int32_t* __restrict__ ids, int64_t rows,
                                        const float* __restrict__ mean,
                                        const float* __restrict__ scale, int dp,
                                        __nv_bfloat16* __restrict__ out) {
    const int groups = dp >> 3;
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= rows * groups) return;
    const int64_t r = t / groups;
    const int c0 = static_cast<int>(t - r * groups) * 8;
    const int64_t src = ids ? ids[r] : r;
    const float* x = X + src * d;
    float v[8];
    if (c0 + 8 <= d) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(x + c0));
        const float4 b = __ldg(reinterpret_cast<const float4*>(x + c0 + 4));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = c0 + i < d ? x[c0 + i] : 0.0f;
    }
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int f = c0 + i;
        h[i] = __float2bfloat16_rn(f < d ? __fdiv_rn(__fsub_rn(v[i], mean[f]), scale[f]) : 0.0f);
    }
    *reinterpret_cast<uint4*>(out + r * dp + c0) = *reinterpret_cast<const uint4*>(h);
}

// Squared norm of each bf16 row (warp per row, fixed summation order).
__global__ void row_sq_bf16_kernel(const __nv_bfloat16* __restrict__ M, int64_t rows, int cols,
                                   float* __restrict__ out) {
    const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    float s = 0.0f;
    for (int c = lane; c < cols; c += 32) {
        const float v = __bfloat162float(M[r * cols + c]);
        s = fmaf(v, v, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[r] = s;
}

struct LossArgs {
    const float* head_part;  // [n_tiles][B][dout]
    int n_tiles;
    const float* b3;
    const float* out_shift;  // y = out_shift + out_scale * (network output)
    const float* out_scale;
    int dout;
    int64_t B;
    const int32_t* ids;      // batch position -> row id (nullable: identity)
    const float* targets;    // [rows x dout], indexed by row id
    const float* teacher;    // [n_teacher x dout]
    int64_t n_teacher;
    const int32_t* row_ptr;  // CSR over row ids
    const int32_t* tails;
    const float* weights;
    const int32_t* neg_ids;  // [B x n_neg] (nullable: drawn from the counter RNG)
    int n_neg;
    uint64_t seed;
    uint64_t step;
    float a, b, mse_w, edge_w, neg_scale;
    float* y_out;            // [B x dout] (nullable)
    float* dY;               // [B x dout]
    double* loss_acc;        // (nullable) += batch mean loss
};

__global__ void loss_kernel(LossArgs p) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    float y[kGemmMaxHead], g[kGemmMaxHead];
    for (int o = 0; o < p.dout; ++o) {
        float s = p.b3[o];
        for (int t = 0; t < p.n_tiles; ++t) s += p.head_part[(t * p.B + i) * p.dout + o];
        y[o] = p.out_shift[o] + p.out_scale[o] * s;
    }
    const int64_t row = p.ids ? p.ids[i] : i;
    const float inv_b = 1.0f / static_cast<float>(p.B);
    double loss = 0.0;
    for (int o = 0; o < p.dout; ++o) {
        const float r = y[o] - p.targets[row * p.dout + o];
        g[o] = 2.0f * p.mse_w * inv_b * r;
        loss += static_cast<double>(p.mse_w) * r * r;
    }
    float wsum = 0.0f;
    const float ce = p.edge_w * inv_b;
    for (int32_t e = p.row_ptr[row]; e < p.row_ptr[row + 1]; ++e) {
        const int64_t j = p.tails[e];
        const float w = p.weights[e];
        wsum += w;
        float diff[kGemmMaxHead], d2 = 0.0f;
        for (int o = 0; o < p.dout; ++o) {
            diff[o] = y[o] - p.teacher[j * p.dout + o];
            d2 += diff[o] * diff[o];
        }
        if (d2 > 0.0f) {
            const float db = powf(d2, p.b);
            const float c = 2.0f * p.a * p.b * db / (d2 * (1.0f + p.a * db));
            for (int o = 0; o < p.dout; ++o) g[o] += ce * w * clip4(c * diff[o]);
            loss += static_cast<double>(p.edge_w) * w * log1p(static_cast<double>(p.a) * db);
        }
    }
    const float rep_w = p.n_neg > 0 ? p.neg_scale * wsum / static_cast<float>(p.n_neg) : 0.0f;
    for (int s = 0; s < p.n_neg; ++s) {
        const int64_t j =
            p.neg_ids ? p.neg_ids[i * p.n_neg + s]
                      : rng_below(rng_word(p.seed, p.step * static_cast<uint64_t>(p.B) + i, s),
                                  static_cast<uint32_t>(p.n_teacher));
        float diff[kGemmMaxHead], d2 = 0.0f;
        for (int o = 0; o < p.dout; ++o) {
            diff[o] = y[o] - p.teacher[j * p.dout + o];
            d2 += diff[o] * diff[o];
        }
        const float db = d2 > 0.0f ? powf(d2, p.b) : 0.0f;
        const float c = -2.0f * p.b / ((0.001f + d2) * (1.0f + p.a * db));
        for (int o = 0; o < p.dout; ++o) g[o] += ce * rep_w * clip4(c * diff[o]);
        loss += static_cast<double>(p.edge_w) * rep_w *
                log1p(1.0 / (static_cast<double>(p.a) * db + 1e-6));
    }
    for (int o = 0; o < p.dout; ++o) {
        p.dY[i * p.dout + o] = g[o] * p.out_scale[o];  // gradient at the network's output
        if (p.y_out) p.y_out[i * p.dout + o] = y[o];
    }
    if (p.loss_acc) atomicAdd(p.loss_acc, loss / static_cast<double>(p.B));
}

// dZ2[i][h] = (sum_o dY[i][o] W3[o][h]) * gelu'(Z2[i][h]), written as bf16
// row-major and transposed (ld B) through a 32 x 32 shared tile.
__global__ void head_backward_kernel(const float* __restrict__ dY, int dout,
                                     const float* __restrict__ W3, const float* __restrict__ Z2,
                                     int64_t B, int H, __nv_bfloat16* __restrict__ dZ2,
                                     __nv_bfloat16* __restrict__ dZ2T) {
    __shared__ float tile[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = static_cast<int64_t>(blockIdx.y) * 32;
    const int h = blockIdx.x * 32 + tx;
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = i0 + r;
        float s = 0.0f;
        for (int o = 0; o < dout; ++o) s = fmaf(dY[i * dout + o], W3[o * H + h], s);
        const __nv_bfloat16 v = __float2bfloat16_rn(s * gelu_grad(Z2[i * H + h]));
        dZ2[i * H + h] = v;
        tile[r][tx] = __bfloat162float(v);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int ho = blockIdx.x * 32 + r;
        dZ2T[static_cast<int64_t>(ho) * B + i0 + tx] = __float2bfloat16_rn(tile[tx][r]);
    }
}

// out[r] = sum_c M[r][c] (bf16 in, FP32 sum; warp per row, fixed order).
__global__ void rowsum_bf16_kernel(const __nv_bfloat16* __restrict__ M, int64_t rows, int64_t cols,
                                   float* __restrict__ out) {
    const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    float s = 0.0f;
    for (int64_t c = lane; c < cols; c += 32) s += __bfloat162float(M[r * cols + c]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[r] = s;
}

// dW3[o][h] = sum_i dY[i][o] A2[i][h]; db3[o] = sum_i dY[i][o].  A block owns
// 32 columns; its 8 thread rows split the batch and are summed in order.
__global__ void head_grad_kernel(const float* __restrict__ dY, int dout,
                                 const __nv_bfloat16* __restrict__ A2, int64_t B, int H,
                                 float* __restrict__ dW3, float* __restrict__ db3) {
    __shared__ float red[kGemmMaxHead][8][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int h = blockIdx.x * 32 + tx;
    float acc[kGemmMaxHead] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int64_t i = ty; i < B; i += 8) {
        const float a = __bfloat162float(A2[i * H + h]);
        for (int o = 0; o < dout; ++o) acc[o] = fmaf(dY[i * dout + o], a, acc[o]);
    }
    for (int o = 0; o < dout; ++o) red[o][ty][tx] = acc[o];
    __syncthreads();
    if (ty == 0) {
        for (int o = 0; o < dout; ++o) {
            float s = 0.0f;
            for (int r = 0; r < 8; ++r) s += red[o][r][tx];
            dW3[o * H + h] = s;
        }
    }
    if (blockIdx.x == 0 && ty == 1) {
        for (int o = 0; o < dout; ++o) {
            float s = 0.0f;
            for (int64_t i = tx; i < B; i += 32) s += dY[i * dout + o];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            if (tx == 0) db3[o] = s;
        }
    }
}

struct Layout {
    int64_t din = 0, dp = 0, H = 0, dout = 0;
    int64_t w1 = 0, b1 = 0, w2 = 0, b2 = 0, w3 = 0, b3 = 0, total = 0;
    void set(int64_t in, int64_t hidden, int64_t out) {
        din = in;
        dp = ceil_div(in, 128) * 128;
        H = hidden;
        dout = out;
        w1 = 0;
        b1 = w1 + H * dp;
        w2 = b1 + H;
        b2 = w2 + H * H;
        w3 = b2 + H;
        b3 = w3 + dout * H;
        total = b3 + dout;
    }
};

// Adam (bias-corrected, epsilon outside the square root) on the flat master
// vector when `update`, then the BF16 copies of W1, W2 and W2^T.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, Layout L, float lr,
                            float bc1, float bc2, int update, __nv_bfloat16* __restrict__ w1b,
                            __nv_bfloat16* __restrict__ w2b, __nv_bfloat16* __restrict__ w2bt) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= L.total) return;
    float wi = w[i];
    if (update) {
        const float gi = g[i];
        const float mi = kBeta1 * m[i] + (1.0f - kBeta1) * gi;
        const float vi = kBeta2 * v[i] + (1.0f - kBeta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        wi -= lr * (mi / bc1) / (sqrtf(vi / bc2) + kAdamEps);
        w[i] = wi;
    }
    if (i < L.b1) {
        w1b[i] = __float2bfloat16_rn(wi);
    } else if (i >= L.w2 && i < L.b2) {
        const int64_t k = i - L.w2;
        const __nv_bfloat16 h = __float2bfloat16_rn(wi);
        w2b[k] = h;
        w2bt[(k % L.H) * L.H + k / L.H] = h;
    }
}

// Network output and gate decision of each row.
struct FinishArgs {
    const float* head_part;  // [n_tiles][rows][dout]
    int n_tiles;
    const float* b3;
    const float* out_shift;
    const float* out_scale;
    int dout;
    int64_t rows;
    const float* amin_val;   // [a_tiles][rows]
    const int32_t* amin_idx;
    int a_tiles;
    const float* row_sq;
    const float* anchor_r2;  // [n_anchors] (nullable: no gate)
    const uint8_t* cell_ok;
    float* out;              // [rows x dout]
    uint8_t* flags;          // (nullable) 1 = plain path
    int32_t* anchor_of;      // (nullable)
    float* anchor_d2;        // (nullable)
};

__global__ void finish_kernel(FinishArgs p) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= p.rows) return;
    if (p.out) {
        for (int o = 0; o < p.dout; ++o) {
            float s = p.b3[o];
            for (int t = 0; t < p.n_tiles; ++t) s += p.head_part[(t * p.rows + r) * p.dout + o];
            p.out[r * p.dout + o] = p.out_shift[o] + p.out_scale[o] * s;
        }
    }
    if (p.a_tiles == 0) return;
    float best = INFINITY;
    int32_t bi = 0;
    for (int t = 0; t < p.a_tiles; ++t) {
        const float v = p.amin_val[t * p.rows + r];
        if (v < best) {
            best = v;
            bi = p.amin_idx[t * p.rows + r];
        }
    }
    const float d2 = fmaxf(p.row_sq[r] + best, 0.0f);
    if (p.anchor_of) p.anchor_of[r] = bi;
    if (p.anchor_d2) p.anchor_d2[r] = d2;
    if (p.flags) p.flags[r] = (p.cell_ok[bi] != 0 && d2 <= p.anchor_r2[bi]) ? 0 : 1;
}

// Number of non-zero flags (integer atomics: the count does not depend on
// the order).
__global__ void count_flags_kernel(const uint8_t* __restrict__ flags, int64_t n,
                                   unsigned long long* __restrict__ count) {
    unsigned long long c = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        c += flags[i] != 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

__global__ void gather_rows_kernel(const float* __restrict__ src, const int32_t* __restrict__ ids,
                                   int64_t n, int d, float* __restrict__ dst) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * d) return;
    const int64_t r = t / d, c = t - r * d;
    dst[t] = src[static_cast<int64_t>(ids[r]) * d + c];
}

__global__ void scatter_rows_kernel(const float* __restrict__ src, const int32_t* __restrict__ ids,
                                    int64_t n, int d, float* __restrict__ dst) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * d) return;
    const int64_t r = t / d, c = t - r * d;
    dst[static_cast<int64_t>(ids[r]) * d + c] = src[t];
}

}  // namespace

void gather_rows(const float* src, const int32_t* ids, int64_t n, int d, float* dst,
                 cudaStream_t s) {
    if (n == 0) return;
    gather_rows_kernel<<<grid_for(n * d), 256, 0, s>>>(src, ids, n, d, dst);
    UMAPB_LAUNCH_CHECK();
}

void scatter_rows(const float* src, const int32_t* ids, int64_t n, int d, float* dst,
                  cudaStream_t s) {
    if (n == 0) return;
    scatter_rows_kernel<<<grid_for(n * d), 256, 0, s>>>(src, ids, n, d, dst);
    UMAPB_LAUNCH_CHECK();
}

int64_t select_flagged(const uint8_t* flags, int64_t n, int32_t* ids, cudaStream_t s) {
    if (n == 0) return 0;
    if (n > 0x7FFFFFFFll) invalid("select_flagged: too many rows");
    cub::CountingInputIterator<int32_t> it(0);
    DevBuf<int32_t> cnt(1, s);
    size_t bytes = 0;
    cub::DeviceSelect::Flagged(nullptr, bytes, it, flags, ids, cnt.get(), static_cast<int>(n), s);
    DevBuf<uint8_t> tmp(bytes, s);
    cub::DeviceSelect::Flagged(tmp.get(), bytes, it, flags, ids, cnt.get(), static_cast<int>(n),
                               s);
    UMAPB_CUDA(cudaGetLastError());
    int32_t h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, cnt.get(), 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return h;
}

// ------------------------------------------------------------- model ---
struct Surrogate {
    Layout L;
    DevBuf<float> mean, scale;          // input standardisation
    DevBuf<float> out_shift, out_scale;  // output affine: the embedding's mean and std
    DevBuf<float> params;
    DevBuf<__nv_bfloat16> w1b, w2b, w2bt;
    int64_t n_anchors = 0;
    DevBuf<__nv_bfloat16> anchors;
    DevBuf<float> anchor_sq, anchor_r2;
    DevBuf<uint8_t> cell_ok;
    float radius = 0.0f;
};

void SurrogateDeleter::operator()(Surrogate* s) const { delete s; }

namespace {

// Scratch of one forward (+ backward) pass over `rows` rows.
struct Pass {
    int64_t rows = 0;
    DevBuf<__nv_bfloat16> X, XT, A1, A1T, A2, dZ2, dZ2T, dZ1T;
    DevBuf<float> Z1, Z2, part, dY, y;
    void alloc(const Layout& L, int64_t n, bool train, cudaStream_t s) {
        rows = n;
        X.alloc(n * L.dp, s);
        A1.alloc(n * L.H, s);
        part.alloc((L.H / 128) * n * L.dout, s);
        if (train) {
            XT.alloc(L.dp * n, s);
            A1T.alloc(L.H * n, s);
            A2.alloc(n * L.H, s);
            dZ2.alloc(n * L.H, s);
            dZ2T.alloc(L.H * n, s);
            dZ1T.alloc(L.H * n, s);
            Z1.alloc(n * L.H, s);
            Z2.alloc(n * L.H, s);
            dY.alloc(n * L.dout, s);
            y.alloc(n * L.dout, s);
        }
    }
};

void standardize(const float* X, int d, const int32_t* ids, int64_t rows, const float* mean,
                 const float* scale, int dp, __nv_bfloat16* out, __nv_bfloat16* out_t,
                 int64_t ld_t, cudaStream_t s) {
    if (rows == 0) return;
    if (!out_t && d % 4 == 0 && dp % 8 == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0 &&
        (reinterpret_cast<uintptr_t>(out) & 15) == 0) {
        const int64_t threads = rows * (dp / 8);
        standardize_rows_kernel<<<static_cast<unsigned>(ceil_div(threads, 256)), 256, 0, s>>>(
            X, d, ids, rows, mean, scale, dp, out);
        UMAPB_LAUNCH_CHECK();
        return;
    }
    if (ceil_div(rows, 32) > 65535) invalid("standardize: too many rows in one pass");
    const dim3 grid(static_cast<unsigned>(dp / 32), static_cast<unsigned>(ceil_div(rows, 32)));
    standardize_kernel<<<grid, dim3(32, 8), 0, s>>>(X, d, ids, rows, mean, scale, dp, out, out_t,
                                                    ld_t);
    UMAPB_LAUNCH_CHECK();
}

// Forward pass over P.rows rows already standardised into P.X; leaves the
// head partial sums in P.part.  Training also keeps Z1, Z2, A1^T, A2.
void forward(const Surrogate& sg, Pass& P, bool train, cudaStream_t s) {
    const Layout& L = sg.L;
    const float* w = sg.params.get();
    GemmOut o1;
    o1.bias = w + L.b1;
    o1.act = P.A1.get();
    if (train) {
        o1.z = P.Z1.get();
        o1.act_t = P.A1T.get();
        o1.ld_t = P.rows;
    }
    gemm_bf16_tn(P.X.get(), sg.w1b.get(), P.rows, L.H, L.dp, kEpiBiasGelu, o1, s);
    GemmOut o2;
    o2.bias = w + L.b2;
    o2.head_w = w + L.w3;
    o2.head_dim = static_cast<int>(L.dout);
    o2.head_part = P.part.get();
    if (train) {
        o2.z = P.Z2.get();
        o2.act = P.A2.get();
    }
    gemm_bf16_tn(P.A1.get(), sg.w2b.get(), P.rows, L.H, L.H, kEpiBiasGeluHead, o2, s);
}

// Backward pass from P.dY into the flat gradient vector `grad`.
void backward(const Surrogate& sg, Pass& P, float* grad, cudaStream_t s) {
    const Layout& L = sg.L;
    const float* w = sg.params.get();
    const int64_t B = P.rows;
    head_backward_kernel<<<dim3(static_cast<unsigned>(L.H / 32), static_cast<unsigned>(B / 32)),
                           dim3(32, 8), 0, s>>>(P.dY.get(), static_cast<int>(L.dout), w + L.w3,
                                                P.Z2.get(), B, static_cast<int>(L.H), P.dZ2.get(),
                                                P.dZ2T.get());
    UMAPB_LAUNCH_CHECK();
    // dZ1 = (dZ2 W2) * gelu'(Z1), kept transposed for dW1 and db1
    GemmOut ob;
    ob.z_in = P.Z1.get();
    ob.act_t = P.dZ1T.get();
    ob.ld_t = B;
    gemm_bf16_tn(P.dZ2.get(), sg.w2bt.get(), B, L.H, L.H, kEpiGeluBwd, ob, s);
    GemmOut og2;
    og2.c = grad + L.w2;
    gemm_bf16_tn(P.dZ2T.get(), P.A1T.get(), L.H, L.H, B, kEpiF32, og2, s);
    GemmOut og1;
    og1.c = grad + L.w1;
    gemm_bf16_tn(P.dZ1T.get(), P.XT.get(), L.H, L.dp, B, kEpiF32, og1, s);
    rowsum_bf16_kernel<<<grid_for(L.H * 32), 256, 0, s>>>(P.dZ1T.get(), L.H, B, grad + L.b1);
    UMAPB_LAUNCH_CHECK();
    rowsum_bf16_kernel<<<grid_for(L.H * 32), 256, 0, s>>>(P.dZ2T.get(), L.H, B, grad + L.b2);
    UMAPB_LAUNCH_CHECK();
    head_grad_kernel<<<static_cast<unsigned>(L.H / 32), dim3(32, 8), 0, s>>>(
        P.dY.get(), static_cast<int>(L.dout), P.A2.get(), B, static_cast<int>(L.H), grad + L.w3,
        grad + L.b3);
    UMAPB_LAUNCH_CHECK();
}

void adam_step(Surrogate& sg, const float* grad, float* m, float* v, int64_t t, float lr,
               bool update, cudaStream_t s) {
    const float bc1 = update ? 1.0f - std::pow(kBeta1, static_cast<float>(t)) : 1.0f;
    const float bc2 = update ? 1.0f - std::pow(kBeta2, static_cast<float>(t)) : 1.0f;
    adam_kernel<<<grid_for(sg.L.total), 256, 0, s>>>(sg.params.get(), grad, m, v, sg.L, lr, bc1,
                                                      bc2, update ? 1 : 0, sg.w1b.get(),
                                                      sg.w2b.get(), sg.w2bt.get());
    UMAPB_LAUNCH_CHECK();
}

void alloc_network(Surrogate& sg, cudaStream_t s) {
    sg.params.alloc(sg.L.total, s);
    sg.w1b.alloc(sg.L.H * sg.L.dp, s);
    sg.w2b.alloc(sg.L.H * sg.L.H, s);
    sg.w2bt.alloc(sg.L.H * sg.L.H, s);
}

void check_gemm(cudaStream_t s) {
    const int e = gemm_take_error(s);
    if (e != 0)
        throw Error(UMAPB_ERR_CUDA,
                    "tensor-core GEMM stopped on a wait timeout (code " + std::to_string(e) + ")");
}

// Glorot-uniform weights (parametric.rs:190-208 uses the same limit), zero
// biases, from the counter RNG.
std::vector<float> init_params(const Layout& L, uint64_t seed) {
    std::vector<float> w(L.total, 0.0f);
    auto fill = [&](int64_t off, int64_t rows, int64_t cols, int64_t ld, int64_t fan_in,
                    uint64_t stream) {
        const double lim = std::sqrt(6.0 / static_cast<double>(fan_in + rows));
        for (int64_t r = 0; r < rows; ++r)
            for (int64_t c = 0; c < cols; ++c)
                w[off + r * ld + c] = static_cast<float>(
                    (2.0 * rng_unit_f64(rng_word(seed, stream, r * cols + c)) - 1.0) * lim);
    };
    fill(L.w1, L.H, L.din, L.dp, L.din, 101);
    fill(L.w2, L.H, L.H, L.H, L.H, 102);
    fill(L.w3, L.dout, L.H, L.H, L.H, 103);
    return w;
}

// Mean and scale of each feature over all rows (parametric.rs:652-675
// rule: scale = std when std > 1e-6, else 1).
void feature_stats(const float* X, int64_t n, int d, std::vector<float>& mean,
                   std::vector<float>& scale, cudaStream_t s) {
    const int64_t blocks = std::min<int64_t>(1024, std::max<int64_t>(1, ceil_div(n, 256)));
    const int64_t rpb = ceil_div(n, blocks);
    DevBuf<double> part(blocks * 2 * d, s);
    col_stats_kernel<<<static_cast<unsigned>(blocks), 128, 0, s>>>(X, n, d, rpb, part.get());
    UMAPB_LAUNCH_CHECK();
    std::vector<double> h(blocks * 2 * d);
    UMAPB_CUDA(cudaMemcpyAsync(h.data(), part.get(), h.size() * 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    mean.assign(d, 0.0f);
    scale.assign(d, 1.0f);
    for (int f = 0; f < d; ++f) {
        double sum = 0.0, sq = 0.0;
        for (int64_t b = 0; b < blocks; ++b) {
            sum += h[b * 2 * d + f];
            sq += h[b * 2 * d + d + f];
        }
        const double mu = sum / static_cast<double>(n);
        const double var = std::max(0.0, sq / static_cast<double>(n) - mu * mu);
        const float sd = static_cast<float>(std::sqrt(var));
        mean[f] = static_cast<float>(mu);
        scale[f] = sd > kScaleEps ? sd : 1.0f;
    }
}

template <typename T>
void upload_vec(DevBuf<T>& dst, const std::vector<T>& v, cudaStream_t s) {
    dst.alloc(v.size(), s);
    if (!v.empty())
        UMAPB_CUDA(cudaMemcpyAsync(dst.get(), v.data(), v.size() * sizeof(T),
                                   cudaMemcpyHostToDevice, s));
}

// Network outputs (and, when the gate exists, nearest anchors) of `rows`
// query rows Q[ids ? ids[r] : r].
void infer_rows(const Surrogate& sg, const float* Q, const int32_t* ids, int64_t rows,
                float* out, uint8_t* flags, int32_t* anchor_of, float* anchor_d2,
                cudaStream_t s) {
    const Layout& L = sg.L;
    const int64_t chunk = std::min<int64_t>(rows, kInferChunk);
    Pass P;
    P.alloc(L, chunk, false, s);
    // the gate runs only when its flags or nearest anchors are asked for
    const bool gate = sg.n_anchors > 0 && (flags || anchor_of || anchor_d2);
    const int a_tiles = gate ? static_cast<int>(ceil_div(sg.n_anchors, 128)) : 0;
    DevBuf<float> row_sq, amin;
    DevBuf<int32_t> amin_idx;
    if (gate) {
        row_sq.alloc(chunk, s);
        amin.alloc(a_tiles * chunk, s);
        amin_idx.alloc(a_tiles * chunk, s);
    }
    for (int64_t r0 = 0; r0 < rows; r0 += chunk) {
        const int64_t n = std::min(chunk, rows - r0);
        P.rows = n;
        if (ids)
            standardize(Q, static_cast<int>(L.din), ids + r0, n, sg.mean.get(), sg.scale.get(),
                        static_cast<int>(L.dp), P.X.get(), nullptr, 0, s);
        else
            standardize(Q + r0 * L.din, static_cast<int>(L.din), nullptr, n, sg.mean.get(),
                        sg.scale.get(), static_cast<int>(L.dp), P.X.get(), nullptr, 0, s);
        if (out) forward(sg, P, false, s);
        if (gate) {
            row_sq_bf16_kernel<<<grid_for(n * 32), 256, 0, s>>>(P.X.get(), n,
                                                                static_cast<int>(L.dp),
                                                                row_sq.get());
            UMAPB_LAUNCH_CHECK();
            GemmOut og;
            og.col_sq = sg.anchor_sq.get();
            og.n_valid = sg.n_anchors;
            og.min_val = amin.get();
            og.min_idx = amin_idx.get();
            gemm_bf16_tn(P.X.get(), sg.anchors.get(), n, sg.n_anchors, L.dp, kEpiRowMin, og, s);
        }
        FinishArgs f{};
        f.head_part = P.part.get();
        f.n_tiles = static_cast<int>(L.H / 128);
        f.b3 = sg.params.get() + L.b3;
        f.out_shift = sg.out_shift.get();
        f.out_scale = sg.out_scale.get();
        f.dout = static_cast<int>(L.dout);
        f.rows = n;
        f.amin_val = amin.get();
        f.amin_idx = amin_idx.get();
        f.a_tiles = a_tiles;
        f.row_sq = row_sq.get();
        f.anchor_r2 = sg.anchor_r2.get();
        f.cell_ok = sg.cell_ok.get();
        f.out = out ? out + r0 * L.dout : nullptr;
        f.flags = (flags && gate) ? flags + r0 : nullptr;
        f.anchor_of = anchor_of ? anchor_of + r0 : nullptr;
        f.anchor_d2 = anchor_d2 ? anchor_d2 + r0 : nullptr;
        finish_kernel<<<grid_for(n), 256, 0, s>>>(f);
        UMAPB_LAUNCH_CHECK();
    }
}

double wall_now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

}  // namespace

SurrogatePtr surrogate_train(const float* X, int64_t n, int d, const float* emb, int dim,
                             const Graph& g, float a, float b, int64_t neg_rate,
                             const umapb_surrogate_params& prm, uint64_t seed,
                             umapb_surrogate_info* info, std::vector<double>* history,
                             cudaStream_t s) {
    if (dim < 1 || dim > kGemmMaxHead) invalid("the surrogate supports 1..4 output components");
    if (prm.hidden < 128 || prm.hidden % 128 != 0)
        invalid("surrogate hidden width must be a positive multiple of 128");
    if (prm.batch_size < 128 || prm.batch_size % 128 != 0)
        invalid("surrogate batch_size must be a positive multiple of 128");
    if (prm.epochs < 1) invalid("surrogate epochs must be >= 1");
    if (!(prm.learning_rate > 0.0f)) invalid("surrogate learning_rate must be > 0");
    if (!(prm.holdout_fraction >= 0.0f && prm.holdout_fraction < 0.5f))
        invalid("surrogate holdout_fraction must be in [0, 0.5)");
    if (prm.n_anchors < 1 || prm.negatives < 0) invalid("surrogate n_anchors must be >= 1");
    const double t0 = wall_now();
    auto sg = SurrogatePtr(new Surrogate());
    Layout& L = sg->L;
    L.set(d, prm.hidden, dim);

    // ---- S1: standardisation and the held-out split
    std::vector<float> mean, scale;
    feature_stats(X, n, d, mean, scale, s);
    upload_vec(sg->mean, mean, s);
    upload_vec(sg->scale, scale, s);
    std::vector<int32_t> train_ids, hold_ids;
    const uint64_t hold_cut =
        static_cast<uint64_t>(static_cast<double>(prm.holdout_fraction) * 4294967296.0);
    for (int64_t i = 0; i < n; ++i) {
        if ((rng_word(seed, 201, i) >> 32) < hold_cut)
            hold_ids.push_back(static_cast<int32_t>(i));
        else
            train_ids.push_back(static_cast<int32_t>(i));
    }
    const int64_t n_train = static_cast<int64_t>(train_ids.size());
    int64_t B = prm.batch_size;
    if (n_train < B) B = (n_train / 128) * 128;
    if (B < 128) invalid("the surrogate needs at least 128 training rows");
    const int64_t steps_per_epoch = n_train / B;

    // the network predicts the embedding in units of its per-axis spread
    std::vector<float> h_e(n * dim);
    UMAPB_CUDA(cudaMemcpyAsync(h_e.data(), emb, h_e.size() * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    {
        std::vector<float> sh(dim), sc(dim);
        for (int o = 0; o < dim; ++o) {
            double sum = 0.0, sq = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                const double v = h_e[i * dim + o];
                sum += v;
                sq += v * v;
            }
            const double mu = sum / static_cast<double>(n);
            const double sd = std::sqrt(std::max(0.0, sq / static_cast<double>(n) - mu * mu));
            sh[o] = static_cast<float>(mu);
            sc[o] = sd > 1e-6 ? static_cast<float>(sd) : 1.0f;
        }
        upload_vec(sg->out_shift, sh, s);
        upload_vec(sg->out_scale, sc, s);
    }

    // ---- S2/S3: network, Adam state, scratch
    alloc_network(*sg, s);
    upload_vec(sg->params, init_params(L, seed), s);
    DevBuf<float> grad(L.total, s), m1(L.total, s), m2(L.total, s);
    UMAPB_CUDA(cudaMemsetAsync(m1.get(), 0, L.total * 4, s));
    UMAPB_CUDA(cudaMemsetAsync(m2.get(), 0, L.total * 4, s));
    adam_step(*sg, grad.get(), m1.get(), m2.get(), 0, 0.0f, false, s);
    Pass P;
    P.alloc(L, B, true, s);
    DevBuf<int32_t> ids_in, perm, keys_in, keys_out;
    upload_vec(ids_in, train_ids, s);
    perm.alloc(n_train, s);
    std::vector<int32_t> hkeys(n_train);
    keys_in.alloc(n_train, s);
    keys_out.alloc(n_train, s);
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys_in.get(), keys_out.get(),
                                    ids_in.get(), perm.get(), static_cast<int>(n_train), 0, 31,
                                    s);
    DevBuf<uint8_t> sort_tmp(sort_bytes, s);
    DevBuf<double> loss_acc(prm.epochs, s);
    UMAPB_CUDA(cudaMemsetAsync(loss_acc.get(), 0, prm.epochs * 8, s));

    LossArgs la{};
    la.head_part = P.part.get();
    la.n_tiles = static_cast<int>(L.H / 128);
    la.b3 = sg->params.get() + L.b3;
    la.out_shift = sg->out_shift.get();
    la.out_scale = sg->out_scale.get();
    la.dout = dim;
    la.B = B;
    la.targets = emb;
    la.teacher = emb;
    la.n_teacher = n;
    la.row_ptr = g.row_ptr.get();
    la.tails = g.tails.get();
    la.weights = g.weights.get();
    la.n_neg = static_cast<int>(prm.negatives);
    la.seed = seed ^ 0x5EED0F5A11CE5ULL;
    la.a = a;
    la.b = b;
    la.mse_w = prm.mse_weight;
    la.edge_w = prm.edge_loss_weight;
    la.neg_scale = static_cast<float>(neg_rate);
    la.dY = P.dY.get();

    // ---- S4: training
    int64_t t = 0;
    for (int64_t ep = 0; ep < prm.epochs; ++ep) {
        // a fresh permutation of the training rows: sort by random keys
        for (int64_t i = 0; i < n_train; ++i)
            hkeys[i] = static_cast<int32_t>(rng_word(seed, 300 + ep, i) >> 33);
        UMAPB_CUDA(cudaMemcpyAsync(keys_in.get(), hkeys.data(), n_train * 4,
                                   cudaMemcpyHostToDevice, s));
        cub::DeviceRadixSort::SortPairs(sort_tmp.get(), sort_bytes, keys_in.get(),
                                        keys_out.get(), ids_in.get(), perm.get(),
                                        static_cast<int>(n_train), 0, 31, s);
        UMAPB_CUDA(cudaGetLastError());
        la.loss_acc = loss_acc.get() + ep;
        for (int64_t st = 0; st < steps_per_epoch; ++st, ++t) {
            const int32_t* bid = perm.get() + st * B;
            standardize(X, d, bid, B, sg->mean.get(), sg->scale.get(), static_cast<int>(L.dp),
                        P.X.get(), P.XT.get(), B, s);
            forward(*sg, P, true, s);
            la.ids = bid;
            la.step = static_cast<uint64_t>(t);
            loss_kernel<<<grid_for(B), 256, 0, s>>>(la);
            UMAPB_LAUNCH_CHECK();
            backward(*sg, P, grad.get(), s);
            adam_step(*sg, grad.get(), m1.get(), m2.get(), t + 1, prm.learning_rate, true, s);
        }
        check_gemm(s);
    }
    std::vector<double> hist(prm.epochs);
    UMAPB_CUDA(cudaMemcpyAsync(hist.data(), loss_acc.get(), prm.epochs * 8,
                               cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    for (double& v : hist) v /= static_cast<double>(std::max<int64_t>(steps_per_epoch, 1));
    const double t1 = wall_now();

    // ---- S5: gate.  Anchors are a seeded sample of the training rows; each
    // anchor's squared radius is the largest squared distance of a training
    // row assigned to it.
    const int64_t C = std::min<int64_t>(prm.n_anchors, n_train);
    std::vector<int32_t> pool = train_ids;
    for (int64_t i = 0; i < C; ++i) {
        const int64_t j =
            i + rng_below(rng_word(seed, 401, i), static_cast<uint32_t>(n_train - i));
        std::swap(pool[i], pool[j]);
    }
    std::vector<int32_t> anchor_rows(pool.begin(), pool.begin() + C);
    DevBuf<int32_t> anchor_ids;
    upload_vec(anchor_ids, anchor_rows, s);
    sg->anchors.alloc(ceil_div(C, 128) * 128 * L.dp, s);
    UMAPB_CUDA(cudaMemsetAsync(sg->anchors.get(), 0, sg->anchors.bytes(), s));
    standardize(X, d, anchor_ids.get(), C, sg->mean.get(), sg->scale.get(),
                static_cast<int>(L.dp), sg->anchors.get(), nullptr, 0, s);
    sg->anchor_sq.alloc(C, s);
    row_sq_bf16_kernel<<<grid_for(C * 32), 256, 0, s>>>(sg->anchors.get(), C,
                                                        static_cast<int>(L.dp),
                                                        sg->anchor_sq.get());
    UMAPB_LAUNCH_CHECK();
    sg->n_anchors = C;
    // all rows: nearest anchor (the network outputs are not needed here)
    DevBuf<int32_t> all_anchor(n, s);
    DevBuf<float> all_d2(n, s);
    infer_rows(*sg, X, nullptr, n, nullptr, nullptr, all_anchor.get(), all_d2.get(), s);
    std::vector<int32_t> h_anchor(n);
    std::vector<float> h_d2(n);
    UMAPB_CUDA(cudaMemcpyAsync(h_anchor.data(), all_anchor.get(), n * 4, cudaMemcpyDeviceToHost,
                               s));
    UMAPB_CUDA(cudaMemcpyAsync(h_d2.data(), all_d2.get(), n * 4, cudaMemcpyDeviceToHost, s));
    // held-out rows: network outputs against the fitted embedding
    const int64_t n_hold = static_cast<int64_t>(hold_ids.size());
    std::vector<float> h_y(n_hold * dim);
    if (n_hold > 0) {
        DevBuf<int32_t> hid;
        upload_vec(hid, hold_ids, s);
        DevBuf<float> yh(n_hold * dim, s);
        infer_rows(*sg, X, hid.get(), n_hold, yh.get(), nullptr, nullptr, nullptr, s);
        UMAPB_CUDA(cudaMemcpyAsync(h_y.data(), yh.get(), h_y.size() * 4, cudaMemcpyDeviceToHost,
                                   s));
    }
    UMAPB_CUDA(cudaStreamSynchronize(s));
    check_gemm(s);

    std::vector<uint8_t> is_hold(n, 0);
    for (int32_t i : hold_ids) is_hold[i] = 1;
    std::vector<float> r2(C, 0.0f);
    for (int64_t i = 0; i < n; ++i)
        if (!is_hold[i]) r2[h_anchor[i]] = std::max(r2[h_anchor[i]], h_d2[i]);
    // the fallback radius: stated, or 5% of the widest 1%-99% extent
    float radius = prm.fallback_radius;
    if (!(radius > 0.0f)) {
        double ext = 0.0;
        std::vector<float> col(n);
        for (int o = 0; o < dim; ++o) {
            for (int64_t i = 0; i < n; ++i) col[i] = h_e[i * dim + o];
            const int64_t lo = n / 100, hi = std::max<int64_t>(lo, n - 1 - n / 100);
            std::nth_element(col.begin(), col.begin() + lo, col.end());
            const float vlo = col[lo];
            std::nth_element(col.begin(), col.begin() + hi, col.end());
            ext = std::max(ext, static_cast<double>(col[hi] - vlo));
        }
        radius = static_cast<float>(0.05 * ext);
    }
    std::vector<int64_t> tot(C, 0), bad(C, 0);
    std::vector<double> errs(n_hold);
    double se = 0.0;
    int64_t within = 0;
    for (int64_t h = 0; h < n_hold; ++h) {
        const int64_t i = hold_ids[h];
        double d2 = 0.0;
        for (int o = 0; o < dim; ++o) {
            const double df = static_cast<double>(h_y[h * dim + o]) - h_e[i * dim + o];
            d2 += df * df;
        }
        se += d2;
        errs[h] = std::sqrt(d2);
        const bool ok = std::sqrt(d2) <= radius;
        within += ok ? 1 : 0;
        ++tot[h_anchor[i]];
        bad[h_anchor[i]] += ok ? 0 : 1;
    }
    // A cell's failure rate is its held-out share outside the radius,
    // smoothed towards the overall share with a weight of kCellPrior rows,
    // so cells with few held-out rows lean on the global evidence.
    const double global_bad =
        n_hold > 0 ? static_cast<double>(n_hold - within) / static_cast<double>(n_hold) : 1.0;
    std::vector<uint8_t> cell(C, 0);
    int64_t trusted = 0;
    for (int64_t c = 0; c < C; ++c) {
        const double rate = (static_cast<double>(bad[c]) + kCellPrior * global_bad) /
                            (static_cast<double>(tot[c]) + kCellPrior);
        cell[c] = rate <= static_cast<double>(prm.max_cell_failure) ? 1 : 0;
        trusted += cell[c];
    }
    int64_t gated = 0;
    for (int64_t h = 0; h < n_hold; ++h) {
        const int64_t i = hold_ids[h];
        const int32_t c = h_anchor[i];
        gated += (cell[c] && h_d2[i] <= r2[c]) ? 0 : 1;
    }
    upload_vec(sg->anchor_r2, r2, s);
    upload_vec(sg->cell_ok, cell, s);
    sg->radius = radius;
    UMAPB_CUDA(cudaStreamSynchronize(s));
    const double t2 = wall_now();
    if (history) *history = hist;
    if (info) {
        info->n_train = n_train;
        info->n_holdout = n_hold;
        info->steps = t;
        info->n_anchors = C;
        info->cells_trusted = trusted;
        info->radius = radius;
        info->train_sec = t1 - t0;
        info->calibrate_sec = t2 - t1;
        info->first_epoch_loss = hist.empty() ? 0.0 : hist.front();
        info->final_epoch_loss = hist.empty() ? 0.0 : hist.back();
        info->holdout_rmse = n_hold > 0 ? std::sqrt(se / static_cast<double>(n_hold)) : 0.0;
        if (n_hold > 0) {
            std::nth_element(errs.begin(), errs.begin() + n_hold / 2, errs.end());
            info->holdout_median_error = errs[n_hold / 2];
        }
        info->holdout_within_radius =
            n_hold > 0 ? static_cast<double>(within) / static_cast<double>(n_hold) : 0.0;
        info->holdout_gated =
            n_hold > 0 ? static_cast<double>(gated) / static_cast<double>(n_hold) : 0.0;
    }
    return sg;
}

void surrogate_infer_async(const Surrogate& sg, const float* Q, int64_t nq, int d, float* out,
                           uint8_t* flags, cudaStream_t s) {
    if (d != sg.L.din) invalid("surrogate input width differs from the fitted rows");
    if (nq == 0) return;
    infer_rows(sg, Q, nullptr, nq, out, flags, nullptr, nullptr, s);
}

void surrogate_gate_async(const Surrogate& sg, const float* Q, int64_t nq, int d, uint8_t* flags,
                          cudaStream_t s) {
    if (d != sg.L.din) invalid("surrogate input width differs from the fitted rows");
    if (nq == 0) return;
    infer_rows(sg, Q, nullptr, nq, nullptr, flags, nullptr, nullptr, s);
}

void surrogate_forward_async(const Surrogate& sg, const float* Q, int64_t nq, int d, float* out,
                             cudaStream_t s) {
    if (d != sg.L.din) invalid("surrogate input width differs from the fitted rows");
    if (nq == 0) return;
    infer_rows(sg, Q, nullptr, nq, out, nullptr, nullptr, nullptr, s);
}

void surrogate_check(cudaStream_t s) { check_gemm(s); }

int64_t surrogate_count_flags(const uint8_t* flags, int64_t nq, cudaStream_t s) {
    check_gemm(s);
    if (!flags || nq == 0) return 0;
    DevBuf<unsigned long long> cnt(1, s);
    UMAPB_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, s));
    count_flags_kernel<<<std::min<int64_t>(grid_for(nq), 4096), 256, 0, s>>>(flags, nq, cnt.get());
    UMAPB_LAUNCH_CHECK();
    unsigned long long h = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, cnt.get(), 8, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    return static_cast<int64_t>(h);
}

void mlp_grad(const umapb_mlp_batch& mb, float* grads, double* loss, float* y, cudaStream_t s) {
    if (mb.batch < 128 || mb.batch % 128 != 0) invalid("mlp batch must be a multiple of 128");
    if (mb.hidden < 128 || mb.hidden % 128 != 0) invalid("mlp hidden must be a multiple of 128");
    if (mb.n_out < 1 || mb.n_out > kGemmMaxHead) invalid("mlp n_out must be in [1, 4]");
    if (mb.n_features < 1 || mb.n_teacher < 1 || mb.n_neg < 0) invalid("mlp sizes");
    Surrogate sg;
    Layout& L = sg.L;
    L.set(mb.n_features, mb.hidden, mb.n_out);
    const int64_t B = mb.batch, din = L.din, dp = L.dp, H = L.H, dout = L.dout;
    // padded master vector from the caller's unpadded layout
    const int64_t u_b1 = H * din, u_w2 = u_b1 + H, u_b2 = u_w2 + H * H, u_w3 = u_b2 + H,
                  u_b3 = u_w3 + dout * H;
    std::vector<float> w(L.total, 0.0f);
    for (int64_t r = 0; r < H; ++r)
        std::copy(mb.params + r * din, mb.params + (r + 1) * din, w.begin() + L.w1 + r * dp);
    std::copy(mb.params + u_b1, mb.params + u_b1 + H, w.begin() + L.b1);
    std::copy(mb.params + u_w2, mb.params + u_w2 + H * H, w.begin() + L.w2);
    std::copy(mb.params + u_b2, mb.params + u_b2 + H, w.begin() + L.b2);
    std::copy(mb.params + u_w3, mb.params + u_w3 + dout * H, w.begin() + L.w3);
    std::copy(mb.params + u_b3, mb.params + u_b3 + dout, w.begin() + L.b3);
    alloc_network(sg, s);
    upload_vec(sg.params, w, s);
    DevBuf<float> grad(L.total, s);
    adam_step(sg, grad.get(), nullptr, nullptr, 0, 0.0f, false, s);
    // inputs: identity standardisation
    std::vector<float> ones(din, 1.0f), zeros(din, 0.0f);
    upload_vec(sg.mean, zeros, s);
    upload_vec(sg.scale, ones, s);
    upload_vec(sg.out_shift, mb.out_shift ? std::vector<float>(mb.out_shift, mb.out_shift + dout)
                                          : std::vector<float>(dout, 0.0f), s);
    upload_vec(sg.out_scale, mb.out_scale ? std::vector<float>(mb.out_scale, mb.out_scale + dout)
                                          : std::vector<float>(dout, 1.0f), s);
    DevBuf<float> xd, td, teach, ew, yd;
    upload_vec(xd, std::vector<float>(mb.x, mb.x + B * din), s);
    upload_vec(td, std::vector<float>(mb.targets, mb.targets + B * dout), s);
    upload_vec(teach, std::vector<float>(mb.teacher, mb.teacher + mb.n_teacher * dout), s);
    const int64_t n_edges = mb.edge_ptr[B];
    std::vector<int32_t> rp(B + 1);
    for (int64_t i = 0; i <= B; ++i) {
        if (mb.edge_ptr[i] < 0 || mb.edge_ptr[i] > n_edges || (i > 0 && mb.edge_ptr[i] < mb.edge_ptr[i - 1]))
            invalid("mlp edge_ptr must be non-decreasing");
        rp[i] = static_cast<int32_t>(mb.edge_ptr[i]);
    }
    for (int64_t e = 0; e < n_edges; ++e)
        if (mb.edge_tail[e] < 0 || mb.edge_tail[e] >= mb.n_teacher)
            invalid("mlp edge_tail out of range");
    for (int64_t e = 0; e < B * mb.n_neg; ++e)
        if (mb.neg_tail[e] < 0 || mb.neg_tail[e] >= mb.n_teacher)
            invalid("mlp neg_tail out of range");
    DevBuf<int32_t> rpd, tails, negs;
    upload_vec(rpd, rp, s);
    upload_vec(tails, std::vector<int32_t>(mb.edge_tail, mb.edge_tail + n_edges), s);
    upload_vec(ew, std::vector<float>(mb.edge_weight, mb.edge_weight + n_edges), s);
    upload_vec(negs, std::vector<int32_t>(mb.neg_tail, mb.neg_tail + B * mb.n_neg), s);
    DevBuf<double> lacc(1, s);
    UMAPB_CUDA(cudaMemsetAsync(lacc.get(), 0, 8, s));
    Pass P;
    P.alloc(L, B, true, s);
    standardize(xd.get(), static_cast<int>(din), nullptr, B, sg.mean.get(), sg.scale.get(),
                static_cast<int>(dp), P.X.get(), P.XT.get(), B, s);
    forward(sg, P, true, s);
    LossArgs la{};
    la.head_part = P.part.get();
    la.n_tiles = static_cast<int>(H / 128);
    la.b3 = sg.params.get() + L.b3;
    la.out_shift = sg.out_shift.get();
    la.out_scale = sg.out_scale.get();
    la.dout = static_cast<int>(dout);
    la.B = B;
    la.targets = td.get();
    la.teacher = teach.get();
    la.n_teacher = mb.n_teacher;
    la.row_ptr = rpd.get();
    la.tails = tails.get();
    la.weights = ew.get();
    la.neg_ids = negs.get();
    la.n_neg = static_cast<int>(mb.n_neg);
    la.a = mb.a;
    la.b = mb.b;
    la.mse_w = mb.mse_weight;
    la.edge_w = mb.edge_loss_weight;
    la.neg_scale = mb.neg_scale;
    la.y_out = P.y.get();
    la.dY = P.dY.get();
    la.loss_acc = lacc.get();
    loss_kernel<<<grid_for(B), 256, 0, s>>>(la);
    UMAPB_LAUNCH_CHECK();
    backward(sg, P, grad.get(), s);
    std::vector<float> gh(L.total);
    UMAPB_CUDA(cudaMemcpyAsync(gh.data(), grad.get(), L.total * 4, cudaMemcpyDeviceToHost, s));
    double lh = 0.0;
    UMAPB_CUDA(cudaMemcpyAsync(&lh, lacc.get(), 8, cudaMemcpyDeviceToHost, s));
    if (y) UMAPB_CUDA(cudaMemcpyAsync(y, P.y.get(), B * dout * 4, cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    check_gemm(s);
    for (int64_t r = 0; r < H; ++r)
        std::copy(gh.begin() + L.w1 + r * dp, gh.begin() + L.w1 + r * dp + din, grads + r * din);
    std::copy(gh.begin() + L.b1, gh.begin() + L.b1 + H, grads + u_b1);
    std::copy(gh.begin() + L.w2, gh.begin() + L.w2 + H * H, grads + u_w2);
    std::copy(gh.begin() + L.b2, gh.begin() + L.b2 + H, grads + u_b2);
    std::copy(gh.begin() + L.w3, gh.begin() + L.w3 + dout * H, grads + u_w3);
    std::copy(gh.begin() + L.b3, gh.begin() + L.b3 + dout, grads + u_b3);
    if (loss) *loss = lh;
}

}  // namespace umapb
