// hostmath.cpp - host arithmetic of the engine (compiled with
// -ffp-contract=off so every a*b+c rounds twice, as the Rust build does).
//
//  * find_ab_params: rust_umap/src/lib.rs:5647-5746.  It runs once per model
//    on the host in FP32 through the C library's powf/expf, which are the
//    functions the Rust build links; its results are pinned bit for bit by
//    the reference test at lib.rs:5781-5795.
//  * symmetric_eigen: replaces nalgebra's SymmetricEigen (lib.rs:3927, 4293)
//    for the small dense problems that stay on the host (Ritz matrices, meta
//    layouts, components below 128 nodes).  Householder tridiagonalisation
//    followed by the implicit QL iteration with Wilkinson-style shifts.
#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <vector>

#include "kernels.cuh"

namespace umapb {
namespace {

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

float curve_loss_from_powers(float a, const std::vector<float>& xp, const std::vector<float>& yv) {
    float loss = 0.0f;
    for (size_t i = 0; i < xp.size(); ++i) {
        const float model = 1.0f / (1.0f + a * xp[i]);
        const float e = model - yv[i];
        loss += e * e;
    }
    return loss / static_cast<float>(xp.size());
}

}  // namespace

void find_ab_params(float spread, float min_dist, float* out_a, float* out_b) {
    constexpr int kPoints = 300;
    const float xmax = spread * 3.0f;
    std::vector<float> xv(kPoints), yv(kPoints), xp(kPoints);
    for (int i = 0; i < kPoints; ++i) {
        const float x = xmax * static_cast<float>(i) / (static_cast<float>(kPoints) - 1.0f);
        xv[i] = x;
        yv[i] = x < min_dist ? 1.0f : expf(-(x - min_dist) / spread);
    }
    float best_a = 1.0f, best_b = 1.0f;
    float best_loss = std::numeric_limits<float>::infinity();
    // coarse grid: 71 values of b in [0.3, 3.0] x 121 values of log10(a) in [-3, 3]
    for (int bi = 0; bi <= 70; ++bi) {
        const float b = 0.3f + 2.7f * static_cast<float>(bi) / 70.0f;
        const float exponent = 2.0f * b;
        for (int i = 0; i < kPoints; ++i) xp[i] = powf(xv[i], exponent);
        for (int ai = 0; ai <= 120; ++ai) {
            const float a = powf(10.0f, -3.0f + 6.0f * static_cast<float>(ai) / 120.0f);
            const float loss = curve_loss_from_powers(a, xp, yv);
            if (loss < best_loss) {
                best_loss = loss;
                best_a = a;
                best_b = b;
            }
        }
    }
    // 8-neighbour pattern search with geometric step decay
    float step_a = std::max(best_a * 0.35f, 0.05f);
    float step_b = 0.2f;
    for (int it = 0; it < 80; ++it) {
        const float a_lo = std::max(best_a - step_a, 1e-6f);
        const float b_lo = std::max(best_b - step_b, 1e-6f);
        const float a_hi = best_a + step_a, b_hi = best_b + step_b;
        const float probes[8][2] = {{a_hi, best_b}, {a_lo, best_b}, {best_a, b_hi},
                                    {best_a, b_lo}, {a_hi, b_hi},   {a_hi, b_lo},
                                    {a_lo, b_hi},   {a_lo, b_lo}};
        bool improved = false;
        for (const auto& pr : probes) {
            const float loss = curve_loss(pr[0], pr[1], xv, yv);
            if (loss < best_loss) {
                best_loss = loss;
                best_a = pr[0];
                best_b = pr[1];
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

void symmetric_eigen(const std::vector<double>& A, int n, std::vector<double>& w,
                     std::vector<double>& V) {
    // Householder reduction: Q^T A Q = T (diagonal d, off-diagonal e), Q in V.
    std::vector<double> Z(A), d(n), e(n);
    auto z = [&](int r, int c) -> double& { return Z[static_cast<size_t>(r) * n + c]; };
    for (int j = 0; j < n; ++j) d[j] = z(n - 1, j);
    for (int i = n - 1; i > 0; --i) {
        double scale = 0.0, h = 0.0;
        for (int k = 0; k < i; ++k) scale += std::fabs(d[k]);
        if (scale == 0.0) {
            e[i] = d[i - 1];
            for (int j = 0; j < i; ++j) {
                d[j] = z(i - 1, j);
                z(i, j) = 0.0;
                z(j, i) = 0.0;
            }
        } else {
            for (int k = 0; k < i; ++k) {
                d[k] /= scale;
                h += d[k] * d[k];
            }
            double f = d[i - 1];
            double g = f > 0 ? -std::sqrt(h) : std::sqrt(h);
            e[i] = scale * g;
            h -= f * g;
            d[i - 1] = f - g;
            for (int j = 0; j < i; ++j) e[j] = 0.0;
            for (int j = 0; j < i; ++j) {
                f = d[j];
                z(j, i) = f;
                g = e[j] + z(j, j) * f;
                for (int k = j + 1; k < i; ++k) {
                    g += z(k, j) * d[k];
                    e[k] += z(k, j) * f;
                }
                e[j] = g;
            }
            f = 0.0;
            for (int j = 0; j < i; ++j) {
                e[j] /= h;
                f += e[j] * d[j];
            }
            const double hh = f / (h + h);
            for (int j = 0; j < i; ++j) e[j] -= hh * d[j];
            for (int j = 0; j < i; ++j) {
                f = d[j];
                g = e[j];
                for (int k = j; k < i; ++k) z(k, j) -= f * e[k] + g * d[k];
                d[j] = z(i - 1, j);
                z(i, j) = 0.0;
            }
        }
        d[i] = h;
    }
    for (int i = 0; i < n - 1; ++i) {
        z(n - 1, i) = z(i, i);
        z(i, i) = 1.0;
        const double h = d[i + 1];
        if (h != 0.0) {
            for (int k = 0; k <= i; ++k) d[k] = z(k, i + 1) / h;
            for (int j = 0; j <= i; ++j) {
                double g = 0.0;
                for (int k = 0; k <= i; ++k) g += z(k, i + 1) * z(k, j);
                for (int k = 0; k <= i; ++k) z(k, j) -= g * d[k];
            }
        }
        for (int k = 0; k <= i; ++k) z(k, i + 1) = 0.0;
    }
    for (int j = 0; j < n; ++j) {
        d[j] = z(n - 1, j);
        z(n - 1, j) = 0.0;
    }
    z(n - 1, n - 1) = 1.0;
    // implicit QL on the tridiagonal matrix, accumulating rotations into Z
    for (int i = 1; i < n; ++i) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    double shift_acc = 0.0, tst1 = 0.0;
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        tst1 = std::max(tst1, std::fabs(d[l]) + std::fabs(e[l]));
        int m = l;
        while (m < n - 1 && std::fabs(e[m]) > eps * tst1) ++m;
        if (m > l) {
            for (int iter = 0; iter < 200; ++iter) {
                double g = d[l];
                double p = (d[l + 1] - g) / (2.0 * e[l]);
                double r = std::hypot(p, 1.0);
                if (p < 0) r = -r;
                d[l] = e[l] / (p + r);
                d[l + 1] = e[l] * (p + r);
                const double dl1 = d[l + 1];
                double h = g - d[l];
                for (int i = l + 2; i < n; ++i) d[i] -= h;
                shift_acc += h;
                p = d[m];
                double c = 1.0, c2 = 1.0, c3 = 1.0, s = 0.0, s2 = 0.0;
                const double el1 = e[l + 1];
                for (int i = m - 1; i >= l; --i) {
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    g = c * e[i];
                    h = c * p;
                    r = std::hypot(p, e[i]);
                    e[i + 1] = s * r;
                    s = e[i] / r;
                    c = p / r;
                    p = c * d[i] - s * g;
                    d[i + 1] = h + s * (c * g + s * d[i]);
                    for (int k = 0; k < n; ++k) {
                        h = z(k, i + 1);
                        z(k, i + 1) = s * z(k, i) + c * h;
                        z(k, i) = c * z(k, i) - s * h;
                    }
                }
                p = -s * s2 * c3 * el1 * e[l] / dl1;
                e[l] = s * p;
                d[l] = c * p;
                if (std::fabs(e[l]) <= eps * tst1) break;
            }
        }
        d[l] += shift_acc;
        e[l] = 0.0;
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    w.resize(n);
    V.assign(static_cast<size_t>(n) * n, 0.0);
    for (int c = 0; c < n; ++c) {
        w[c] = d[order[c]];
        for (int r = 0; r < n; ++r) V[static_cast<size_t>(r) * n + c] = z(r, order[c]);
    }
}

}  // namespace umapb
