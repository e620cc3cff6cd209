// TEST INFRASTRUCTURE ONLY (never linked by the product): the k-means++
// initialisation of AOCL-DA restated on the CPU, for pinning the GPU handle's
// choice of initial centres and for the CPU baseline's setup.
//
// Follows clustering/kmeans/kmeans.cpp:1524-1664 (kmeans_plusplus) with
// kmeans.cpp:1491-1521 (compute_distances_to_point, euclidean branch) and the
// engine seeding of kmeans.cpp:1814-1822: the same engine (std::mt19937_64
// seeded with `seed`), the first centre from std::uniform_int_distribution<>
// over [0, n-1], then for every further centre n_trials = 2 + (int)log(k)
// draws of std::discrete_distribution<> over the current minimum squared
// distances, each candidate's cost sum_i max(0, min(w_i, d_i(candidate))),
// repeated candidates skipped, the first strictly smaller finite cost wins,
// and the winner's weight set to zero.  Weights are clamped to zero when
// negative or non-finite, and a data set whose distances to the first centre
// are all zero takes rows 0..k-1.
//
// Squared distances use the GEMM form of euclidean_gemm_distance
// (metrics/euclidean_gemm_distance.cpp:60-153): fl(-2 x.c + fl(|x|^2 +
// |c|^2)).  The reference's dot product comes from BLAS gemm, whose
// summation order depends on the BLAS build; here it is one sequential fma
// chain over the features (with `gemm` null) or the caller's cblas_sgemm /
// cblas_dgemm (the CPU baseline).  Squared norms are the sequential sum
// norms[i] += v*v of compute_squared_row_norms (utilities/da_utils.cpp:775-796)
// as GCC contracts it (one fma per feature).  The candidate cost accumulates
// in the working precision T, serially, as the reference does; cost_fp64 = 1
// accumulates in fp64 instead (to classify a disagreement).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <random>
#include <vector>

namespace {

typedef void (*sgemm_fn)(int, int, int, int, int, int, float, const float *, int,
                         const float *, int, float, float *, int);
typedef void (*dgemm_fn)(int, int, int, int, int, int, double, const double *, int,
                         const double *, int, double, double *, int);

inline float fma_t(float a, float b, float c) { return std::fmaf(a, b, c); }
inline double fma_t(double a, double b, double c) { return std::fma(a, b, c); }

template <typename T> struct Gemm;
template <> struct Gemm<float> {
    static void run(void *f, int n, int t, int d, const float *X, const float *Y, float *out) {
        // out (n x t, row-major) = X (n x d) . Y^T (Y: t x d, row-major)
        reinterpret_cast<sgemm_fn>(f)(101, 111, 112, n, t, d, 1.0f, X, d, Y, d, 0.0f, out, t);
    }
};
template <> struct Gemm<double> {
    static void run(void *f, int n, int t, int d, const double *X, const double *Y, double *out) {
        reinterpret_cast<dgemm_fn>(f)(101, 111, 112, n, t, d, 1.0, X, d, Y, d, 0.0, out, t);
    }
};

// cosine = 1: spherical k-means (kmeans.cpp:1495-1510), the distance
// max(0, 1 - cos) with cos = fl(fl(dot inv_i) inv_c) (normalise) or dot;
// inv = 1 / sqrt(|x|^2), 0 for a zero row (kmeans.cpp:681-703).
template <typename T>
int kmeanspp(int n, int d, const T *X, int k, long long seed, int cost_fp64, void *gemm,
             int32_t *chosen, int cosine = 0, int normalise = 0) {
    if (n < 1 || d < 1 || k < 1 || k > n) return -1;
    std::mt19937_64 gen;
    gen.seed((uint64_t)seed);
    std::vector<T> xn(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        T s = T(0);
        for (int f = 0; f < d; ++f) s = fma_t(X[(size_t)i * d + f], X[(size_t)i * d + f], s);
        xn[i] = s;
    }
    std::vector<T> inv;
    if (cosine && normalise) {
        inv.resize(n);
        for (int i = 0; i < n; ++i) inv[i] = xn[i] > T(0) ? T(1) / std::sqrt(xn[i]) : T(0);
    }
    const int n_trials = 2 + (int)std::log((double)k);
    // squared distances of every row to the candidate rows cand[0..t)
    std::vector<T> dots;
    auto distances = [&](const int *cand, int t, T *out /* t x n */) {
        if (gemm) {
            std::vector<T> Y((size_t)t * d);
            for (int c = 0; c < t; ++c)
                for (int f = 0; f < d; ++f) Y[(size_t)c * d + f] = X[(size_t)cand[c] * d + f];
            dots.resize((size_t)n * t);
            Gemm<T>::run(gemm, n, t, d, X, Y.data(), dots.data());
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            for (int c = 0; c < t; ++c) {
                T s;
                if (gemm) {
                    s = dots[(size_t)i * t + c];
                } else {
                    s = T(0);
                    for (int f = 0; f < d; ++f)
                        s = fma_t(X[(size_t)i * d + f], X[(size_t)cand[c] * d + f], s);
                }
                if (cosine) {
                    const T cs = inv.empty() ? s : (s * inv[i]) * inv[cand[c]];
                    out[(size_t)c * n + i] = std::max(T(0), T(1) - cs);
                    continue;
                }
                const T nn = xn[i] + xn[cand[c]];
                out[(size_t)c * n + i] = fma_t(T(-2), s, nn);
            }
        }
    };
    std::uniform_int_distribution<> dis_int(0, n - 1);
    const int first = dis_int(gen);
    chosen[0] = first;
    std::vector<T> w(n), dk((size_t)n_trials * n);
    distances(&first, 1, w.data());
    w[first] = T(0);
    bool coincident = true;
    for (int i = 0; i < n; ++i) {
        if (!std::isfinite(w[i]) || w[i] < T(0)) w[i] = T(0);
        if (w[i] > T(0)) coincident = false;
    }
    if (coincident) {
        for (int c = 0; c < k; ++c) chosen[c] = c;
        return 1;
    }
    std::vector<int> cand(n_trials);
    for (int c = 1; c < k; ++c) {
        std::discrete_distribution<> weighted(w.begin(), w.end());
        for (int t = 0; t < n_trials; ++t) cand[t] = weighted(gen);
        distances(cand.data(), n_trials, dk.data());
        // each candidate's cost is one serial sum (the trials in parallel)
        std::vector<T> cost(n_trials);
        std::vector<double> cost64(n_trials);
#pragma omp parallel for schedule(static, 1)
        for (int t = 0; t < n_trials; ++t) {
            const T *dc = dk.data() + (size_t)t * n;
            T s = T(0);
            double s64 = 0.0;
            for (int i = 0; i < n; ++i) {
                const T m = std::max(T(0), std::min(w[i], dc[i]));
                s += m;
                s64 += (double)m;
            }
            cost[t] = s;
            cost64[t] = s64;
        }
        int best = 0, best_t = -1;
        T best_cost = std::numeric_limits<T>::infinity();
        double best_cost64 = std::numeric_limits<double>::infinity();
        for (int t = 0; t < n_trials; ++t) {
            bool repeat = false;
            for (int u = 0; u < t; ++u)
                if (cand[u] == cand[t]) repeat = true;
            if (repeat) continue;
            const bool better = cost_fp64 ? (std::isfinite(cost64[t]) && cost64[t] < best_cost64)
                                          : (std::isfinite(cost[t]) && cost[t] < best_cost);
            if (better) {
                best_cost = cost[t];
                best_cost64 = cost64[t];
                best = cand[t];
                best_t = t;
            }
        }
        chosen[c] = best;
        if (best_t >= 0) {
            const T *dc = dk.data() + (size_t)best_t * n;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) w[i] = std::max(T(0), std::min(w[i], dc[i]));
        }
        w[best] = T(0);
    }
    return 0;
}

} // namespace

extern "C" {
// Row-major X (n x d, leading dimension d).  Writes the k chosen row indices;
// returns 0, 1 (coincident data: rows 0..k-1) or -1 (bad arguments).
int orc_kmeanspp_s(int n, int d, const float *X, int k, long long seed, int cost_fp64,
                   void *sgemm, int32_t *chosen) {
    return kmeanspp<float>(n, d, X, k, seed, cost_fp64, sgemm, chosen);
}
int orc_kmeanspp_d(int n, int d, const double *X, int k, long long seed, int cost_fp64,
                   void *dgemm, int32_t *chosen) {
    return kmeanspp<double>(n, d, X, k, seed, cost_fp64, dgemm, chosen);
}
// Spherical k-means++ (cosine distance; normalise: the "normalize data" option).
int orc_kmeanspp_cos_s(int n, int d, const float *X, int k, long long seed, int normalise,
                       int32_t *chosen) {
    return kmeanspp<float>(n, d, X, k, seed, 0, nullptr, chosen, 1, normalise);
}
int orc_kmeanspp_cos_d(int n, int d, const double *X, int k, long long seed, int normalise,
                       int32_t *chosen) {
    return kmeanspp<double>(n, d, X, k, seed, 0, nullptr, chosen, 1, normalise);
}
}

extern "C" {
// Random-samples initialisation (kmeans.cpp:1403-1424 with da_std::sample,
// utilities/da_std.hpp:102-118): selection sampling over the rows 0..n-1,
// std::mt19937_64 seeded with `seed`, one std::uniform_int_distribution over
// [0, remaining - 1] per row visited (da_int = 32-bit).  Writes min(k, n)
// row indices in increasing order.
int orc_random_rows(int n, int k, long long seed, int32_t *out) {
    if (n < 1 || k < 1) return -1;
    std::mt19937_64 gen;
    gen.seed((uint64_t)seed);
    int32_t need = std::min(k, n), pop = n, m = 0;
    for (int32_t i = 0; need > 0; ++i, --pop) {
        std::uniform_int_distribution<int32_t> d(0, pop - 1);
        if (d(gen) < need) {
            out[m++] = i;
            --need;
        }
    }
    return m;
}
}
