/*
 * oracle.c -- CPU restatement of the AOCL-DA distance / kNN / k-means hot
 * path.  TEST INFRASTRUCTURE ONLY: the reference used by tests/, smoke() and
 * the cpu_baseline leg of bench.py.  The product (libaoclda_b200.so) never
 * links, loads or calls this code.
 *
 * Every function cites the AOCL-DA source it restates (paths relative to the
 * AOCL-DA tree).  All matrices here are dense row-major (rows x d).
 *
 * Built as liboracle.so by oracle/Makefile with -O2 -ffp-contract=off so that
 * only the explicit fma() calls below are fused.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* Pair kernels                                                        */
/* ------------------------------------------------------------------ */

/* Squared euclidean in the order of sqeuclidean_kernel_packed_impl
 * (source/core/metrics/metrics_kernels.hpp:419-496) with the KC slicing of
 * LoopFour_packed (partitioning_infrastructure.hpp:175-192): per slice,
 * g1 continues from the previous slice, g2 starts at 0; groups of four dims
 * feed g1,g1,g2,g2; g1 += g2 after the groups; remainder dims feed g1. */
#define SQEUC_BODY(T, FMA)                                                         \
    T g1 = 0;                                                                      \
    for (int s0 = 0; s0 < d; s0 += kc) {                                           \
        int kcs = (d - s0) < kc ? (d - s0) : kc;                                   \
        int n4 = kcs & ~3;                                                         \
        T g2 = 0;                                                                  \
        int i = 0;                                                                 \
        for (; i < n4; i += 4) {                                                   \
            T t0 = a[s0 + i] - b[s0 + i], t1 = a[s0 + i + 1] - b[s0 + i + 1];      \
            T t2 = a[s0 + i + 2] - b[s0 + i + 2], t3 = a[s0 + i + 3] - b[s0 + i + 3]; \
            g1 = FMA(t0, t0, g1);                                                  \
            g1 = FMA(t1, t1, g1);                                                  \
            g2 = FMA(t2, t2, g2);                                                  \
            g2 = FMA(t3, t3, g2);                                                  \
        }                                                                          \
        g1 = g1 + g2;                                                              \
        for (; i < kcs; ++i) {                                                     \
            T t = a[s0 + i] - b[s0 + i];                                           \
            g1 = FMA(t, t, g1);                                                    \
        }                                                                          \
    }                                                                              \
    return g1;

static float sqeuc_s(const float *a, const float *b, int d, int kc) { SQEUC_BODY(float, fmaf) }
static double sqeuc_d(const double *a, const double *b, int d, int kc) { SQEUC_BODY(double, fma) }

/* cosine_kernel_packed_impl (metrics_kernels.hpp:670-749): one fma chain */
static float dot_s(const float *a, const float *b, int d) {
    float g = 0;
    for (int i = 0; i < d; ++i) g = fmaf(a[i], b[i], g);
    return g;
}
static double dot_d(const double *a, const double *b, int d) {
    double g = 0;
    for (int i = 0; i < d; ++i) g = fma(a[i], b[i], g);
    return g;
}
/* manhattan_kernel_packed_impl (metrics_kernels.hpp:584-666): g + |a-b| */
static float manh_s(const float *a, const float *b, int d) {
    float g = 0;
    for (int i = 0; i < d; ++i) g = g + fabsf(a[i] - b[i]);
    return g;
}
static double manh_d(const double *a, const double *b, int d) {
    double g = 0;
    for (int i = 0; i < d; ++i) g = g + fabs(a[i] - b[i]);
    return g;
}
/* minkowski_kernel_packed_impl (metrics_kernels.hpp:752-827) */
static float mink_s(const float *a, const float *b, int d, float p) {
    float g = 0;
    for (int i = 0; i < d; ++i) g = g + powf(fabsf(a[i] - b[i]), p);
    return g;
}
static double mink_d(const double *a, const double *b, int d, double p) {
    double g = 0;
    for (int i = 0; i < d; ++i) g = g + pow(fabs(a[i] - b[i]), p);
    return g;
}

/* metric ids (aoclda_metrics.h:44-59) */
enum { M_EUC = 0, M_SQEUC = 1, M_MINK = 2, M_MANH = 3, M_COS = 4, M_EUC_GEMM = 5,
       M_SQEUC_GEMM = 6, M_IP = 7 };

static float sqnorm_s(const float *x, int d) {
    float s = 0;
    for (int i = 0; i < d; ++i) s = fmaf(x[i], x[i], s);
    return s;
}
static double sqnorm_d(const double *x, int d) {
    double s = 0;
    for (int i = 0; i < d; ++i) s = fma(x[i], x[i], s);
    return s;
}
/* cosine norms with the eps -> 1 rule (cosine_distance.cpp:117-146) */
static float cnorm_s(const float *x, int d) {
    double s = 0;
    for (int i = 0; i < d; ++i) s = fma((double)x[i], (double)x[i], s);
    float v = (float)sqrt(s);
    return v <= FLT_EPSILON ? 1.0f : v;
}
static double cnorm_d(const double *x, int d) {
    double s = 0;
    for (int i = 0; i < d; ++i) s = fma(x[i], x[i], s);
    double v = sqrt(s);
    return v <= DBL_EPSILON ? 1.0 : v;
}

/* Pairwise distance value for the public metrics (pairwise_distances.cpp:37-75). */
#define PAIR_VALUE(SFX, T, SQRT, POW, FMA)                                              \
    static T pair_##SFX(int metric, const T *a, const T *b, int d, T p, int kc, T na, T nb, \
                        T ca, T cb) {                                                   \
        switch (metric) {                                                               \
        case M_EUC: return SQRT(sqeuc_##SFX(a, b, d, kc));                              \
        case M_SQEUC: return sqeuc_##SFX(a, b, d, kc);                                  \
        case M_MANH: return manh_##SFX(a, b, d);                                        \
        case M_COS: return (T)1 - dot_##SFX(a, b, d) / (ca * cb);                       \
        case M_MINK:                                                                    \
            if (p == (T)2) return SQRT(sqeuc_##SFX(a, b, d, kc));                       \
            if (p == (T)1) return manh_##SFX(a, b, d);                                  \
            return POW(mink_##SFX(a, b, d, p), (T)(1.0 / (double)p));                   \
        case M_EUC_GEMM: return SQRT(FMA((T)-2, dot_##SFX(a, b, d), na + nb));          \
        case M_SQEUC_GEMM: return FMA((T)-2, dot_##SFX(a, b, d), na + nb);              \
        default: return dot_##SFX(a, b, d);                                             \
        }                                                                               \
    }
PAIR_VALUE(s, float, sqrtf, powf, fmaf)
PAIR_VALUE(d, double, sqrt, pow, fma)

/* D (m x n, row-major) of the public pairwise API; Y == NULL means X vs X. */
#define PAIRWISE(SFX, T)                                                                  \
    void orc_pairwise_##SFX(int m, int n, int d, const T *X, const T *Y, T *D, T p,        \
                            int metric, int kc) {                                          \
        int xisy = (Y == NULL);                                                            \
        if (xisy) { Y = X; n = m; }                                                        \
        T *nx = malloc(sizeof(T) * m), *ny = malloc(sizeof(T) * n);                        \
        T *cx = malloc(sizeof(T) * m), *cy = malloc(sizeof(T) * n);                        \
        for (int i = 0; i < m; ++i) { nx[i] = sqnorm_##SFX(X + (size_t)i * d, d); cx[i] = cnorm_##SFX(X + (size_t)i * d, d); } \
        for (int j = 0; j < n; ++j) { ny[j] = sqnorm_##SFX(Y + (size_t)j * d, d); cy[j] = cnorm_##SFX(Y + (size_t)j * d, d); } \
        for (int i = 0; i < m; ++i)                                                        \
            for (int j = 0; j < n; ++j) {                                                  \
                T v = pair_##SFX(metric, X + (size_t)i * d, Y + (size_t)j * d, d, p, kc,   \
                                 nx[i], ny[j], cx[i], cy[j]);                              \
                if (xisy && i == j && (metric == M_COS || metric == M_EUC_GEMM ||          \
                                       metric == M_SQEUC_GEMM))                            \
                    v = 0;                                                                 \
                D[(size_t)i * n + j] = v;                                                  \
            }                                                                              \
        free(nx); free(ny); free(cx); free(cy);                                            \
    }
PAIRWISE(s, float)
PAIRWISE(d, double)

/* ------------------------------------------------------------------ */
/* Brute-force kNN                                                     */
/* ------------------------------------------------------------------ */
/* Selection key of a kNN metric (nearest_neighbors.cpp:337-347: euclidean
 * ranks on the squared distance and takes sqrt on output; GEMM-form squared
 * distances are clamped at 0, nearest_neighbors.cpp:662-665; inner product
 * ranks largest-first). */
#define KNN_KEY(SFX, T, FMA, POW)                                                         \
    static T knn_key_##SFX(int metric, const T *q, const T *x, int d, T p, int kc, T nq,    \
                           T nx, T cq, T cx) {                                              \
        switch (metric) {                                                                   \
        case M_EUC: case M_SQEUC: return sqeuc_##SFX(x, q, d, kc);                          \
        case M_EUC_GEMM: case M_SQEUC_GEMM: {                                               \
            T v = FMA((T)-2, dot_##SFX(q, x, d), nq + nx);                                  \
            return v < 0 ? 0 : v;                                                           \
        }                                                                                   \
        case M_MANH: return manh_##SFX(x, q, d);                                            \
        case M_COS: return (T)1 - dot_##SFX(q, x, d) / (cq * cx);                           \
        case M_IP: return -dot_##SFX(q, x, d);                                              \
        default:                                                                            \
            if (p == (T)2) return sqeuc_##SFX(x, q, d, kc);                                 \
            if (p == (T)1) return manh_##SFX(x, q, d);                                      \
            return POW(mink_##SFX(x, q, d, p), (T)(1.0 / (double)p));                       \
        }                                                                                   \
    }
KNN_KEY(s, float, fmaf, powf)
KNN_KEY(d, double, fma, pow)

/* Exact top-k under the (key, index) order: ties go to the lower index.
 * out_ind / out_dist are q-major (q*k + r).  Distances returned as the
 * reference returns them (sqrt for euclidean, sign restored for inner
 * product). */
#define KNN(SFX, T, SQRT)                                                                 \
    void orc_knn_##SFX(int nx, int d, const T *X, int nq, const T *Q, int k, int metric,   \
                       T p, int kc, int32_t *out_ind, T *out_dist) {                       \
        T *nxv = malloc(sizeof(T) * nx), *cxv = malloc(sizeof(T) * nx);                    \
        for (int i = 0; i < nx; ++i) { nxv[i] = sqnorm_##SFX(X + (size_t)i * d, d); cxv[i] = cnorm_##SFX(X + (size_t)i * d, d); } \
        int sq = (metric == M_EUC || metric == M_EUC_GEMM || (metric == M_MINK && p == (T)2)); \
        _Pragma("omp parallel for schedule(dynamic)")                                      \
        for (int q = 0; q < nq; ++q) {                                                     \
            const T *qq = Q + (size_t)q * d;                                               \
            T nqv = sqnorm_##SFX(qq, d), cqv = cnorm_##SFX(qq, d);                         \
            T *bk = malloc(sizeof(T) * (k + 1));                                           \
            int *bi = malloc(sizeof(int) * (k + 1));                                       \
            int cnt = 0;                                                                   \
            for (int i = 0; i < nx; ++i) {                                                 \
                T key = knn_key_##SFX(metric, qq, X + (size_t)i * d, d, p, kc, nqv, nxv[i], cqv, cxv[i]); \
                if (key != key) continue;                                                  \
                if (cnt == k && !(key < bk[k - 1])) continue;                              \
                int pos = cnt < k ? cnt : k - 1;                                           \
                while (pos > 0 && key < bk[pos - 1]) { bk[pos] = bk[pos - 1]; bi[pos] = bi[pos - 1]; --pos; } \
                bk[pos] = key; bi[pos] = i;                                                \
                if (cnt < k) ++cnt;                                                        \
            }                                                                              \
            for (int r = 0; r < k; ++r) {                                                  \
                out_ind[(size_t)q * k + r] = r < cnt ? bi[r] : -1;                         \
                T v = r < cnt ? bk[r] : (T)INFINITY;                                       \
                if (sq) v = SQRT(v);                                                       \
                if (metric == M_IP) v = -v;                                                \
                out_dist[(size_t)q * k + r] = v;                                           \
            }                                                                              \
            free(bk); free(bi);                                                            \
        }                                                                                  \
        free(nxv); free(cxv);                                                              \
    }
KNN(s, float, sqrtf)
KNN(d, double, sqrt)

/* The reference's own running top-k for one query and one thread
 * (nearest_neighbors.cpp:677-697 with nearest_neighbors_utils.hpp:73-101,
 * 106-116, 191-224): fill k slots in order, then replace the FIRST maximum
 * whenever a candidate is <= it, finally stable-sort by distance.  Used to
 * reproduce the reference's tie order (OMP_NUM_THREADS=1, one train block
 * of the whole set). */
void orc_knn_reference_ties_d(int nx, const double *keys, int k, int32_t *ind) {
    double *kd = malloc(sizeof(double) * k);
    int *ki = malloc(sizeof(int) * k);
    for (int i = 0; i < k; ++i) { kd[i] = keys[i]; ki[i] = i; }
    int mi = 0;
    for (int i = 1; i < k; ++i) if (kd[i] > kd[mi]) mi = i;
    for (int i = k; i < nx; ++i) {
        if (keys[i] <= kd[mi]) {
            kd[mi] = keys[i]; ki[mi] = i;
            mi = 0;
            for (int j = 1; j < k; ++j) if (kd[j] > kd[mi]) mi = j;
        }
    }
    /* stable sort by distance (insertion sort keeps equal keys in order) */
    for (int i = 1; i < k; ++i) {
        double v = kd[i]; int id = ki[i]; int j = i - 1;
        while (j >= 0 && kd[j] > v) { kd[j + 1] = kd[j]; ki[j + 1] = ki[j]; --j; }
        kd[j + 1] = v; ki[j + 1] = id;
    }
    for (int i = 0; i < k; ++i) ind[i] = ki[i];
    free(kd); free(ki);
}

/* ------------------------------------------------------------------ */
/* k-means                                                             */
/* ------------------------------------------------------------------ */
/* Lloyd assignment in working precision (kmeans_lloyd.hpp:189-198,
 * kmeans_kernels.cpp:209-234): label = argmin_j fl(-2 x.c_j + |c_j|^2),
 * strict '<' (ties keep the lower j).  The dot product is one fma chain.
 * Also returns, per row, the gap between the best and second-best value in
 * fp64 arithmetic (for classifying near-ties). */
void orc_kmeans_assign_s(int n, int d, const float *X, int k, const float *C, int32_t *labels,
                         double *gap64) {
    float *cn = malloc(sizeof(float) * k);
    for (int j = 0; j < k; ++j) cn[j] = sqnorm_s(C + (size_t)j * d, d);
    _Pragma("omp parallel for schedule(static)")
    for (int i = 0; i < n; ++i) {
        const float *x = X + (size_t)i * d;
        float best = INFINITY; int bj = 0;
        double b1 = INFINITY, b2 = INFINITY;
        for (int j = 0; j < k; ++j) {
            float v = fmaf(-2.0f, dot_s(x, C + (size_t)j * d, d), cn[j]);
            if (v < best) { best = v; bj = j; }
            if (!gap64) continue;
            double e = 0;
            for (int f = 0; f < d; ++f) { double t = (double)x[f] - (double)C[(size_t)j * d + f]; e += t * t; }
            if (e < b1) { b2 = b1; b1 = e; } else if (e < b2) b2 = e;
        }
        labels[i] = bj;
        if (gap64) gap64[i] = b2 - b1;
    }
    free(cn);
}
void orc_kmeans_assign_d(int n, int d, const double *X, int k, const double *C, int32_t *labels,
                         double *gap64) {
    double *cn = malloc(sizeof(double) * k);
    for (int j = 0; j < k; ++j) cn[j] = sqnorm_d(C + (size_t)j * d, d);
    _Pragma("omp parallel for schedule(static)")
    for (int i = 0; i < n; ++i) {
        const double *x = X + (size_t)i * d;
        double best = INFINITY; int bj = 0;
        double b1 = INFINITY, b2 = INFINITY;
        for (int j = 0; j < k; ++j) {
            double v = fma(-2.0, dot_d(x, C + (size_t)j * d, d), cn[j]);
            if (v < best) { best = v; bj = j; }
            if (!gap64) continue;
            double e = 0;
            for (int f = 0; f < d; ++f) { double t = x[f] - C[(size_t)j * d + f]; e += t * t; }
            if (e < b1) { b2 = b1; b1 = e; } else if (e < b2) b2 = e;
        }
        labels[i] = bj;
        if (gap64) gap64[i] = b2 - b1;
    }
    free(cn);
}

/* Centroid update in fp64 (kmeans_lloyd.hpp:275-405): C_j = sum / max(n_j,1),
 * an empty cluster becomes the zero vector.  Sums accumulate in row order. */
void orc_kmeans_update_d(int n, int d, const double *Xd, const int32_t *labels, int k,
                         double *C_out, int32_t *counts) {
    double *s = calloc((size_t)k * d, sizeof(double));
    for (int j = 0; j < k; ++j) counts[j] = 0;
    for (int i = 0; i < n; ++i) {
        int l = labels[i];
        counts[l]++;
        for (int f = 0; f < d; ++f) s[(size_t)l * d + f] += Xd[(size_t)i * d + f];
    }
    for (int j = 0; j < k; ++j) {
        int c = counts[j] > 0 ? counts[j] : 1;
        for (int f = 0; f < d; ++f) C_out[(size_t)j * d + f] = s[(size_t)j * d + f] / c;
    }
    free(s);
}

/* Inertia sum_i |x_i - c_{l_i}|^2 in fp64 (kmeans.cpp:1061-1124). */
double orc_kmeans_inertia_d(int n, int d, const double *X, const int32_t *labels,
                            const double *C) {
    double acc = 0;
    for (int i = 0; i < n; ++i) {
        const double *x = X + (size_t)i * d, *c = C + (size_t)labels[i] * d;
        double r = 0;
        for (int f = 0; f < d; ++f) { double t = x[f] - c[f]; r += t * t; }
        acc += r;
    }
    return acc;
}

/* Full Lloyd run with supplied initial centres (kmeans.cpp:996-1058 control
 * flow: convergence by unchanged labels after the second iteration, or by
 * |shift|_F < tol |C_prev|_F; relabel pass after tol-convergence / max_iter).
 * Assignment in working precision T (float here), sums / shift / inertia in
 * fp64.  Outputs final centres, labels, n_iter and inertia. */
void orc_kmeans_lloyd_s(int n, int d, const float *X, int k, const float *C0, int max_iter,
                        double tol, float *C_out, int32_t *labels_out, int32_t *n_iter_out,
                        double *inertia_out) {
    double *Xd = malloc(sizeof(double) * (size_t)n * d);
    for (size_t i = 0; i < (size_t)n * d; ++i) Xd[i] = X[i];
    float *Cp = malloc(sizeof(float) * (size_t)k * d), *Cc = malloc(sizeof(float) * (size_t)k * d);
    double *Cn = malloc(sizeof(double) * (size_t)k * d);
    int32_t *lp = calloc(n, sizeof(int32_t)), *lc = calloc(n, sizeof(int32_t));
    int32_t *cnt = malloc(sizeof(int32_t) * k);
    memcpy(Cc, C0, sizeof(float) * (size_t)k * d);
    int it, converged = 0;
    for (it = 0; it < max_iter; ++it) {
        float *t = Cp; Cp = Cc; Cc = t;
        int32_t *tl = lp; lp = lc; lc = tl;
        orc_kmeans_assign_s(n, d, X, k, Cp, lc, NULL);
        orc_kmeans_update_d(n, d, Xd, lc, k, Cn, cnt);
        double normc = 0, shift = 0;
        for (size_t e = 0; e < (size_t)k * d; ++e) {
            Cc[e] = (float)Cn[e];
            normc += (double)Cp[e] * (double)Cp[e];
            double df = (double)Cp[e] - (double)Cc[e];
            shift += df * df;
        }
        int conv = 0;
        if (it > 1) {
            conv = 2;
            for (int i = 0; i < n; ++i) if (lc[i] != lp[i]) { conv = 0; break; }
        }
        if (conv == 0 && sqrt(shift) < tol * sqrt(normc)) conv = 1;
        converged = conv;
        if (converged) break;
    }
    if (converged == 1 || it == max_iter) orc_kmeans_assign_s(n, d, X, k, Cc, lc, NULL);
    double *Cd = malloc(sizeof(double) * (size_t)k * d);
    for (size_t e = 0; e < (size_t)k * d; ++e) Cd[e] = Cc[e];
    *inertia_out = orc_kmeans_inertia_d(n, d, Xd, lc, Cd);
    *n_iter_out = it;
    memcpy(C_out, Cc, sizeof(float) * (size_t)k * d);
    memcpy(labels_out, lc, sizeof(int32_t) * n);
    free(Xd); free(Cp); free(Cc); free(Cn); free(lp); free(lc); free(cnt); free(Cd);
}
void orc_kmeans_lloyd_d(int n, int d, const double *X, int k, const double *C0, int max_iter,
                        double tol, double *C_out, int32_t *labels_out, int32_t *n_iter_out,
                        double *inertia_out) {
    double *Cp = malloc(sizeof(double) * (size_t)k * d), *Cc = malloc(sizeof(double) * (size_t)k * d);
    int32_t *lp = calloc(n, sizeof(int32_t)), *lc = calloc(n, sizeof(int32_t));
    int32_t *cnt = malloc(sizeof(int32_t) * k);
    memcpy(Cc, C0, sizeof(double) * (size_t)k * d);
    int it, converged = 0;
    for (it = 0; it < max_iter; ++it) {
        double *t = Cp; Cp = Cc; Cc = t;
        int32_t *tl = lp; lp = lc; lc = tl;
        orc_kmeans_assign_d(n, d, X, k, Cp, lc, NULL);
        orc_kmeans_update_d(n, d, X, lc, k, Cc, cnt);
        double normc = 0, shift = 0;
        for (size_t e = 0; e < (size_t)k * d; ++e) {
            normc += Cp[e] * Cp[e];
            double df = Cp[e] - Cc[e];
            shift += df * df;
        }
        int conv = 0;
        if (it > 1) {
            conv = 2;
            for (int i = 0; i < n; ++i) if (lc[i] != lp[i]) { conv = 0; break; }
        }
        if (conv == 0 && sqrt(shift) < tol * sqrt(normc)) conv = 1;
        converged = conv;
        if (converged) break;
    }
    if (converged == 1 || it == max_iter) orc_kmeans_assign_d(n, d, X, k, Cc, lc, NULL);
    *inertia_out = orc_kmeans_inertia_d(n, d, X, lc, Cc);
    *n_iter_out = it;
    memcpy(C_out, Cc, sizeof(double) * (size_t)k * d);
    memcpy(labels_out, lc, sizeof(int32_t) * n);
    free(Cp); free(Cc); free(lp); free(lc); free(cnt);
}

/* One Lloyd iteration as used by the CPU baseline timing: assignment in
 * fp32 plus fp64 centroid update; returns the number of changed labels. */
int orc_kmeans_iteration_s(int n, int d, const float *X, int k, float *C, int32_t *labels) {
    int32_t *nl = malloc(sizeof(int32_t) * n);
    orc_kmeans_assign_s(n, d, X, k, C, nl, NULL);
    int changed = 0;
    double *s = calloc((size_t)k * d, sizeof(double));
    int32_t *cnt = calloc(k, sizeof(int32_t));
    for (int i = 0; i < n; ++i) {
        if (nl[i] != labels[i]) ++changed;
        labels[i] = nl[i];
        cnt[nl[i]]++;
        for (int f = 0; f < d; ++f) s[(size_t)nl[i] * d + f] += X[(size_t)i * d + f];
    }
    for (int j = 0; j < k; ++j)
        for (int f = 0; f < d; ++f) C[(size_t)j * d + f] = (float)(s[(size_t)j * d + f] / (cnt[j] ? cnt[j] : 1));
    free(nl); free(s); free(cnt);
    return changed;
}

/* ------------------------------------------------------------------ */
/* Spherical (cosine) k-means                                          */
/* ------------------------------------------------------------------ */
/* The "distance" = "cosine" option of kmeans_options.hpp:111-121, Lloyd
 * iterations (kmeans_lloyd.hpp:106-271, 373-405; kmeans.cpp:681-703,
 * 1065-1098, 1478-1485):
 *   inv_i  = 1 / sqrt(|x_i|^2) (0 for a zero row; |x|^2 one fma chain) --
 *            safe_inv of the row norm;
 *   assign = argmin_j fl(-dot(x_i, c_j)) on the rows as given (strict '<',
 *            ties keep the lower j): the -C A^T GEMM with zero norms, here
 *            the same comparison as fl(-2 dot + 0);
 *   update = per cluster the fp64 sum of the rows, each scaled to
 *            fl(x_i inv_i) when normalise (kmeans_lloyd.hpp:279-300), divided
 *            by max(count, 1), rounded to T; then every centre (and the
 *            initial ones) scaled to unit length: sq = sum c^2 in fp64 in
 *            feature order, c = fl(c / sqrt(sq)) in fp64, a zero row kept
 *            (normalize_rows_inplace of da_utils.cpp:807-853 uses the factor
 *            1 for it).  The reference normalises in T; normalising the
 *            rounded mean in fp64 changes no direction by more than an ulp;
 *   shift / convergence as orc_kmeans_lloyd_s;
 *   inertia = sum_i (1 - fl(dot(x_i, c_{l_i}) inv_i)) with each term in T
 *            (normalise off: 1 - dot), summed in fp64. */
#define ORC_SPH_DEFINE(T, SFX, DOT, SQN, SQRT)                                              \
static void sph_unit_##SFX(T *C, int k, int d) {                                            \
    for (int j = 0; j < k; ++j) {                                                           \
        T *c = C + (size_t)j * d;                                                           \
        double sq = 0;                                                                      \
        for (int f = 0; f < d; ++f) sq = fma((double)c[f], (double)c[f], sq);               \
        const double r = sq > 0 ? 1.0 / sqrt(sq) : 1.0;                                     \
        for (int f = 0; f < d; ++f) c[f] = (T)((double)c[f] * r);                           \
    }                                                                                       \
}                                                                                           \
static void sph_inv_##SFX(int n, int d, const T *X, T *inv) {                               \
    for (int i = 0; i < n; ++i) {                                                           \
        const T sq = SQN(X + (size_t)i * d, d);                                             \
        inv[i] = sq > 0 ? (T)1 / SQRT(sq) : (T)0;                                           \
    }                                                                                       \
}                                                                                           \
void orc_kmeans_assign_sph_##SFX(int n, int d, const T *X, int k, const T *C,               \
                                 int32_t *labels, double *gap) {                            \
    _Pragma("omp parallel for schedule(static)")                                            \
    for (int i = 0; i < n; ++i) {                                                           \
        const T *x = X + (size_t)i * d;                                                     \
        T best = INFINITY; int bj = 0;                                                      \
        double b1 = INFINITY, b2 = INFINITY;                                                \
        for (int j = 0; j < k; ++j) {                                                       \
            const T dt = DOT(x, C + (size_t)j * d, d);                                      \
            const T v = -dt;                                                                \
            if (v < best) { best = v; bj = j; }                                             \
            if (!gap) continue;                                                             \
            double e = 0;                                                                   \
            for (int f = 0; f < d; ++f) e += (double)x[f] * (double)C[(size_t)j * d + f];   \
            e = -e;                                                                         \
            if (e < b1) { b2 = b1; b1 = e; } else if (e < b2) b2 = e;                       \
        }                                                                                   \
        labels[i] = bj;                                                                     \
        if (gap) gap[i] = b2 - b1;                                                          \
    }                                                                                       \
}                                                                                           \
double orc_kmeans_inertia_sph_##SFX(int n, int d, const T *X, const int32_t *labels,        \
                                    const T *C, int normalise) {                            \
    T *inv = malloc(sizeof(T) * (size_t)(n > 0 ? n : 1));                                   \
    sph_inv_##SFX(n, d, X, inv);                                                            \
    double acc = 0;                                                                         \
    for (int i = 0; i < n; ++i) {                                                           \
        const T dt = DOT(X + (size_t)i * d, C + (size_t)labels[i] * d, d);                  \
        const T cs = normalise ? dt * inv[i] : dt;                                          \
        acc += (double)((T)1 - cs);                                                         \
    }                                                                                       \
    free(inv);                                                                              \
    return acc;                                                                             \
}                                                                                           \
void orc_kmeans_sph_lloyd_##SFX(int n, int d, const T *X, int k, const T *C0, int max_iter, \
                                double tol, int normalise, T *C_out, int32_t *labels_out,   \
                                int32_t *n_iter_out, double *inertia_out) {                 \
    T *inv = malloc(sizeof(T) * (size_t)n);                                                 \
    double *Xs = malloc(sizeof(double) * (size_t)n * d);                                    \
    sph_inv_##SFX(n, d, X, inv);                                                            \
    for (int i = 0; i < n; ++i)                                                             \
        for (int f = 0; f < d; ++f) {                                                       \
            const T v = X[(size_t)i * d + f];                                               \
            Xs[(size_t)i * d + f] = (double)(normalise ? v * inv[i] : v);                   \
        }                                                                                   \
    T *Cp = malloc(sizeof(T) * (size_t)k * d), *Cc = malloc(sizeof(T) * (size_t)k * d);     \
    double *Cn = malloc(sizeof(double) * (size_t)k * d);                                    \
    int32_t *lp = calloc(n, sizeof(int32_t)), *lc = calloc(n, sizeof(int32_t));             \
    int32_t *cnt = malloc(sizeof(int32_t) * k);                                             \
    memcpy(Cc, C0, sizeof(T) * (size_t)k * d);                                              \
    sph_unit_##SFX(Cc, k, d);                                                               \
    int it, converged = 0;                                                                  \
    for (it = 0; it < max_iter; ++it) {                                                     \
        T *t = Cp; Cp = Cc; Cc = t;                                                         \
        int32_t *tl = lp; lp = lc; lc = tl;                                                 \
        orc_kmeans_assign_sph_##SFX(n, d, X, k, Cp, lc, NULL);                              \
        orc_kmeans_update_d(n, d, Xs, lc, k, Cn, cnt);                                      \
        for (size_t e = 0; e < (size_t)k * d; ++e) Cc[e] = (T)Cn[e];                        \
        sph_unit_##SFX(Cc, k, d);                                                           \
        double normc = 0, shift = 0;                                                        \
        for (size_t e = 0; e < (size_t)k * d; ++e) {                                        \
            normc += (double)Cp[e] * (double)Cp[e];                                         \
            const double df = (double)Cp[e] - (double)Cc[e];                                \
            shift += df * df;                                                               \
        }                                                                                   \
        int conv = 0;                                                                       \
        if (it > 1) {                                                                       \
            conv = 2;                                                                       \
            for (int i = 0; i < n; ++i) if (lc[i] != lp[i]) { conv = 0; break; }            \
        }                                                                                   \
        if (conv == 0 && sqrt(shift) < tol * sqrt(normc)) conv = 1;                         \
        converged = conv;                                                                   \
        if (converged) break;                                                               \
    }                                                                                       \
    if (converged == 1 || it == max_iter) orc_kmeans_assign_sph_##SFX(n, d, X, k, Cc, lc, NULL); \
    *inertia_out = orc_kmeans_inertia_sph_##SFX(n, d, X, lc, Cc, normalise);                \
    *n_iter_out = it;                                                                       \
    memcpy(C_out, Cc, sizeof(T) * (size_t)k * d);                                           \
    memcpy(labels_out, lc, sizeof(int32_t) * n);                                            \
    free(inv); free(Xs); free(Cp); free(Cc); free(Cn); free(lp); free(lc); free(cnt);       \
}
ORC_SPH_DEFINE(float, s, dot_s, sqnorm_s, sqrtf)
ORC_SPH_DEFINE(double, d, dot_d, sqnorm_d, sqrt)

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
