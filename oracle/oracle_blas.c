/* TEST INFRASTRUCTURE ONLY (never linked by the product): the reference's
 * CPU Lloyd iteration restated with a BLAS gemm, timed by bench.py as the CPU
 * baseline ("port") of the k-means workload.
 *
 * Structure of kmeans_lloyd.hpp:106-271 (lloyd_iteration, multi-threaded
 * branch): the rows are cut into blocks of 512 (float) / 256 (double) rows
 * (max_block_size, kmeans.cpp:497-517) handed out to OpenMP threads with a
 * dynamic schedule; per block one gemm forms W = -2 C A_block^T (C column-
 * major n_clusters x n_features, A row-major, i.e. the reference's
 * A_blas_trans = NoTrans case); the argmin over the clusters of W + |c_j|^2
 * with a strict '<' (ties keep the lower index,
 * kmeans_kernels.cpp:209-234); the label counts and the sums of the rows of
 * each cluster accumulate in thread-local arrays in the working precision
 * (kmeans_lloyd.hpp:275-361, row-major branch) and are merged under a lock
 * (:209-228); then the centres are scaled by max(count, 1)
 * (:364-405).  The gemm is the caller's cblas_sgemm (a function pointer:
 * OpenBLAS in bench.py, set to one thread per call, as BLAS runs inside the
 * reference's parallel region).  The argmin is written as a min pass and a
 * first-equal pass so that the compiler vectorises it (the reference uses
 * AVX-512 intrinsics); the label it gives is the strict-'<' label. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef void (*sgemm_fn)(int, int, int, int, int, int, float, const float *, int,
                         const float *, int, float, float *, int);

enum { COL_MAJOR = 102, NO_TRANS = 111 };

/* n_iter Lloyd iterations from C (k x d row-major, updated in place) over A
 * (n x d row-major, ld d); labels (n) hold the previous labels on entry and
 * the last iteration's labels on exit.  Returns the number of labels that
 * changed in the last iteration, or -1 on an allocation failure. */
int orc_lloyd_blas_s(int n, int d, const float *A, int k, float *C, int32_t *labels,
                     int n_iter, void *gemm, int n_threads) {
    const int bsz = 512;
    const int n_blocks = (n + bsz - 1) / bsz;
#ifdef _OPENMP
    if (n_threads < 1) n_threads = omp_get_max_threads();
#else
    n_threads = 1;
#endif
    float *Ccm = malloc(sizeof(float) * (size_t)k * d);
    float *cn = malloc(sizeof(float) * (size_t)k);
    float *sums = malloc(sizeof(float) * (size_t)k * d);
    int32_t *cnt = malloc(sizeof(int32_t) * (size_t)k);
    if (!Ccm || !cn || !sums || !cnt) {
        free(Ccm); free(cn); free(sums); free(cnt);
        return -1;
    }
    int changed = 0;
    for (int it = 0; it < n_iter; ++it) {
        for (int j = 0; j < k; ++j) {
            float s = 0.f;
            for (int f = 0; f < d; ++f) {
                const float c = C[(size_t)j * d + f];
                Ccm[j + (size_t)f * k] = c;
                s = fmaf(c, c, s);
            }
            cn[j] = s;
        }
        memset(sums, 0, sizeof(float) * (size_t)k * d);
        memset(cnt, 0, sizeof(int32_t) * (size_t)k);
        changed = 0;
#pragma omp parallel num_threads(n_threads) reduction(+ : changed)
        {
            float *W = malloc(sizeof(float) * (size_t)k * bsz);
            float *lsum = calloc((size_t)k * d, sizeof(float));
            int32_t *lcnt = calloc((size_t)k, sizeof(int32_t));
#pragma omp for schedule(dynamic) nowait
            for (int b = 0; b < n_blocks; ++b) {
                const int i0 = b * bsz;
                const int bs = (i0 + bsz <= n) ? bsz : n - i0;
                ((sgemm_fn)gemm)(COL_MAJOR, NO_TRANS, NO_TRANS, k, bs, d, -2.0f, Ccm, k,
                                 A + (size_t)i0 * d, d, 0.0f, W, k);
                for (int i = 0; i < bs; ++i) {
                    const float *w = W + (size_t)i * k;
                    float m = w[0] + cn[0];
                    for (int j = 1; j < k; ++j) {
                        const float v = w[j] + cn[j];
                        m = v < m ? v : m;
                    }
                    int lab = 0;
                    for (int j = 0; j < k; ++j)
                        if (w[j] + cn[j] == m) { lab = j; break; }
                    if (labels[i0 + i] != lab) ++changed;
                    labels[i0 + i] = lab;
                    lcnt[lab] += 1;
                    const float *x = A + (size_t)(i0 + i) * d;
                    float *dst = lsum + lab; /* centres column-major */
                    for (int f = 0; f < d; ++f) dst[(size_t)f * k] += x[f];
                }
            }
#pragma omp critical
            {
                for (int j = 0; j < k; ++j) cnt[j] += lcnt[j];
                for (size_t e = 0; e < (size_t)k * d; ++e) sums[e] += lsum[e];
            }
            free(W); free(lsum); free(lcnt);
        }
        for (int j = 0; j < k; ++j) {
            const float c = (float)(cnt[j] > 0 ? cnt[j] : 1);
            for (int f = 0; f < d; ++f) C[(size_t)j * d + f] = sums[j + (size_t)f * k] / c;
        }
    }
    free(Ccm); free(cn); free(sums); free(cnt);
    return changed;
}
