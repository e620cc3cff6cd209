/*
 * aoclda_b200_ext.h -- B200-specific entry points of libaoclda_b200.so.
 *
 * None of these has a counterpart in the AOCL-DA C API; they expose what a
 * GPU library needs beyond it (stream binding, kernel timing, access to the
 * k-means initial centres).  Plain C types only.
 */
#ifndef AOCLDA_B200_EXT_H
#define AOCLDA_B200_EXT_H

#include "aoclda_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bind the handle's work to a caller-owned CUDA stream (a cudaStream_t passed
 * as void*); NULL restores the handle's own non-blocking stream.  Calls still
 * return only after their results are complete. */
da_status da_b200_set_stream(da_handle handle, void *stream);

/* Recreate the handle's own stream with a CUDA stream priority: 0 is the
 * default, negative values are higher priorities (clamped to the device's
 * range).  Blocks of a higher-priority stream's kernels are scheduled first
 * as SMs free up, so that a latency-critical handle's work overtakes a busy
 * one's.  Work in flight on the old stream completes first. */
da_status da_b200_set_stream_priority(da_handle handle, da_int priority);

/* Kernel timing: when enabled, every launch of the named hot kernels is
 * bracketed by CUDA events on the handle's stream and accumulated.  Intended
 * for measurement (it serialises launches); off by default. */
da_status da_b200_set_kernel_timing(da_handle handle, da_int enable);
/* Total milliseconds and launch count accumulated for `kernel` ("knn_chunks",
 * "knn_merge", "kmeans_assign", "kmeans_sort", "kmeans_update", ...). */
da_status da_b200_get_kernel_time(da_handle handle, const char *kernel, double *total_ms,
                                  da_int *launches);
da_status da_b200_reset_kernel_time(da_handle handle);

/* Free and total device memory, in bytes, of the current device
 * (da_status_arch_not_supported without one).  For admission control by
 * callers that keep several handles busy at once. */
da_status da_b200_device_memory(unsigned long long *free_bytes, unsigned long long *total_bytes);

/* kNN: give `handle` the training data (and labels / targets) already set on
 * `source` -- same precision, storage order and device -- without a second
 * device copy: both handles hold the same device rows (and the tensor-core
 * bf16 copies when `source` has built them, i.e. after its first tensor-core
 * search), which stay allocated until the last of them lets go.  `handle`
 * keeps its own options and per-call buffers, so the two handles can search
 * at the same time on their own streams.  Host pointers are taken as
 * da_nn_set_data would take them.  A later da_nn_set_data on either handle
 * gives that handle fresh device buffers.  Replaces, for a server with one
 * handle per worker, a da_nn_set_data_{s,d} (nearest_neighbors_public.cpp)
 * per worker. */
da_status da_b200_nn_share_data(da_handle handle, da_handle source);

/* Named statistics of the last call: "relabelled_rows" (k-means rows of the
 * last tensor-core assignment whose label needed the exact fp32 re-score),
 * "tensor_core" (1 when the last k-means compute used the tensor cores). */
da_status da_b200_get_stat(da_handle handle, const char *name, double *value);

/* k-means: run only the configured initialisation method ("initialization
 * method", "seed", "n_clusters") on the data set and write the n_clusters x
 * n_features initial centres to C (storage order of the handle, leading
 * dimension ldc).  The same centres are the starting point of
 * da_kmeans_compute_? with n_init = 1. */
da_status da_b200_kmeans_init_centres_d(da_handle handle, double *C, da_int ldc);
da_status da_b200_kmeans_init_centres_s(da_handle handle, float *C, da_int ldc);

/* No counterpart in the AOCL-DA API.  Steps of a k-means (Lloyd) fit of one
 * fp32 data set split row-wise over several handles (one per process / GPU),
 * for a caller that runs the Lloyd loop of da_kmeans_compute_s and reduces
 * one integer buffer over the processes per iteration.  Every handle holds
 * its shard (da_kmeans_set_data_s) and the same options.  The results --
 * labels, centres, iteration count -- equal those of da_kmeans_compute_s
 * on the unsplit data with supplied initial centres and n_init = 1 (the
 * inertia to fp64 rounding: the shards' inertias are added).
 *
 * da_b200_kmeans_shard_colmax_s: max |x| per feature over the shard
 *   (n_features floats); the caller takes the element-wise maximum.
 * da_b200_kmeans_shard_begin_s: starts a fit from the initial centres
 *   (k x d row-major, host) with the whole data set's column maxima and row
 *   count, which fix the fixed-point scales of the centroid sums.
 * da_b200_kmeans_shard_partial_s: assigns the shard's rows to the current
 *   centres (the plain fp32 labels) and writes, on the handle's stream, into
 *   the caller's DEVICE buffer acc of DA_B200_KMEANS_SHARD_ACC_LEN(k, d)
 *   int64: [0, k*d) the fixed-point centroid sums, [k*d, k*d+k) the counts,
 *   [k*d+k] = 1 if a label changed since the previous partial step.  The
 *   element-wise sum of acc over all shards (an integer all-reduce, exact in
 *   any order) is the unsplit data's.
 * da_b200_kmeans_shard_finalize_s: the new centres from the reduced acc
 *   (centre j, feature f = (double)sum * 2^-s_f / max(count, 1) rounded to
 *   fp32, s_f = min(62 - L, 44) - E_f clamped to [-126, 127], n <= 2^L,
 *   colmax[f] < 2^E_f); scalars[0] = sum |C_old|^2, scalars[1] =
 *   sum |C_old - C_new|^2 (fp64, a fixed order); flags[0] = any label
 *   changed on any shard, flags[1] = empty clusters.  Synchronises.
 * da_b200_kmeans_shard_inertia_s: the shard's inertia against the current
 *   centres (fp64), with relabel != 0 after a new assignment to them.
 * da_b200_kmeans_shard_result_s: current centres (k x d row-major) and the
 *   shard's labels; either pointer may be null. */
#define DA_B200_KMEANS_SHARD_ACC_LEN(k, d) ((size_t)(k) * (size_t)(d) + (size_t)(k) + 1u)
da_status da_b200_kmeans_shard_colmax_s(da_handle handle, float *colmax);
da_status da_b200_kmeans_shard_begin_s(da_handle handle, const float *colmax_global,
                                       da_int n_global, const float *centres);
da_status da_b200_kmeans_shard_partial_s(da_handle handle, long long *acc);
da_status da_b200_kmeans_shard_finalize_s(da_handle handle, const long long *acc,
                                          double *scalars, da_int *flags);
da_status da_b200_kmeans_shard_inertia_s(da_handle handle, da_int relabel, double *inertia);
da_status da_b200_kmeans_shard_result_s(da_handle handle, float *centres, da_int *labels);

/* No counterpart in the AOCL-DA API.  Lloyd k-means on n_inst independent
 * fp32 data sets at once (different n, d and k): instance i has n_samples[i]
 * rows of n_features[i] values (row-major host array A[i], leading dimension
 * lda[i]) and n_clusters[i] initial centres (row-major k x d host array
 * C_init[i]).  Every instance gives exactly what da_kmeans_compute_s gives
 * for that data with "precision mode" = "plain", "initialization method" =
 * "supplied", n_init = 1, the same max_iter and convergence tolerance, and
 * "empty clusters" = "ignore": centres (C_out[i], k x d row-major), labels
 * (labels_out[i]), iteration count, convergence code (0: max_iter reached,
 * 1: centre shift below tol, 2: labels unchanged) and inertia (fp64 sum, to
 * within rounding).  All instances advance together on the device: in each
 * Lloyd iteration persistent blocks take (instance, tile) items off work
 * queues (the assignment, then the update of the changed rows' centroid
 * sums), and the whole fit is one CUDA graph.  The assignment's tile shape
 * for each (row width, k range) is picked by timing the candidates the
 * first time the process meets that shape (the choice is kept; results do
 * not depend on it).  Limits: k <= n and k * d <= 8192 per instance; finite
 * data (else da_status_invalid_input).  `stream`: a cudaStream_t the inputs
 * are uploaded on (NULL: the legacy default stream); the call returns when
 * the results are on the host. */
da_status da_b200_kmeans_batched_s(da_int n_inst, const da_int *n_samples,
                                   const da_int *n_features, const da_int *n_clusters,
                                   const float *const *A, const da_int *lda,
                                   const float *const *C_init, da_int max_iter, double tol,
                                   float *const *C_out, da_int *const *labels_out,
                                   da_int *n_iter, double *inertia, da_int *converged,
                                   void *stream);

/* Device times, in milliseconds, of the calling thread's last successful
 * da_b200_kmeans_batched_s call: the upload of the data sets and initial
 * centres, the fit (the CUDA graph of all Lloyd iterations, the final
 * relabelling and the inertia) and the download of centres and labels. */
da_status da_b200_kmeans_batched_timing(double *upload_ms, double *fit_ms, double *download_ms);

/* No counterpart in the AOCL-DA API.  Brute-force euclidean k nearest
 * neighbours for callers that cannot allocate device memory (code running
 * inside a device allocator or memory-pool callback, real-time pipelines that
 * forbid allocation after start-up, hosts whose device memory another
 * framework has reserved).  It allocates nothing: its working memory is one
 * fixed array of DA_B200_KNN_NOALLOC_SCRATCH_BYTES in the library's device
 * code, held on every GPU that loads the library until the process exits.
 *
 * X (n x d), Q (nq x d): row-major fp32 device arrays with the same leading
 * dimension ld (a multiple of 4, ld >= d), 16-byte aligned, each holding
 * rows x ld elements.  Results, on the device: dist (nq x k, row-major) and
 * ind (nq x k, 0-based training-row indices), the same neighbours and
 * distances, bit for bit, as da_nn_kneighbors_s with metric "euclidean" on
 * row-major data; ties between equal distances go to the lower index.
 * 1 <= k <= min(n, 256).  nq * k * 8 + 256 bytes must fit in the scratch
 * array (else da_status_invalid_array_dimension).
 *
 * The work is enqueued on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and the call returns without waiting for it.  The first call on a
 * device looks up the scratch array's address; make it before any stream
 * capture on that device.  The address is kept per device and context: after
 * cudaDeviceReset (or with another context current) the next call looks it
 * up again.  Calls share the scratch array: calls whose work overlaps on the
 * GPU race on it. */
#define DA_B200_KNN_NOALLOC_SCRATCH_BYTES (32u << 20)
da_status da_b200_knn_euclidean_noalloc_s(const float *X, da_int n, const float *Q, da_int nq,
                                          da_int d, da_int ld, da_int k, float *dist,
                                          da_int *ind, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* AOCLDA_B200_EXT_H */
