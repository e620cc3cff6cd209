// Host-callable launchers of the B200 kernels.  All pointers are DEVICE
// pointers; every launcher enqueues on `stream` and returns the launch error.
//
// Device data layout (chosen for sm_100a, not taken from the reference):
//   * a sample matrix is row-major, rows x ld with ld = d rounded up to a
//     multiple of 4 elements (16-byte rows for fp32, 32-byte for fp64), pad
//     columns are zero;
//   * labels / indices are int32;
//   * centroid sums are fp64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace b200 {

inline int pad4(int d) { return (d + 3) & ~3; }

// Element-wise metric families of the direct (non-GEMM) distance engine.
// The accumulation order of each family follows the AOCL-DA micro-kernels
// (source/core/metrics/metrics_kernels.hpp).
enum AccKind : int {
    ACC_SQEUC = 0,     // sum (a-b)^2, two accumulators (metrics_kernels.hpp:419-496)
    ACC_DOT = 1,       // sum a*b, one fma chain (cosine kernel, metrics_kernels.hpp:670-749)
    ACC_MANHATTAN = 2, // sum |a-b|, one add chain (metrics_kernels.hpp:584-666)
    ACC_MINKOWSKI = 3  // sum |a-b|^p, one add chain (metrics_kernels.hpp:752-827)
};

// Post-operation applied to an accumulated pair value.
enum PostKind : int {
    POST_NONE = 0,       // squared euclidean / manhattan: value as accumulated
    POST_SQRT = 1,       // euclidean
    POST_COSINE = 2,     // 1 - dot / (|x| |y|)
    POST_GEMM_SQ = 3,    // |x|^2 + |y|^2 - 2 dot (GEMM-form squared euclidean)
    POST_GEMM_SQRT = 4,  // sqrt of POST_GEMM_SQ (no clamp, as the reference)
    POST_POW = 5,        // (sum)^(1/p)
    POST_NEG = 6,        // -dot: inner product ranked largest-first
    POST_GEMM_SQ_CLAMP = 7 // max(0, GEMM-form squared euclidean) -- kNN selection key
};


// ---------------------------------------------------------------- ingest --
// Dense column-major (rows x cols, ld = rows) -> padded row-major (rows x ldo).
template <typename T>
cudaError_t launch_colmajor_to_rowmajor(const T *src, int rows, int cols, T *dst, int ldo,
                                        cudaStream_t s);
// Row-major (rows x ldo) -> dense column-major (rows x cols, ld = ldc).
template <typename T>
cudaError_t launch_rowmajor_to_colmajor(const T *src, int rows, int cols, int ldi, T *dst,
                                        long ldc, cudaStream_t s);

// ------------------------------------------------------------- row norms --
// out[i] = sum_j x_ij^2 as a sequential fma chain in j (the order of the
// reference's norm loops, euclidean_gemm_distance.cpp:65-95).
template <typename T>
cudaError_t launch_row_sqnorms(const T *X, int ld, int rows, int d, T *out, cudaStream_t s);
// out[i] = ||x_i||_2 (accumulated in fp64), replaced by 1 when <= eps
// (cosine_distance.cpp:117-146).
template <typename T>
cudaError_t launch_row_norms_eps1(const T *X, int ld, int rows, int d, T *out,
                                  cudaStream_t s);

// --------------------------------------------------------- pairwise tile --
struct PairwiseArgs {
    int acc;       // AccKind
    int post;      // PostKind
    int kc;        // KC slice length of the reference's blocking (multiple of 4)
    double p;      // Minkowski exponent
    bool x_is_y;   // cosine / gemm: diagonal forced to 0
    bool out_rowmajor; // D row-major (m x n, ld = n) or column-major (ld = m)
    // radius search (row-major D only): with `hits`, every stored value
    // D(i, j) <= thr also counts into hits[i * radius_chunks(n) + j / RADIUS_CHUNK]
    // (integer atomics; hits zeroed by the caller)
    double thr = 0.0;
    int *hits = nullptr;
};
// D(i,j) = dist(x_i, y_j), i < m (rows of X), j < n (rows of Y).
template <typename T>
cudaError_t launch_pairwise(const T *X, int ldx, int m, const T *Y, int ldy, int n, int d,
                            const T *xn, const T *yn, const PairwiseArgs &a, T *D,
                            cudaStream_t s);

// Radius neighbours from a block of distances D (rows x n, row-major, ld),
// each row cut into radius_chunks(n) chunks of RADIUS_CHUNK columns: the
// ordered compaction (index order) of each (row, chunk) piece's (column,
// value) pairs with D <= thr at out offsets start[row * chunks + chunk] (one
// CTA per piece).
constexpr int RADIUS_CHUNK = 16384;
int radius_chunks(int n);
template <typename T>
cudaError_t launch_radius_emit(const T *D, int rows, int n, size_t ld, T thr,
                               const long long *start, int *idx, T *val, cudaStream_t s);
// The output offsets of all (row, chunk) pieces from their hit counts (hits,
// made by the distance kernel: PairwiseArgs::hits) in one launch (a chained
// scan in (row, chunk) order over groups of 32 pieces, dist_simt.cu):
// start[row * chunks + chunk] = the hits of the pieces before it, total[0] =
// all hits.  Its waits on other warps are bounded: err[0] = 1 when one ran
// out (test_wait: the first group never publishes and the waits run out at
// once).  work: radius_scan_work_bytes(rows, n).  D, ld and thr are unused.
template <typename T>
cudaError_t launch_radius_count_scan(const T *D, int rows, int n, size_t ld, T thr, void *work,
                                     long long *start, long long *total, int *err, int test_wait,
                                     cudaStream_t s, const int *hits = nullptr);
size_t radius_scan_work_bytes(int rows, int n);

// ------------------------------------------------------------ kNN fused --
struct KnnArgs {
    int acc, post, kc;
    double p;
    int k;          // neighbours requested
    int chunk_rows; // train rows per chunk (multiple of the tile width)
    int n_chunks;
};
// Stage 1: per (query tile, train chunk) running top-k of the selection key,
// written as sorted (key, index) lists: part_key[(q * n_chunks + c) * k + r].
template <typename T>
cudaError_t launch_knn_chunks(const T *Q, int ldq, int nq, const T *X, int ldx, int nx,
                              int d, const T *qn, const T *xn, const KnnArgs &a,
                              T *part_key, int *part_idx, int *err_flag, cudaStream_t s);
// Stage 2: merge the n_chunks lists of every query into the final sorted
// top-k; out_key receives the value returned to the user (sqrt applied for
// euclidean, sign restored for inner product).
template <typename T>
cudaError_t launch_knn_merge(const T *part_key, const int *part_idx, int nq, int n_chunks,
                             int k, int out_transform, T *out_key, int *out_idx,
                             cudaStream_t s);
// Which tile widths the fused kernel uses; chunk_rows must be a multiple.
int knn_tile_rows_train(bool fp64);
int knn_max_k(bool fp64);

// ---------------------------------------------- kNN tensor-core pass ---
// fp32 euclidean / squared euclidean / cosine: bf16x3 tcgen05 candidate pass with a
// certified threshold per query, exact re-score of the survivors in the plain
// kernel's order.  Results (q-major, as launch_knn_merge) equal the plain
// path's; queries the pass cannot certify are flagged in `fallback`
// (*n_fallback of them) for the plain path.
int knn_tc_supported(int nx, int d, int k);
size_t knn_tc_list_cap();                   // list entries per query
size_t knn_tc_query_bytes(int nq, int d);   // size of qbuf
int *knn_tc_counts(void *qbuf, int nq, int d); // per-query list lengths inside qbuf
// dst[i] = src[idx[i]] (rows of ld floats); out[idx[i]] = (key, ind)[i] (rows of k)
cudaError_t launch_rows_gather(const float *src, int ld, const int *idx, int m, float *dst,
                               cudaStream_t s);
cudaError_t launch_results_scatter(const float *key, const int *ind, const int *idx, int m, int k,
                                   float *out_key, int *out_idx, cudaStream_t s);
cudaError_t launch_knn_tc_train_prep(const float *X, int ld, int nx, int d, void *Xh, void *Xl,
                                     int ldbf, float *xnorm2, float *xmax, cudaStream_t s);
// Cosine distance instead (the plain path's value 1 - x.q / (|x| |q|)): the
// plain path's norms of the training rows (xnorm) and of this batch's queries
// (qnorm), and the reciprocals of the former (xinv, launch_recip).
struct KnnTcCosine {
    const float *xnorm, *xinv, *qnorm;
};
cudaError_t launch_recip(const float *v, int n, float *out, cudaStream_t s);
cudaError_t launch_knn_tc(const float *X, const void *Xh, const void *Xl, const float *xnorm2,
                          const float *xmax, int nx, int ld, int ldbf, int d, const float *Q,
                          int nq, int k, int kc, int take_sqrt, void *qbuf, void *list,
                          int *fallback, int *n_fallback, int *err, float *out_key,
                          int *out_idx, cudaStream_t s, const KnnTcCosine *cosine = nullptr);

// ------------------------------------------------------------- k-means ---
struct KmeansWork {
    // per-iteration device scratch owned by the handle
    int *labels;          // n
    int *labels_prev;     // n
    int *counts;          // k
    int *block_counts;    // n_blocks * k
    int *offsets;         // k + 1
    int *sorted_rows;     // n
    double *chunk_sums;   // n_seg_chunks_max * ld
    int *seg_chunk_start; // k + 1  (first chunk of each cluster)
    double *scalars;      // [0]=normc^2 [1]=shift^2 [2]=inertia ...
    int *flags;           // [0]=labels changed [1]=n_empty
};
int kmeans_assign_block_rows();
int kmeans_max_clusters_fused();
// Lloyd assignment: label_i = argmin_j (|c_j|^2 - 2 x_i.c_j), ties -> lower j.
// Also writes per-block label histograms (for the counting sort) and raises
// flags[0] when a label differs from labels_prev (if labels_prev != null).
template <typename T>
cudaError_t launch_kmeans_assign(const T *X, int ldx, int n, int d, const T *C, int ldc,
                                 int k, const T *cnorm, int *labels, const int *labels_prev,
                                 int *block_counts, int *flags, cudaStream_t s);
// Counting sort of rows by label: offsets (exclusive scan of counts) and a
// stable scatter of row ids (rows of one cluster stay in ascending order).
cudaError_t launch_kmeans_sort(const int *labels, int n, int k, const int *block_counts,
                               int *counts, int *offsets, int *seg_chunk_start,
                               int seg_rows, int *sorted_rows, int *flags, cudaStream_t s);
// Deterministic centroid update: fp64 sums over fixed row chunks of every
// cluster, combined in chunk order; C_new = sum / max(count,1) (an empty
// cluster becomes the zero vector, kmeans_lloyd.hpp:364-377).  Also computes
// |C_prev|_F^2 and |C_prev - C_new|_F^2 in fp64 into scalars[0], scalars[1].
template <typename T>
cudaError_t launch_kmeans_update(const T *X, int ldx, int n, int d, int k,
                                 const int *sorted_rows, const int *offsets,
                                 const int *seg_chunk_start, int seg_rows, double *chunk_sums,
                                 const int *counts, const T *C_prev, T *C_new, int ldc,
                                 double *scalars, int *flags, cudaStream_t s);
// Fixed-point centroid update for fp32 data (order-independent integer sums,
// so deterministic without sorting): supported when the shared-memory
// accumulators (k x d int64) fit.  launch_col_absmax gives the per-feature
// max |x| (as float bits) and a non-finite flag, from which the host derives
// scale[f] = 2^s_f (fp32) and inv_scale[f] = 2^-s_f (fp64), with
// n max|x_f| 2^s_f < 2^62 and max|x_f| 2^s_f < 2^44.  accum (fx_accum_bytes) holds
// two sets of global sums and counts used alternately (parity): the update
// of parity p reads set p and clears set 1-p, so both must be zero before
// the first call.  ticket is a zero-initialised counter left at zero.
int fx_update_supported(int k, int d);
size_t fx_accum_bytes(int k, int d);
cudaError_t launch_col_absmax(const float *X, int ld, int n, int d, unsigned *colmax,
                              int *nonfinite, cudaStream_t s);
cudaError_t launch_kmeans_update_fx(const float *X, int ld, int n, int d, int k,
                                    const int *labels, const float *scale,
                                    const double *inv_scale, void *accum, int parity,
                                    const float *C_prev, float *C_new, int *counts,
                                    double *block_partials, double *scalars, int *flags,
                                    unsigned *ticket, cudaStream_t s);
// The rows whose label changed in an assignment, appended by the assignment
// kernels when `count` is set: count[0] counts them all, the first `cap` are
// listed as (rows, olds, news).  count[0] must be 0 on entry.
struct ChangeList {
    int *count = nullptr;
    int *rows = nullptr, *olds = nullptr, *news = nullptr;
    int cap = 0;
};
// Device state of a Lloyd loop run as a CUDA graph (WHILE node): the next
// iteration's index, the limits, and the outcome written by the finalize.
struct LloydLoopState {
    int it;       // index of the iteration the next finalize ends
    int max_iter;
    int conv;     // 0, 1 (centre shift below tol), 2 (no label changed)
    int n_iter;   // the host loop's iteration count at its end
    double tol;
};
// One Lloyd update inside the graph loop: new centres in place in C, the
// convergence test of iteration ls->it, and cudaGraphSetConditional(cond, 0)
// when the loop ends.  Accumulator set 0 holds the sums and counts of the
// labels before this iteration's assignment; with at most chg.cap changed
// rows they are brought up to date by adding each changed row's fixed-point
// features to its new cluster and subtracting them from its old one (exact
// integer arithmetic: the same sums as a recount), else recounted over all
// rows.  The finalize re-arms the iteration's counters: flags[0..1],
// rearm[0] and rearm[2] (the relabel list's counts), chg.count.
//
// amb: the rows the tensor-core pass left uncertified (at most KM_AMB_MAXC
// candidate clusters each, or none: scan every cluster); they get their exact
// fp32 labels here (the plain path's fma order against the centres C and
// their norms cnorm), in the same launch as the delta update.  recount: one
// int the launch sets to 1 when the sums are recounted instead (the changed
// certified rows plus the listed rows exceed chg.cap).
struct AmbList {
    const int *rows = nullptr, *cand = nullptr, *ncand = nullptr, *count = nullptr;
};
constexpr int KM_AMB_MAXC = 4; // candidate clusters kept per uncertified row
cudaError_t launch_kmeans_update_fx_loop(const float *X, int ld, int n, int d, int k,
                                         int *labels, const float *scale,
                                         const double *inv_scale, void *accum, float *C,
                                         int *counts, double *block_partials, double *scalars,
                                         int *flags, unsigned *ticket, LloydLoopState *ls,
                                         unsigned long long cond, const ChangeList &chg,
                                         int *rearm, const float *cnorm, const AmbList &amb,
                                         int *recount, cudaStream_t s);
// One shard's share of a data set split across processes, packed for one
// integer all-reduce: acc[0, k*d) the fixed-point sums (two's complement,
// from zero), acc[k*d, k*d+k) the counts, acc[k*d+k] = (*changed != 0).
// counts is int scratch of k entries.
cudaError_t launch_kmeans_sums_fx(const float *X, int ld, int n, int d, int k, const int *labels,
                                  const float *scale, long long *acc, int *counts,
                                  const int *changed, cudaStream_t s);
// New centres from the all-reduced acc (layout above): the single-device
// finalize with int64 counts; flags[1] += empty clusters.
cudaError_t launch_kmeans_finalize_shards(int k, int d, int ld, const long long *acc,
                                          const double *inv_scale, const float *C_prev,
                                          float *C_new, double *block_partials, double *scalars,
                                          int *flags, unsigned *ticket, cudaStream_t s);
// Raises (never lowers) func's dynamic shared-memory limit on the current
// device, once per size (thread-safe).
cudaError_t ensure_smem_limit(const void *func, size_t smem);

// ------------------------------------------------------------ IVF-flat ---
// Scan of the probed inverted lists (exact top-k in (key, global index)
// order).  X: list-ordered rows (ld a multiple of 4), xn their squared norms,
// gid their global indices, loff the n_list + 1 row offsets of the lists;
// probe: n_probe list ids per query.  The key and the output distance by
// `out`: IVF_OUT_SQ / IVF_OUT_SQRT the GEMM-form squared distance (its
// square root where non-negative), IVF_OUT_IP key -q.x and distance q.x,
// IVF_OUT_COS key -q.x and distance 1 - q.x (rows and queries normalised).
// Outputs q-major (q * k + r): index -1 and the distance of an infinite key
// (+inf; -inf for the inner product) for empty slots.
enum { IVF_OUT_SQ = 0, IVF_OUT_SQRT = 1, IVF_OUT_IP = 2, IVF_OUT_COS = 3 };
size_t ivf_scan_smem(int k, bool fp64);
template <typename T>
cudaError_t launch_ivf_scan(const T *Q, const T *qn, int ld, int nq, const int *probe,
                            int n_probe, const long long *loff, const T *X, const T *xn,
                            const int *gid, int k, int out, T *out_d, int *out_i,
                            cudaStream_t s);
// Squared row norms of the centres (sequential fma chain over features).
template <typename T>
cudaError_t launch_centre_norms(const T *C, int ldc, int k, int d, T *out, cudaStream_t s);
// Inertia sum_i |x_i - c_{l_i}|^2 accumulated in fp64 (fixed block order).
template <typename T>
cudaError_t launch_kmeans_inertia(const T *X, int ldx, int n, int d, const T *C, int ldc,
                                  const int *labels, double *block_partials, double *out,
                                  cudaStream_t s);
// ------------------------------------------- spherical (cosine) k-means ---
// Inverse row norms inv_i = 1 / sqrt(sqnorm_i) (0 for a zero row) and, when
// Xs is given, the normalised rows Xs = fl(x_i inv_i) (same layout as X,
// padding columns zero).
template <typename T>
cudaError_t launch_sph_data(const T *X, int ld, int n, int d, const T *sqnorm, T *inv, T *Xs,
                            cudaStream_t s);
// Centre rows scaled to unit length in place: c = fl(c / sqrt(sum c^2)) in
// fp64 (a zero row stays zero).  With C_prev, scalars[0] = |C_prev|_F^2 and
// scalars[1] = |C_prev - C|_F^2 of the normalised C (fixed order).
template <typename T>
cudaError_t launch_sph_centres(const T *C_prev, T *C, int k, int d, int ld, double *block_partials,
                               double *scalars, cudaStream_t s);
// Inertia sum_i (1 - cos_i), cos_i = fl(dot(x_i, c_{l_i}) inv_i) (inv null:
// the dot itself); the dot is one fma chain in T, the sum fp64.
template <typename T>
cudaError_t launch_sph_inertia(const T *X, int ld, int n, int d, const T *C, const int *labels,
                               const T *inv, double *block_partials, double *out, cudaStream_t s);
// In place on D (m x k, row- or column-major, holding -dot as the pairwise
// POST_NEG output): D = 1 - clamp(dot inv_i, -1, 1), inv_i = 1 / sqrt(sqnorm_i)
// (0 for a zero row; sqnorm null: inv_i = 1).
template <typename T>
cudaError_t launch_sph_transform(T *D, int m, int k, bool rowmajor, const T *sqnorm,
                                 cudaStream_t s);
// k-means++ distances of every row to `t` candidate rows:
// D[c*n + i] = (|x_i|^2 + |x_cand|^2) - 2 x_i.x_cand (GEMM form, no clamp);
// with `cosine` the spherical distance max(0, 1 - cos) of cos_dist_kpp
// (xinv: the rows' inverse norms, or null for data used as given).
template <typename T>
cudaError_t launch_kpp_dist(const T *X, int ldx, int n, int d, const T *xnorm,
                            const int *cand, int t, T *D, cudaStream_t s,
                            const T *xinv = nullptr, int cosine = 0);
// For each candidate c: cost_c = sum_i max(0, min(w_i, D_ci)) (fp64, fixed order).
template <typename T>
cudaError_t launch_kpp_cost(const T *w, const T *D, int n, int t, double *block_partials,
                            double *cost, cudaStream_t s);
// w_i = max(0, min(w_i, D_ci)) for the chosen candidate (in place).
template <typename T>
cudaError_t launch_kpp_update(T *w, const T *Dc, int n, int chosen, cudaStream_t s);
// Device-side k-means++ draws (kmeans_kpp.cu): weights grouped in blocks
// of 2,048 (kpp_num_blocks(n) block sums).
int kpp_num_blocks(int n);
// w_i = 0 where negative, not finite or i == first; block sums; flag[0] |= 1
// when a weight is positive.
template <typename T>
cudaError_t launch_kpp_clamp(T *w, int n, int first, double *bs, int *flag, cudaStream_t s);
// The rows std::discrete_distribution over w gives for the nt canonical draws
// U[0..nt) (cand), uncertified draws redone sequentially (exact_count[0] +=
// their number); force_exact redoes all of them.
template <typename T>
cudaError_t launch_kpp_draw(const T *w, int n, const double *bs, const double *U, int nt,
                            int force_exact, int *cand, int *unc, int *exact_count,
                            cudaStream_t s);
// Distances of every row to the t candidate rows (D[c*n + i], as
// launch_kpp_dist) and cost[c] = the serial sum in T, index order from 0, of
// max(0, min(w_i, D[c*n + i])) -- the reference's value, computed exactly
// (kmeans_kpp.cu) -- stored as double.  work: kpp_cost_work_bytes(n, t).
template <typename T>
cudaError_t launch_kpp_dist_cost(const T *X, int ldx, int n, int d, const T *xnorm,
                                 const int *cand, int t, const T *w, T *D, double *cost,
                                 void *work, cudaStream_t s, const T *xinv = nullptr,
                                 int cosine = 0);
size_t kpp_cost_work_bytes(int n, int t);
// Choose among the nt candidates by cost (chosen[c]), w_i = max(0, min(w_i,
// D_best,i)), w_best = 0, block sums of the new w.
template <typename T>
cudaError_t launch_kpp_select_update(T *w, const T *D, int n, const double *cost,
                                     const int *cand, int nt, int *chosen, int c, double *bs,
                                     cudaStream_t s);

// ------------------------------------------------- tensor-core k-means ---
// 1 when the tcgen05 assignment handles (k clusters, d features) with the
// given bf16 split (1 or 3 terms).
int tc_assign_supported(int k, int d, int split);
// X fp32 (ld) -> Xh = bf16(x), Xl = bf16(x - Xh) (Xl may be null), row-major
// with ldo = 64 * ceil(d / 64), zero padded.
cudaError_t launch_split_bf16(const float *X, int ld, int rows, int d, void *Xh, void *Xl,
                              int ldo, cudaStream_t s);
// Centre operands of the tensor-core pass: B = -2 C as bf16 hi (+ lo), the
// |c|^2 hi/lo pair (Baug, npad x 64) and, when Aaug_once != null, the constant
// ones operand (128 x 64).
cudaError_t launch_prep_centres(const float *C, int ld, int k, int d, int ldo,
                                const float *cnorm, void *Bh, void *Bl, void *Baug,
                                void *Aaug_once, cudaStream_t s);
// out[i] = |x_i| (fp32); *maxv = max_i |x_i| when maxv != null.
cudaError_t launch_row_norm_max(const float *X, int ld, int rows, int d, float *out, float *maxv,
                                cudaStream_t s);
// launch_centre_norms + launch_prep_centres in one launch (Aaug already set).
cudaError_t launch_prep_centres_norms(const float *C, int ld, int k, int d, int ldo,
                                      float *cnorm, void *Bh, void *Bl, void *Baug,
                                      cudaStream_t s);
// Tensor-core candidate assignment: rows with a single candidate within the
// error bound get their exact fp32 label; the others are appended to amb_rows
// with up to 4 candidate clusters each (amb_ncand = 0: scan all).  *amb_count
// must be 0 on entry.  Certified rows whose label changed go to `chg`.
// cmax_sq_floor: a lower bound on max_j |c_j|^2 for the error bound, for
// centres whose cnorm entries are not their norms (spherical k-means: cnorm
// zero, the score -2 x.c, unit-length centres).
cudaError_t launch_kmeans_assign_tc(int split, const void *Xh, const void *Xl, int n, int ldbf,
                                    const void *Bh, const void *Bl, const void *Baug,
                                    const void *Aaug, int k, const float *xnorm,
                                    const float *cnorm, int *labels, const int *labels_prev,
                                    int *flags, int *amb_rows, int *amb_cand, int *amb_ncand,
                                    int *amb_count, int *err, const ChangeList &chg,
                                    cudaStream_t s, float cmax_sq_floor = 0.f);
// Exact fp32 labels of the rows listed by the tensor-core pass (changed
// ones to `chg`).
cudaError_t launch_kmeans_rescore(const float *X, int ld, int d, const float *C, int k,
                                  const float *cnorm, const int *amb_rows, const int *amb_cand,
                                  const int *amb_ncand, const int *amb_count, int max_rows,
                                  int *labels, const int *labels_prev, int *flags,
                                  const ChangeList &chg, cudaStream_t s);

} // namespace b200
