// k-means (Lloyd) handle, host side.  Control flow, option semantics and
// status codes follow source/core/clustering/kmeans/kmeans.cpp; every pass
// over the data runs on the GPU (kmeans_simt.cu), the random draws of the
// initialisation use the same std:: generators as the reference on the host.
#include "alg.hpp"
#include <cstdlib>

namespace b200 {

enum { INIT_RANDOM = 0, INIT_KPP = 1, INIT_SUPPLIED = 2, INIT_RPART = 3, INIT_AFK = 4 };
enum { ALG_LLOYD = 0, ALG_ELKAN = 1, ALG_HW = 2, ALG_MACQ = 3 };
enum { EC_IGNORE = 0, EC_ERROR = 1, EC_SPLIT = 2 };
static constexpr int SEG_ROWS = 64; // rows per fp64 partial-sum chunk

template <typename T>
KMeans<T>::KMeans(ErrorRecord *e, CudaCtx *c, bool single) {
    err = e;
    cuda = c;
    opts.single = single;
    register_common_options(opts);
    // kmeans_options.hpp:46-137
    const da_int imax = std::numeric_limits<da_int>::max();
    opts.add_int("n_clusters", 1, LB::greaterequal, imax, UB::p_inf, 1);
    opts.add_int("n_init", 1, LB::greaterequal, imax, UB::p_inf, 10);
    opts.add_int("max_iter", 1, LB::greaterequal, imax, UB::p_inf, 300);
    opts.add_int("low precision max_iter", 1, LB::greaterequal, imax, UB::p_inf, 200);
    opts.add_int("seed", -1, LB::greaterequal, imax, UB::p_inf, 0);
    opts.add_int("afk-mc2 samples", 1, LB::greaterequal, imax, UB::p_inf, 50);
    opts.add_string("initialization method",
                    {{"random", INIT_RANDOM},
                     {"k-means++", INIT_KPP},
                     {"supplied", INIT_SUPPLIED},
                     {"random partitions", INIT_RPART},
                     {"afk-mc2", INIT_AFK}},
                    "k-means++");
    opts.add_string("algorithm",
                    {{"lloyd", ALG_LLOYD}, {"elkan", ALG_ELKAN}, {"hartigan-wong", ALG_HW},
                     {"macqueen", ALG_MACQ}},
                    "lloyd");
    opts.add_string("mixed precision", {{"yes", 1}, {"no", 0}}, "no");
    opts.add_string("empty clusters", {{"ignore", EC_IGNORE}, {"error", EC_ERROR}, {"split", EC_SPLIT}},
                    "ignore");
    opts.add_string("distance", {{"euclidean", 0}, {"cosine", 1}}, "euclidean");
    opts.add_string("normalize data", {{"yes", 1}, {"no", 0}}, "yes");
    opts.add_real("convergence tolerance", 0.0, LB::greaterequal, 0.0, UB::p_inf, 1.0e-4);
    // B200 option (no counterpart in the reference): "bf16" / "bf16x3" run the
    // assignment on the tensor cores (one bf16 term, or the three-term hi/lo
    // split) with a certified candidate pass whose labels equal the "plain"
    // fp32 path's; fp64 data always use "plain".
    opts.add_string("precision mode", {{"plain", 0}, {"bf16", 1}, {"bf16x3", 3}}, "bf16x3");
    opts.add_real("low precision convergence tolerance", 0.0, LB::greaterequal, 0.0, UB::p_inf,
                  1.0e-2);
}

template <typename T> KMeans<T>::~KMeans() {
    drop_loop_graph();
    if (h_small) cudaFreeHost(h_small);
}

template <typename T> void KMeans<T>::refresh() {
    best_n_iter = 0;
    best_inertia = 0;
    best_lp_n_iter = 0;
    warn_maxit = false;
}

// kmeans.cpp:249-293
template <typename T>
da_status KMeans<T>::set_data(da_int n, da_int d, const T *A, da_int lda) {
    refresh();
    const da_order ord = order();
    da_status s = check_2d(*err, ord, n, d, A, lda, "n_samples", "n_features", "A", "lda", 1, 1,
                           opts.key("check data") == 1);
    if (s != da_status_success) return s;
    A_host = A;
    lda_host = lda;
    data_order = ord;
    n_samples = n;
    n_features = d;
    initdone = true;
    model_trained = false;
    // the device copy is refreshed on the next use, in the same allocation
    // when it is large enough (no free / malloc per new data set)
    dx_loaded = false;
    // n_clusters is re-bounded by the number of samples (kmeans_options.hpp:153-170)
    da_int kc = opts.i("n_clusters");
    opts.rebound_int("n_clusters", 1, LB::greaterequal, n, UB::lessequal);
    opts.set_int("n_clusters", std::min(kc, n));
    if (cuda->init(*err) == da_status_success) {
        s = ensure_device_data();
        if (s != da_status_success) return s;
    } else {
        err->clear();
    }
    if (kc > n)
        return err->warn(da_status_incompatible_options,
                         "The requested number of clusters has been decreased from " +
                             std::to_string(kc) + " to " + std::to_string(n) +
                             " due to the size of the data array.");
    return da_status_success;
}

template <typename T> da_status KMeans<T>::ensure_device_data() {
    da_status s = cuda->init(*err);
    if (s != da_status_success) return s;
    if (dx_loaded && dX.p) return da_status_success;
    ld = pad4(n_features);
    if (!dX.ensure((size_t)n_samples * ld * sizeof(T)) || !dXn.ensure((size_t)n_samples * sizeof(T)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(upload_matrix<T>(data_order, n_samples, n_features, A_host, lda_host, dX.as<T>(), ld,
                              dStage, cuda->stream),
             "upload of A");
    B200_TRY(launch_row_sqnorms<T>(dX.as<T>(), ld, n_samples, n_features, dXn.as<T>(), cuda->stream),
             "row norms");
    dXbf_stale = true;
    fx_stale = true;
    sph_ready = 0;
    dx_loaded = true;
    return da_status_success;
}

// kmeans.cpp:295-348
template <typename T> da_status KMeans<T>::set_init_centres(const T *C, da_int ldc) {
    if (!initdone)
        return err->error(da_status_no_data,
                          "No data has been passed to the handle. Please call "
                          "da_kmeans_set_data_s or da_kmeans_set_data_d.");
    if (order() != data_order)
        return err->error(da_status_incompatible_options,
                          "The storage order option was changed after data was set.");
    const da_int k = opts.i("n_clusters");
    da_status s = check_2d(*err, data_order, k, n_features, C, ldc, "n_clusters", "n_features",
                           "C", "ldc", 1, 1, opts.key("check data") == 1);
    if (s != da_status_success) return s;
    C_supplied.assign((size_t)k * n_features, T(0));
    for (da_int j = 0; j < n_features; ++j)
        for (da_int i = 0; i < k; ++i)
            C_supplied[i + (size_t)j * k] =
                data_order == column_major ? C[i + (size_t)j * ldc] : C[(size_t)i * ldc + j];
    centres_supplied = true;
    return da_status_success;
}

template <typename T> da_status KMeans<T>::alloc_work() {
    const size_t n = n_samples, k = n_clusters;
    const size_t nblk = (n + kmeans_assign_block_rows() - 1) / kmeans_assign_block_rows();
    const size_t nchunks = n / SEG_ROWS + k + 1;
    const size_t nfin = (k * n_features + 255) / 256;
    bool ok = dC0.ensure(k * ld * sizeof(T)) && dC1.ensure(k * ld * sizeof(T)) &&
              dCn.ensure(k * sizeof(T)) && dL0.ensure(n * sizeof(int)) &&
              dL1.ensure(n * sizeof(int)) && dCounts.ensure(k * sizeof(int)) &&
              dBlockCounts.ensure(nblk * k * sizeof(int)) &&
              dOffsets.ensure((k + 1) * sizeof(int)) && dSorted.ensure(n * sizeof(int)) &&
              dChunkSums.ensure(nchunks * ld * sizeof(double)) &&
              dSegStart.ensure((k + 1) * sizeof(int)) &&
              dScalars.ensure((8 + 2 * nfin) * sizeof(double)) && dFlags.ensure(8 * sizeof(int)) &&
              dPartials.ensure(148 * 8 * 16 * sizeof(double));
    if (!ok) return err->error(da_status_memory_error, "Device memory allocation failed.");
    if (!h_small && cudaMallocHost(&h_small, 256) != cudaSuccess) {
        cudaGetLastError();
        return err->error(da_status_memory_error, "Pinned host allocation failed.");
    }
    if (cudaMemsetAsync(dC0.p, 0, k * ld * sizeof(T), cuda->stream) != cudaSuccess ||
        cudaMemsetAsync(dC1.p, 0, k * ld * sizeof(T), cuda->stream) != cudaSuccess ||
        cudaMemsetAsync(dL0.p, 0, n * sizeof(int), cuda->stream) != cudaSuccess ||
        cudaMemsetAsync(dL1.p, 0, n * sizeof(int), cuda->stream) != cudaSuccess)
        return cuda_status(*err, cudaGetLastError(), "memset");
    return da_status_success;
}

// Column-major host centres (k x d) -> device row-major centres.
template <typename T>
static cudaError_t upload_centres(const std::vector<T> &Cc, int k, int d, int ld, T *dC,
                                  cudaStream_t s) {
    std::vector<T> rm((size_t)k * ld, T(0));
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < d; ++j) rm[(size_t)i * ld + j] = Cc[i + (size_t)j * k];
    cudaError_t e = cudaMemcpyAsync(dC, rm.data(), rm.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}
template <typename T>
static cudaError_t download_centres(const T *dC, int k, int d, int ld, std::vector<T> &Cc,
                                    cudaStream_t s) {
    std::vector<T> rm((size_t)k * ld);
    cudaError_t e = cudaMemcpyAsync(rm.data(), dC, rm.size() * sizeof(T), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(s);
    Cc.assign((size_t)k * d, T(0));
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < d; ++j) Cc[i + (size_t)j * k] = rm[(size_t)i * ld + j];
    return e;
}

// Host element of the user's data array (A is kept alive by the caller, as
// the reference's pointer-storing set_data requires).
template <typename T> static inline T host_at(const KMeans<T> &km, da_int i, da_int j) {
    return km.data_order == column_major ? km.A_host[i + (size_t)j * km.lda_host]
                                         : km.A_host[(size_t)i * km.lda_host + j];
}

// kmeans.cpp:1524-1664.  The host draws from the reference's engine in the
// reference's order (the first centre, then n_trials canonical doubles per
// further centre, consumed by std::discrete_distribution one each); the
// device maps the draws to rows (kmeans_kpp.cu), computes the candidates'
// distances and their costs -- the reference's serial sums in the working
// precision, reproduced exactly -- chooses and updates the weights, with no
// host round trip per centre.
template <typename T> da_status KMeans<T>::kmeans_plusplus(T *dC) {
    cudaStream_t st = cuda->stream;
    const da_int n = n_samples, k = n_clusters, d = n_features;
    const da_int n_trials = 2 + (da_int)std::log(k);
    const int nb = kpp_num_blocks((int)n);
    if (!dW.ensure((size_t)n * sizeof(T)) || !dKD.ensure((size_t)n * n_trials * sizeof(T)) ||
        !dCand.ensure((size_t)(2 * n_trials + k + 2) * sizeof(int)) ||
        !dKppU.ensure((size_t)std::max<da_int>(1, (k - 1) * n_trials) * sizeof(double)) ||
        !dKppBs.ensure((size_t)(nb + n_trials) * sizeof(double)) ||
        !dPartials.ensure(kpp_cost_work_bytes((int)n, (int)n_trials)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    int *dCandv = dCand.as<int>();
    int *dUnc = dCandv + n_trials;
    int *dChosen = dUnc + n_trials;
    int *dFlag = dChosen + k;       // [0] a positive weight, [1] redone draws
    double *dBs = dKppBs.as<double>();
    double *dCost = dBs + nb;
    std::uniform_int_distribution<> dis_int(0, n - 1);
    const int first = dis_int(mt_gen);
    int init_words[3] = {first, 0, 0};
    // chosen[0] = first; flags cleared
    B200_TRY(cudaMemcpyAsync(dChosen, &init_words[0], sizeof(int), cudaMemcpyHostToDevice, st),
             "copy");
    B200_TRY(cudaMemcpyAsync(dFlag, &init_words[1], 2 * sizeof(int), cudaMemcpyHostToDevice, st),
             "copy");
    // w: distances to the first centre, clamped (kmeans.cpp:1561-1590)
    // spherical k-means: the cosine distance of compute_distances_to_point
    const T *xinv = (sph && sph_norm) ? dXinv.as<T>() : nullptr;
    const int cosine = sph ? 1 : 0;
    B200_TRY(launch_kpp_dist<T>(dX.as<T>(), ld, n, d, dXn.as<T>(), dChosen, 1, dW.as<T>(), st,
                                xinv, cosine),
             "k-means++ distances");
    B200_TRY(launch_kpp_clamp<T>(dW.as<T>(), (int)n, first, dBs, dFlag, st), "k-means++ weights");
    int flags[2] = {0, 0};
    B200_TRY(cudaMemcpyAsync(flags, dFlag, sizeof(flags), cudaMemcpyDeviceToHost, st), "copy");
    B200_TRY(cudaStreamSynchronize(st), "k-means++");
    std::vector<int> chosen(k, 0);
    if (!flags[0]) {
        // all rows coincide with the first centre: rows 0..k-1
        for (da_int i = 0; i < k; ++i) chosen[i] = i;
    } else if (k > 1) {
        // the draws of std::discrete_distribution, in the reference's order
        std::vector<double> U((size_t)(k - 1) * n_trials);
        for (double &u : U) u = std::generate_canonical<double, std::numeric_limits<double>::digits>(mt_gen);
        B200_TRY(cudaMemcpyAsync(dKppU.p, U.data(), U.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, st), "copy");
        const double *dU = dKppU.as<double>();
        const char *fe = std::getenv("AOCLDA_B200_KPP_EXACT_DRAWS");
        const int force_exact = (fe && fe[0] == '1') ? 1 : 0;
        for (da_int c = 1; c < k; ++c) {
            B200_TRY(launch_kpp_draw<T>(dW.as<T>(), (int)n, dBs, dU + (size_t)(c - 1) * n_trials,
                                        (int)n_trials, force_exact, dCandv, dUnc, dFlag + 1, st),
                     "k-means++ draws");
            B200_TRY(launch_kpp_dist_cost<T>(dX.as<T>(), ld, n, d, dXn.as<T>(), dCandv, n_trials,
                                             dW.as<T>(), dKD.as<T>(), dCost, dPartials.p, st,
                                             xinv, cosine),
                     "k-means++ distances and costs");
            B200_TRY(launch_kpp_select_update<T>(dW.as<T>(), dKD.as<T>(), (int)n, dCost, dCandv,
                                                 (int)n_trials, dChosen, (int)c, dBs, st),
                     "k-means++ update");
        }
        B200_TRY(cudaMemcpyAsync(chosen.data(), dChosen, k * sizeof(int), cudaMemcpyDeviceToHost, st),
                 "copy");
        B200_TRY(cudaMemcpyAsync(flags, dFlag, sizeof(flags), cudaMemcpyDeviceToHost, st), "copy");
        B200_TRY(cudaStreamSynchronize(st), "k-means++");
        cuda->stats["kmeans_pp_exact_draws"] += (double)flags[1];
    }
    std::vector<T> Cc((size_t)k * d);
    for (da_int c = 0; c < k; ++c)
        for (da_int j = 0; j < d; ++j) Cc[c + (size_t)j * k] = host_at(*this, chosen[c], j);
    B200_TRY(upload_centres<T>(Cc, k, d, ld, dC, st), "centres");
    return da_status_success;
}

// kmeans.cpp:1667-1808 (AFK-MC^2), evaluated on the host from the caller's data.
template <typename T> da_status KMeans<T>::afk_mcmc(std::vector<T> &Cc) {
    const da_int n = n_samples, k = n_clusters, d = n_features;
    std::vector<T> xn(n, T(0));
    for (da_int i = 0; i < n; ++i)
        for (da_int j = 0; j < d; ++j) xn[i] += host_at(*this, i, j) * host_at(*this, i, j);
    // spherical k-means on normalised data: inverse row norms (kmeans.cpp:681-703)
    std::vector<T> inv;
    if (sph && sph_norm) {
        inv.resize(n);
        for (da_int i = 0; i < n; ++i) {
            const T nr = std::sqrt(xn[i]);
            inv[i] = nr > T(0) ? T(1) / nr : T(0);
        }
    }
    std::uniform_int_distribution<> dis_int(0, n - 1);
    const da_int c1 = dis_int(mt_gen);
    Cc.assign((size_t)k * d, T(0));
    // a chosen row as a centre: scaled by its inverse norm for normalised
    // spherical data (kmeans.cpp:1692-1697, 1803-1807)
    auto place = [&](da_int c, da_int row) {
        const T r = inv.empty() ? T(1) : inv[row];
        for (da_int j = 0; j < d; ++j) Cc[c + (size_t)j * k] = host_at(*this, row, j) * r;
    };
    place(0, c1);
    // d(x, c1)^2 in GEMM form, or the cosine distance (kmeans.cpp:1489-1510)
    std::vector<T> w3(n), q(n);
    T dot_c = T(0);
    for (da_int j = 0; j < d; ++j) dot_c += host_at(*this, c1, j) * host_at(*this, c1, j);
    T sum = T(0);
    for (da_int i = 0; i < n; ++i) {
        T s = T(0);
        for (da_int j = 0; j < d; ++j) s += host_at(*this, i, j) * host_at(*this, c1, j);
        T v;
        if (sph) {
            const T cs = inv.empty() ? s : s * inv[i] * inv[c1];
            v = std::max(T(0), T(1) - cs);
        } else {
            v = T(-2) * s + (xn[i] + dot_c);
        }
        w3[i] = std::max(T(0), v);
        sum += w3[i];
    }
    const T inv2n = T(1) / T(2 * n);
    for (da_int i = 0; i < n; ++i)
        q[i] = (std::isfinite(sum) && sum > T(0)) ? T(0.5) * w3[i] / sum + inv2n : T(1) / T(n);
    auto nearest = [&](da_int idx, da_int nc) {
        T best = std::numeric_limits<T>::infinity();
        for (da_int c = 0; c < nc; ++c) {
            T dist = T(0);
            if (sph) {
                for (da_int j = 0; j < d; ++j) dist += host_at(*this, idx, j) * Cc[c + (size_t)j * k];
                dist = std::max(T(0), T(1) - (inv.empty() ? dist : dist * inv[idx]));
            } else {
                for (da_int j = 0; j < d; ++j) {
                    T t = host_at(*this, idx, j) - Cc[c + (size_t)j * k];
                    dist += t * t;
                }
            }
            if (dist < best) best = dist;
        }
        return best;
    };
    std::discrete_distribution<> q_dist(q.begin(), q.end());
    std::uniform_real_distribution<T> unif(T(0), T(1));
    for (da_int i = 1; i < k; ++i) {
        da_int x = q_dist(mt_gen);
        T dx = nearest(x, i);
        for (da_int step = 0; step < afk_samples; ++step) {
            da_int y = q_dist(mt_gen);
            T dy = nearest(y, i);
            T dxqy = dx * q[y];
            if (dxqy == T(0) || (dy * q[x]) / dxqy > unif(mt_gen)) {
                x = y;
                dx = dy;
            }
        }
        place(i, x);
    }
    return da_status_success;
}

// kmeans.cpp:1400-1486: the method's centres, scaled to unit length for
// spherical k-means (kmeans.cpp:1478-1485).
template <typename T> da_status KMeans<T>::init_centres(T *dC) {
    da_status s = init_centres_raw(dC);
    if (s != da_status_success || !sph) return s;
    B200_TRY(launch_sph_centres<T>(nullptr, dC, (int)n_clusters, (int)n_features, ld,
                                   dPartials.as<double>(), nullptr, cuda->stream),
             "centre normalisation");
    B200_TRY(cudaStreamSynchronize(cuda->stream), "centre normalisation");
    return da_status_success;
}

// Inverse row norms and, for normalised data, the normalised rows of the
// data set (kmeans.cpp:681-703), once per data set.
template <typename T> da_status KMeans<T>::prepare_sph() {
    if (!sph) return da_status_success;
    const int want = sph_norm ? 3 : 1;
    if ((sph_ready & want) == want) return da_status_success;
    if (!dXinv.ensure((size_t)n_samples * sizeof(T)) ||
        (sph_norm && !dXs.ensure((size_t)n_samples * ld * sizeof(T))))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(launch_sph_data<T>(dX.as<T>(), ld, (int)n_samples, (int)n_features, dXn.as<T>(),
                                dXinv.as<T>(), sph_norm ? dXs.as<T>() : nullptr, cuda->stream),
             "row normalisation");
    B200_TRY(cudaStreamSynchronize(cuda->stream), "row normalisation");
    sph_ready |= want;
    return da_status_success;
}

template <typename T> da_status KMeans<T>::init_centres_raw(T *dC) {
    const da_int n = n_samples, k = n_clusters, d = n_features;
    std::vector<T> Cc;
    switch (init_method) {
    case INIT_RANDOM: {
        // selection sampling (da_std.hpp:102-118)
        std::vector<da_int> pick;
        da_int need = std::min(k, n), pop = n;
        for (da_int i = 0; need > 0; ++i, --pop) {
            std::uniform_int_distribution<da_int> dd(0, pop - 1);
            if (dd(mt_gen) < need) {
                pick.push_back(i);
                --need;
            }
        }
        Cc.assign((size_t)k * d, T(0));
        for (da_int c = 0; c < k; ++c)
            for (da_int j = 0; j < d; ++j) Cc[c + (size_t)j * k] = host_at(*this, pick[c], j);
        break;
    }
    case INIT_RPART: {
        std::uniform_int_distribution<> dis(0, k - 1);
        std::vector<int> lab(n);
        for (da_int i = 0; i < n; ++i) lab[i] = dis(mt_gen);
        // means of the random partition, computed with the device update kernels
        B200_TRY(cudaMemcpyAsync(dL0.p, lab.data(), n * sizeof(int), cudaMemcpyHostToDevice,
                                 cuda->stream), "copy");
        B200_TRY(launch_kmeans_sort(dL0.as<int>(), n, k, dBlockCounts.as<int>(), dCounts.as<int>(),
                                    dOffsets.as<int>(), dSegStart.as<int>(), SEG_ROWS,
                                    dSorted.as<int>(), dFlags.as<int>(), cuda->stream), "sort");
        T *other = (dC == dC0.as<T>()) ? dC1.as<T>() : dC0.as<T>();
        B200_TRY(launch_kmeans_update<T>(dX.as<T>(), ld, n, d, k, dSorted.as<int>(),
                                         dOffsets.as<int>(), dSegStart.as<int>(), SEG_ROWS,
                                         dChunkSums.as<double>(), dCounts.as<int>(), other, dC, ld,
                                         dScalars.as<double>(), dFlags.as<int>(), cuda->stream),
                 "update");
        B200_TRY(cudaStreamSynchronize(cuda->stream), "init");
        return da_status_success;
    }
    case INIT_KPP: return kmeans_plusplus(dC);
    case INIT_AFK: {
        da_status s = afk_mcmc(Cc);
        if (s != da_status_success) return s;
        break;
    }
    default: Cc = C_supplied; break;
    }
    B200_TRY(upload_centres<T>(Cc, k, d, ld, dC, cuda->stream), "centres");
    return da_status_success;
}

// Fixed-point centroid update (fp32 data): per-feature scales 2^s_f with
// n * max_i |x_if| * 2^s_f < 2^62 (computed once per data set), partial-sum
// buffers for one CTA per SM.  Data holding inf or NaN keep the sorted fp64
// update.
template <typename T> da_status KMeans<T>::prepare_fx() {
    use_fx = false;
    if constexpr (std::is_same_v<T, float>) {
        const int n = n_samples, k = n_clusters, d = n_features;
        if (!fx_update_supported(k, d)) return da_status_success;
        cudaStream_t st = cuda->stream;
        const float *src = update_rows();
        if (fx_src != static_cast<const void *>(src)) fx_stale = true;
        const size_t accb = fx_accum_bytes(k, d);
        if (!dFxScale.ensure((size_t)2 * d * sizeof(double) + (size_t)d * 4 + 16) ||
            !dFxAcc.ensure(accb))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        // both accumulator sets start at zero (each update clears the other)
        B200_TRY(cudaMemsetAsync(dFxAcc.p, 0, accb, st), "memset");
        fx_parity = 0;
        if (!dFxTicket.p) {
            if (!dFxTicket.ensure(16))
                return err->error(da_status_memory_error, "Device memory allocation failed.");
            B200_TRY(cudaMemsetAsync(dFxTicket.p, 0, 16, st), "memset");
        }
        if (fx_stale) {
            double *scale = dFxScale.as<double>();
            unsigned *colmax = reinterpret_cast<unsigned *>(scale + 2 * d);
            int *nonfinite = reinterpret_cast<int *>(colmax + d);
            B200_TRY(launch_col_absmax(src, ld, n, d, colmax, nonfinite, st), "column maxima");
            std::vector<unsigned> hmax(d + 1);
            B200_TRY(cudaMemcpyAsync(hmax.data(), colmax, (d + 1) * sizeof(unsigned),
                                     cudaMemcpyDeviceToHost, st), "copy");
            B200_TRY(cudaStreamSynchronize(st), "column maxima");
            fx_data_ok = hmax[d] == 0;
            if (fx_data_ok) {
                // scale[f] = 2^s_f as fp32 (bytes 0..4d), inv_scale[f] = 2^-s_f as
                // fp64 (from byte 8d); s_f keeps n max|x| 2^s_f < 2^62 and
                // max|x| 2^s_f < 2^44 (the quantiser's range), and 2^s_f within
                // the fp32 range
                int L = 0;
                while ((1LL << L) < (long long)n) ++L;
                std::vector<float> scf(d);
                std::vector<double> inv(d);
                for (int f = 0; f < d; ++f) {
                    float m;
                    std::memcpy(&m, &hmax[f], sizeof(float));
                    int E = 0;
                    if (m > 0.f) std::frexp((double)m, &E); // m < 2^E
                    int sf = std::min(62 - L, 44) - E;
                    sf = std::max(-126, std::min(127, sf));
                    scf[f] = std::ldexp(1.0f, sf);
                    inv[f] = std::ldexp(1.0, -sf);
                }
                B200_TRY(cudaMemcpyAsync(scale, scf.data(), d * sizeof(float),
                                         cudaMemcpyHostToDevice, st), "copy");
                B200_TRY(cudaMemcpyAsync(scale + d, inv.data(), d * sizeof(double),
                                         cudaMemcpyHostToDevice, st), "copy");
                B200_TRY(cudaStreamSynchronize(st), "scales");
            }
            fx_stale = false;
            fx_src = src;
        }
        use_fx = fx_data_ok;
    }
    return da_status_success;
}

// Device state of the tensor-core assignment (fp32 data only): bf16 copy of
// X, row norms |x_i|, bf16 centres, scalars and the relabel list.
template <typename T> da_status KMeans<T>::prepare_tc() {
    use_tc = false;
    if constexpr (std::is_same_v<T, float>) {
        const int split = (int)opts.key("precision mode");
        if (split == 0 || !tc_assign_supported(n_clusters, n_features, split))
            return da_status_success;
        const int nkb = (n_features + 63) / 64;
        const int npad = (n_clusters + 15) & ~15;
        const bool fresh = tc_split != split || ldbf != nkb * 64 || dXbf_stale;
        ldbf = nkb * 64;
        const size_t xb = (size_t)n_samples * ldbf * 2;
        if (!dXh.ensure(xb) || (split == 3 && !dXl.ensure(xb)) ||
            !dXnrm.ensure((size_t)n_samples * 4) || !dBh.ensure((size_t)npad * ldbf * 2) ||
            !dBl.ensure((size_t)npad * ldbf * 2) || !dBaug.ensure((size_t)npad * 64 * 2) ||
            !dAaug.ensure(128 * 64 * 2) || !dCtmp.ensure((size_t)npad * 4) ||
            !dTcScal.ensure(64) || !dAmb.ensure((size_t)n_samples * 4 * 6))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        cudaStream_t st = cuda->stream;
        if (fresh) {
            B200_TRY(launch_split_bf16(dX.as<float>(), ld, n_samples, n_features, dXh.p,
                                       split == 3 ? dXl.p : nullptr, ldbf, st), "bf16 copy");
            B200_TRY(launch_row_norm_max(dX.as<float>(), ld, n_samples, n_features,
                                         dXnrm.as<float>(), nullptr, st), "row norms");
            tc_split = split;
            dXbf_stale = false;
            aaug_ready = false;
        }
        B200_TRY(cudaMemsetAsync(dTcScal.p, 0, 64, st), "memset");
        use_tc = true;
    }
    return da_status_success;
}

// Spherical k-means assigns with zero centre norms (the score -2 x.c of
// unit-length centres): the tensor-core error bound takes max |c|^2 from
// this bound instead -- a centre normalised in fp64 and rounded to fp32 has
// |c|^2 <= (1 + 2^-24)^2 -- with margin.
static constexpr float SPH_CMAX_SQ = 1.001f;

// Assignment of every row to its nearest centre (labels of the plain fp32
// formula), on the tensor cores when use_tc, else on the CUDA cores.
template <typename T> da_status KMeans<T>::assign(const T *dC, int *dL, const int *dLprev) {
    cudaStream_t st = cuda->stream;
    const int n = n_samples, k = n_clusters, d = n_features;
    if constexpr (std::is_same_v<T, float>) {
        if (use_tc) {
            int *amb_cnt = reinterpret_cast<int *>(dTcScal.as<char>() + 16);
            int *errf = reinterpret_cast<int *>(dTcScal.as<char>() + 20);
            int *amb_rows = dAmb.as<int>();
            int *amb_ncand = amb_rows + n;
            int *amb_cand = amb_rows + 2 * (size_t)n;
            const bool s3 = tc_split == 3;
            if (chg_capture && aaug_ready) {
                // the graph loop's body: norms and operands in one launch; the
                // counters were re-armed by the previous iteration's finalize
                B200_TRY(launch_prep_centres_norms(dC, ld, k, d, ldbf, dCn.as<float>(), dBh.p,
                                                   s3 ? dBl.p : nullptr, dBaug.p, st),
                         "centre operands");
            } else {
                B200_TRY(launch_prep_centres(dC, ld, k, d, ldbf, dCn.as<float>(), dBh.p,
                                             s3 ? dBl.p : nullptr, dBaug.p,
                                             aaug_ready ? nullptr : dAaug.p, st), "centre operands");
                aaug_ready = true;
                B200_TRY(cudaMemsetAsync(amb_cnt, 0, 3 * sizeof(int), st), "memset");
            }
            ChangeList chg;
            if (chg_capture) {
                chg.count = dChg.as<int>();
                chg.rows = chg.count + 1;
                chg.olds = chg.rows + chg_cap;
                chg.news = chg.olds + chg_cap;
                chg.cap = chg_cap;
            }
            B200_TRY(cuda->timed("kmeans_assign", [&] {
                return launch_kmeans_assign_tc(tc_split, dXh.p, s3 ? dXl.p : nullptr, n, ldbf,
                                               dBh.p, s3 ? dBl.p : nullptr, dBaug.p, dAaug.p, k,
                                               dXnrm.as<float>(), dCn.as<float>(), dL, dLprev,
                                               dFlags.as<int>(), amb_rows, amb_cand, amb_ncand,
                                               amb_cnt, errf, chg, st, sph ? SPH_CMAX_SQ : 0.f);
            }), "tensor-core assign");
            // the graph loop re-scores the listed rows in its update launch
            // (fx_rescore_delta_kernel)
            if (chg_capture) return da_status_success;
            B200_TRY(cuda->timed("kmeans_rescore", [&] {
                return launch_kmeans_rescore(dX.as<float>(), ld, d, dC, k, dCn.as<float>(),
                                             amb_rows, amb_cand, amb_ncand, amb_cnt, n, dL,
                                             dLprev, dFlags.as<int>(), chg, st);
            }), "relabel");
            return da_status_success;
        }
    }
    B200_TRY(cuda->timed("kmeans_assign", [&] {
        return launch_kmeans_assign<T>(dX.as<T>(), ld, n, d, dC, ld, k, dCn.as<T>(), dL, dLprev,
                                       nullptr, dFlags.as<int>(), st);
    }), "assign");
    return da_status_success;
}

// One Lloyd pass (kmeans_lloyd.hpp:106-271): assignment against dCprev and,
// if `update`, the new centres in dCnew plus the shift norms.
template <typename T>
da_status KMeans<T>::lloyd_step(const T *dCprev, T *dCnew, int *dL, const int *dLprev, bool update,
                                double *h_scal, int *h_flags) {
    cudaStream_t st = cuda->stream;
    const int n = n_samples, k = n_clusters, d = n_features;
    if (sph) // -C X^T of kmeans_lloyd.hpp:144-146: the norms term is zero
        B200_TRY(cudaMemsetAsync(dCn.p, 0, k * sizeof(T), st), "memset");
    else
        B200_TRY(launch_centre_norms<T>(dCprev, ld, k, d, dCn.as<T>(), st), "centre norms");
    B200_TRY(cudaMemsetAsync(dFlags.p, 0, 8 * sizeof(int), st), "memset");
    {
        da_status sa = assign(dCprev, dL, dLprev);
        if (sa != da_status_success) return sa;
    }
    if (update && use_fx) {
        if constexpr (std::is_same_v<T, float>) {
            const double *scale = dFxScale.as<double>();
            B200_TRY(cuda->timed("kmeans_update", [&] {
                return launch_kmeans_update_fx(
                    update_rows(), ld, n, d, k, dL, reinterpret_cast<const float *>(scale),
                    scale + d, dFxAcc.p, fx_parity,
                    dCprev, dCnew, dCounts.as<int>(), dScalars.as<double>() + 8,
                    dScalars.as<double>(), dFlags.as<int>(), dFxTicket.as<unsigned>(), st);
            }), "update");
            fx_parity ^= 1;
        }
    } else if (update) {
        B200_TRY(cuda->timed("kmeans_sort", [&] {
            return launch_kmeans_sort(dL, n, k, dBlockCounts.as<int>(), dCounts.as<int>(),
                                      dOffsets.as<int>(), dSegStart.as<int>(), SEG_ROWS,
                                      dSorted.as<int>(), dFlags.as<int>(), st);
        }), "sort");
        B200_TRY(cuda->timed("kmeans_update", [&] {
            return launch_kmeans_update<T>(update_rows(), ld, n, d, k, dSorted.as<int>(),
                                           dOffsets.as<int>(), dSegStart.as<int>(), SEG_ROWS,
                                           dChunkSums.as<double>(), dCounts.as<int>(), dCprev,
                                           dCnew, ld, dScalars.as<double>(), dFlags.as<int>(), st);
        }), "update");
    }
    if (update && sph) // unit-length centres and their shift (kmeans_lloyd.hpp:373-405)
        B200_TRY(launch_sph_centres<T>(dCprev, dCnew, k, d, ld, dPartials.as<double>(),
                                       dScalars.as<double>(), st),
                 "centre normalisation");
    if (h_scal) {
        B200_TRY(cudaMemcpyAsync(h_scal, dScalars.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st),
                 "copy");
    }
    if (h_flags) {
        B200_TRY(cudaMemcpyAsync(h_flags, dFlags.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st),
                 "copy");
    }
    int tc_state[3] = {0, 0, 0};
    if (use_tc)
        B200_TRY(cudaMemcpyAsync(tc_state, dTcScal.as<char>() + 16, 3 * sizeof(int),
                                 cudaMemcpyDeviceToHost, st), "copy");
    B200_TRY(cudaStreamSynchronize(st), "Lloyd iteration");
    (void)d;
    if (use_tc) {
        amb_last = tc_state[0];
        cuda->stats["relabelled_rows"] = (double)amb_last;
        cuda->stats["full_scan_rows"] = (double)tc_state[2];
        if (tc_state[1] != 0)
            return err->error(da_status_internal_error,
                              "The tensor-core assignment kernel timed out waiting on a "
                              "pipeline barrier (code " + std::to_string(tc_state[1]) + ").");
    }
    return da_status_success;
}

// Empty-cluster splitting (kmeans.cpp:1127-1330), on the host.
template <typename T> da_status KMeans<T>::split_empty(T *dC, int *dL, bool &split) {
    split = false;
    const da_int n = n_samples, k = n_clusters, d = n_features;
    std::vector<int> lab(n);
    std::vector<T> Cc;
    B200_TRY(cudaMemcpyAsync(lab.data(), dL, n * sizeof(int), cudaMemcpyDeviceToHost, cuda->stream),
             "copy");
    B200_TRY(download_centres<T>(dC, k, d, ld, Cc, cuda->stream), "copy");
    std::vector<da_int> cnt(k, 0);
    for (da_int i = 0; i < n; ++i) cnt[lab[i]]++;
    da_int n_empty = 0;
    for (da_int c = 0; c < k; ++c) n_empty += cnt[c] == 0;
    if (n_empty == 0) return da_status_success;
    std::vector<T> w(n);
    // spherical k-means: 1 - cos with the rows' inverse norms (kmeans.cpp:1171-1192)
    std::vector<T> inv;
    if (sph && sph_norm) {
        inv.resize(n);
        B200_TRY(cudaMemcpyAsync(inv.data(), dXinv.p, n * sizeof(T), cudaMemcpyDeviceToHost,
                                 cuda->stream), "copy");
        B200_TRY(cudaStreamSynchronize(cuda->stream), "copy");
    }
    auto dist_to = [&](da_int i, da_int c) {
        T s = T(0);
        if (sph) {
            for (da_int j = 0; j < d; ++j) s += host_at(*this, i, j) * Cc[c + (size_t)j * k];
            return T(1) - (inv.empty() ? s : s * inv[i]);
        }
        for (da_int j = 0; j < d; ++j) {
            T t = host_at(*this, i, j) - Cc[c + (size_t)j * k];
            s += t * t;
        }
        return s;
    };
    // spherical: a centre row scaled to unit length in T (kmeans.cpp:1243-1269)
    auto unit = [&](da_int c) {
        T sq = T(0);
        for (da_int j = 0; j < d; ++j) sq += Cc[c + (size_t)j * k] * Cc[c + (size_t)j * k];
        if (!(sq > T(0))) return;
        const T r = T(1) / std::sqrt(sq);
        for (da_int j = 0; j < d; ++j) Cc[c + (size_t)j * k] *= r;
    };
    for (da_int i = 0; i < n; ++i) w[i] = dist_to(i, lab[i]);
    for (da_int c = 0; c < k; ++c) {
        if (cnt[c] != 0) continue;
        da_int bi = -1;
        T bd = T(-1);
        for (da_int i = 0; i < n; ++i)
            if (cnt[lab[i]] > 1 && std::isfinite(w[i]) && w[i] > bd) {
                bd = w[i];
                bi = i;
            }
        if (bi < 0) break;
        const da_int old = lab[bi], nold = cnt[old];
        const T ib = inv.empty() ? T(1) : inv[bi]; // the donor row as the update sums it
        for (da_int j = 0; j < d; ++j) {
            T &cv = Cc[old + (size_t)j * k];
            cv = (cv * T(nold) - host_at(*this, bi, j) * ib) / T(nold - 1);
        }
        for (da_int j = 0; j < d; ++j) Cc[c + (size_t)j * k] = host_at(*this, bi, j) * ib;
        if (sph) {
            unit(old);
            unit(c);
        }
        cnt[old] -= 1;
        cnt[c] = 1;
        lab[bi] = (int)c;
        w[bi] = T(0);
        if (n_empty > 1)
            for (da_int i = 0; i < n; ++i)
                if (lab[i] == old) w[i] = dist_to(i, old);
    }
    B200_TRY(upload_centres<T>(Cc, k, d, ld, dC, cuda->stream), "copy");
    B200_TRY(cudaMemcpyAsync(dL, lab.data(), n * sizeof(int), cudaMemcpyHostToDevice, cuda->stream),
             "copy");
    B200_TRY(cudaStreamSynchronize(cuda->stream), "split");
    split = true;
    return da_status_success;
}

// ------------------------------------------- Lloyd loop as a CUDA graph ----
// Iterations 1.. of run_lloyd (fp32 on the tensor cores, fixed-point update,
// empty clusters ignored, no kernel timing) as one graph launch: a WHILE conditional node
// whose body is one Lloyd iteration working in place on the centres dC and
// the labels dL (every kernel reads a row's or element's old value before
// the same thread writes the new one), with the convergence test on the
// device (fx_finalize_kernel), so the host waits once per fit instead of
// once per iteration.  The decisions are the host loop's: the same fp64
// scalars, the same comparisons.
template <typename T> void KMeans<T>::drop_loop_graph() {
    if (loop_exec) cudaGraphExecDestroy(loop_exec);
    if (loop_graph) cudaGraphDestroy(loop_graph);
    loop_exec = nullptr;
    loop_graph = nullptr;
    loop_key.clear();
}

template <typename T> bool KMeans<T>::build_loop_graph(T *dC, int *dL) {
    if constexpr (!std::is_same_v<T, float>) {
        (void)dC, (void)dL;
        return false;
    } else {
        cudaStream_t st = cuda->stream;
        const int n = n_samples, k = n_clusters, d = n_features;
        cudaGraph_t g = nullptr;
        if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
        cudaGraphConditionalHandle cond = 0;
        cudaGraphNodeParams p = {};
        cudaGraphNode_t node;
        bool ok = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault) ==
                  cudaSuccess;
        if (ok) {
            p.type = cudaGraphNodeTypeConditional;
            p.conditional.handle = cond;
            p.conditional.type = cudaGraphCondTypeWhile;
            p.conditional.size = 1;
            ok = cudaGraphAddNode(&node, g, nullptr, 0, &p) == cudaSuccess;
        }
        cudaGraph_t body = ok ? p.conditional.phGraph_out[0] : nullptr;
        if (ok)
            ok = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            // the assignment lists its changed rows for the incremental update;
            // the centre norms come with the operands (aaug_ready: iteration 0
            // set the constant operand), the counters are re-armed by the
            // finalize of the previous iteration (and before the graph starts)
            chg_capture = true;
            bool launched = aaug_ready && assign(dC, dL, dL) == da_status_success;
            chg_capture = false;
            ChangeList chg;
            chg.count = dChg.as<int>();
            chg.rows = chg.count + 1;
            chg.olds = chg.rows + chg_cap;
            chg.news = chg.olds + chg_cap;
            chg.cap = chg_cap;
            const double *scale = dFxScale.as<double>();
            AmbList amb;
            amb.rows = dAmb.as<int>();
            amb.ncand = amb.rows + n;
            amb.cand = amb.rows + 2 * (size_t)n;
            amb.count = reinterpret_cast<const int *>(dTcScal.as<char>() + 16);
            launched = launched &&
                       launch_kmeans_update_fx_loop(
                           dX.as<float>(), ld, n, d, k, dL, reinterpret_cast<const float *>(scale),
                           scale + d, dFxAcc.p, dC, dCounts.as<int>(), dScalars.as<double>() + 8,
                           dScalars.as<double>(), dFlags.as<int>(), dFxTicket.as<unsigned>(),
                           dLoop.as<LloydLoopState>(), (unsigned long long)cond, chg,
                           reinterpret_cast<int *>(dTcScal.as<char>() + 16), dCn.as<float>(), amb,
                           chg.news + chg_cap, st) == cudaSuccess;
            cudaGraph_t captured = nullptr;
            const bool ended = cudaStreamEndCapture(st, &captured) == cudaSuccess;
            ok = launched && ended;
        }
        if (ok) ok = cudaGraphInstantiate(&loop_exec, g, 0) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            err->clear();
            loop_exec = nullptr;
            cudaGraphDestroy(g);
            return false;
        }
        loop_graph = g;
        return true;
    }
}

template <typename T>
da_status KMeans<T>::lloyd_graph(T *dC, int *dL, da_int &n_iter_out, int &converged, bool &ran) {
    ran = false;
    if constexpr (!std::is_same_v<T, float>) {
        (void)dC, (void)dL, (void)n_iter_out, (void)converged;
        return da_status_success;
    } else {
        cudaStream_t st = cuda->stream;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            cudaGetLastError();
            return da_status_success; // the caller captures: run the host loop
        }
        if (!dLoop.ensure(sizeof(LloydLoopState))) return da_status_success;
        // changed-row list: up to n / 16 rows (more: the update recounts)
        chg_cap = (int)std::min<da_int>(n_samples, std::max<da_int>(8192, n_samples / 16));
        // [count][rows][olds][news][recount word]
        if (!dChg.ensure((size_t)(3 * (size_t)chg_cap + 2) * sizeof(int))) return da_status_success;
        const std::vector<uintptr_t> key = {
            (uintptr_t)st, (uintptr_t)dC, (uintptr_t)dL, (uintptr_t)dX.p, (uintptr_t)dCn.p,
            (uintptr_t)dFlags.p, (uintptr_t)dFxAcc.p, (uintptr_t)dFxScale.p,
            (uintptr_t)dScalars.p, (uintptr_t)dCounts.p, (uintptr_t)dFxTicket.p,
            (uintptr_t)dLoop.p, (uintptr_t)dXh.p, (uintptr_t)dXl.p, (uintptr_t)dXnrm.p,
            (uintptr_t)dBh.p, (uintptr_t)dBl.p, (uintptr_t)dBaug.p, (uintptr_t)dAaug.p,
            (uintptr_t)dCtmp.p, (uintptr_t)dTcScal.p, (uintptr_t)dAmb.p, (uintptr_t)n_samples,
            (uintptr_t)n_clusters, (uintptr_t)n_features, (uintptr_t)ld, (uintptr_t)use_tc,
            (uintptr_t)tc_split, (uintptr_t)ldbf, (uintptr_t)dChg.p, (uintptr_t)chg_cap};
        if (!loop_exec || key != loop_key) {
            drop_loop_graph();
            if (!build_loop_graph(dC, dL)) return da_status_success;
            loop_key = key;
        }
        char *hb = static_cast<char *>(h_small);
        LloydLoopState *hs = reinterpret_cast<LloydLoopState *>(hb + 128);
        LloydLoopState *ho = reinterpret_cast<LloydLoopState *>(hb + 160);
        int *tc_state = reinterpret_cast<int *>(hb + 192);
        *hs = LloydLoopState{1, (int)max_iter, 0, 0, (double)tol};
        tc_state[0] = tc_state[1] = tc_state[2] = 0;
        B200_TRY(cudaMemcpyAsync(dLoop.p, hs, sizeof(LloydLoopState), cudaMemcpyHostToDevice, st),
                 "copy");
        // the graph keeps the sums and counts of the current labels in
        // accumulator set 0; iteration 0 left them in set 1 - fx_parity
        if (fx_parity == 0) {
            const size_t kd = (size_t)n_clusters * n_features;
            char *acc = dFxAcc.as<char>();
            B200_TRY(cudaMemcpyAsync(acc, acc + kd * 8, kd * 8, cudaMemcpyDeviceToDevice, st), "copy");
            B200_TRY(cudaMemcpyAsync(acc + 2 * kd * 8, acc + 2 * kd * 8 + (size_t)n_clusters * 4,
                                     (size_t)n_clusters * 4, cudaMemcpyDeviceToDevice, st), "copy");
        }
        // the first graph iteration's counters (later ones: re-armed by the finalize)
        B200_TRY(cudaMemsetAsync(dChg.p, 0, sizeof(int), st), "memset");
        B200_TRY(cudaMemsetAsync(dFlags.p, 0, 8 * sizeof(int), st), "memset");
        if (use_tc) {
            int *amb_cnt = reinterpret_cast<int *>(dTcScal.as<char>() + 16);
            B200_TRY(cudaMemsetAsync(amb_cnt, 0, sizeof(int), st), "memset");
            B200_TRY(cudaMemsetAsync(amb_cnt + 2, 0, sizeof(int), st), "memset");
        }
        B200_TRY(cudaGraphLaunch(loop_exec, st), "Lloyd loop graph");
        B200_TRY(cudaMemcpyAsync(ho, dLoop.p, sizeof(LloydLoopState), cudaMemcpyDeviceToHost, st),
                 "copy");
        if (use_tc)
            B200_TRY(cudaMemcpyAsync(tc_state, dTcScal.as<char>() + 16, 3 * sizeof(int),
                                     cudaMemcpyDeviceToHost, st), "copy");
        // both accumulator sets zero again for the host-loop steps that follow
        B200_TRY(cudaMemsetAsync(dFxAcc.p, 0, fx_accum_bytes(n_clusters, n_features), st),
                 "memset");
        B200_TRY(cudaStreamSynchronize(st), "Lloyd loop graph");
        fx_parity = 0;
        if (use_tc) {
            amb_last = tc_state[0];
            cuda->stats["relabelled_rows"] = (double)amb_last;
            cuda->stats["full_scan_rows"] = (double)tc_state[2];
            if (tc_state[1] != 0)
                return err->error(da_status_internal_error,
                                  "The tensor-core assignment kernel timed out waiting on a "
                                  "pipeline barrier (code " + std::to_string(tc_state[1]) + ").");
        }
        n_iter_out = ho->n_iter;
        converged = ho->conv;
        ran = true;
        return da_status_success;
    }
}

// perform_kmeans (kmeans.cpp:996-1058)
template <typename T>
da_status KMeans<T>::run_lloyd(T *&dCcur, T *&dCprev, int *&dLcur, int *&dLprev, da_int &n_iter,
                               int &converged, double &inertia, bool &empty_found) {
    double *h_scal = static_cast<double *>(h_small);
    int *h_flags = reinterpret_cast<int *>(static_cast<char *>(h_small) + 64);
    converged = 0;
    empty_found = false;
    // iterations 1.. as one graph launch where the loop allows it
    const bool graph = use_fx && use_tc && empty_mode == EC_IGNORE && !cuda->timing && !sph;
    da_int it = 0;
    for (it = 0; it < max_iter; ++it) {
        if (graph && it == 1) {
            bool ran = false;
            da_int nit = 0;
            int conv = 0;
            da_status s = lloyd_graph(dCcur, dLcur, nit, conv, ran);
            if (s != da_status_success) return s;
            cuda->stats["graph_loop"] = ran ? 1.0 : 0.0;
            if (ran) {
                converged = conv;
                it = nit;
                break;
            }
        }
        std::swap(dCprev, dCcur);
        std::swap(dLprev, dLcur);
        da_status s = lloyd_step(dCprev, dCcur, dLcur, dLprev, true, h_scal, h_flags);
        if (s != da_status_success) return s;
        if (empty_mode != EC_IGNORE && h_flags[1] > 0) {
            if (empty_mode == EC_ERROR) {
                empty_found = true;
                return da_status_success;
            }
            bool split = false;
            s = split_empty(dCcur, dLcur, split);
            if (s != da_status_success) return s;
            if (split) continue;
        }
        // convergence_test (kmeans.cpp:1359-1397)
        int conv = 0;
        if (it > 1 && h_flags[0] == 0) conv = 2;
        if (conv == 0 && std::sqrt(h_scal[1]) < tol * std::sqrt(h_scal[0])) conv = 1;
        converged = conv;
        if (converged > 0) break;
    }
    n_iter = it;
    if (converged == 1 || it == max_iter) {
        // relabel against the final centres without updating them
        std::swap(dLprev, dLcur);
        da_status s = lloyd_step(dCcur, nullptr, dLcur, nullptr, false, nullptr, nullptr);
        if (s != da_status_success) return s;
    }
    if (sph)
        B200_TRY(launch_sph_inertia<T>(dX.as<T>(), ld, n_samples, n_features, dCcur, dLcur,
                                       sph_norm ? dXinv.as<T>() : nullptr, dPartials.as<double>(),
                                       dScalars.as<double>() + 2, cuda->stream), "inertia");
    else
        B200_TRY(launch_kmeans_inertia<T>(dX.as<T>(), ld, n_samples, n_features, dCcur, ld, dLcur,
                                          dPartials.as<double>(), dScalars.as<double>() + 2,
                                          cuda->stream), "inertia");
    B200_TRY(cudaMemcpyAsync(h_scal + 2, dScalars.as<double>() + 2, sizeof(double),
                             cudaMemcpyDeviceToHost, cuda->stream), "copy");
    B200_TRY(cudaStreamSynchronize(cuda->stream), "inertia");
    inertia = h_scal[2];
    return da_status_success;
}

// Option reading and consistency checks of kmeans.cpp:359-458.
template <typename T> da_status KMeans<T>::read_options() {
    n_clusters = opts.i("n_clusters");
    init_method = opts.key("initialization method");
    n_init = opts.i("n_init");
    max_iter = opts.i("max_iter");
    tol = opts.r("convergence tolerance");
    seed = opts.i("seed");
    afk_samples = opts.i("afk-mc2 samples");
    algorithm = opts.key("algorithm");
    empty_mode = opts.key("empty clusters");
    const bool spherical = opts.key("distance") == 1;
    sph = spherical;
    sph_norm = opts.key("normalize data") == 1;
    da_status warn_status = da_status_success;
    std::string warn_msg;
    if (n_init > 1 && init_method == INIT_SUPPLIED) {
        warn_msg = "n_init was set to " + std::to_string(n_init) +
                   " but the initialization method was set to 'supplied'. The k-means "
                   "algorithm will only be run once.";
        n_init = 1;
        warn_status = da_status_incompatible_options;
    }
    if (algorithm == ALG_HW && (n_clusters == 1 || n_clusters >= n_samples))
        return err->error(da_status_incompatible_options,
                          "The Hartigan-Wong algorithm requires 1 < k < n_samples.");
    if (spherical && algorithm == ALG_HW)
        return err->error(da_status_incompatible_options,
                          "Cosine distance is not compatible with the Hartigan-Wong algorithm. "
                          "Please use Lloyd, Elkan, or MacQueen.");
    if (algorithm == ALG_HW || algorithm == ALG_MACQ)
        return err->error(da_status_not_implemented,
                          "The B200 library implements Lloyd's algorithm (and Elkan, whose "
                          "iterates are Lloyd's); Hartigan-Wong and MacQueen are not provided.");
    if (n_clusters > n_samples)
        return err->error(da_status_incompatible_options,
                          "n_clusters = " + std::to_string(n_clusters) + ", and n_samples = " +
                              std::to_string(n_samples) + ". Constraint: n_clusters <= n_samples.");
    if (init_method == INIT_SUPPLIED && !centres_supplied)
        return err->error(da_status_no_data,
                          "The initialization method was set to 'supplied' but no initial "
                          "centres have been provided.");
    if (n_clusters > 12288)
        return err->error(da_status_not_implemented,
                          "More than 12288 clusters are not supported by the B200 library.");
    if (warn_status != da_status_success) return err->warn(warn_status, warn_msg);
    return da_status_success;
}

// kmeans.cpp:351-783
template <typename T> da_status KMeans<T>::compute() {
    if (!initdone)
        return err->error(da_status_no_data,
                          "No data has been passed to the handle. Please call "
                          "da_kmeans_set_data_s or da_kmeans_set_data_d.");
    if (order() != data_order)
        return err->error(da_status_incompatible_options,
                          "The storage order option was changed after data was set.");
    da_status warn_status = da_status_success;
    std::string warn_msg;
    {
        da_status s0 = read_options();
        if (s0 != da_status_success && err->severity == DA_ERROR) return s0;
        if (s0 != da_status_success) {
            warn_status = s0;
            warn_msg = err->message;
            err->clear();
        }
    }
    da_status s = ensure_device_data();
    if (s != da_status_success) return s;
    s = alloc_work();
    if (s != da_status_success) return s;
    s = prepare_sph();
    if (s != da_status_success) return s;
    s = prepare_tc();
    if (s != da_status_success) return s;
    s = prepare_fx();
    if (s != da_status_success) return s;
    cuda->stats["tensor_core"] = use_tc ? 1.0 : 0.0;
    cuda->stats["fixed_point_update"] = use_fx ? 1.0 : 0.0;
    if (init_method != INIT_SUPPLIED) {
        if (seed == -1) {
            std::random_device r;
            seed = std::abs((da_int)r());
        }
        mt_gen.seed(seed);
    }
    best_inertia = std::numeric_limits<double>::infinity();
    bool valid = false, first_valid = true;
    for (da_int run = 0; run < n_init; ++run) {
        T *dCcur = dC0.as<T>(), *dCprev = dC1.as<T>();
        int *dLcur = dL0.as<int>(), *dLprev = dL1.as<int>();
        s = init_centres(dCcur);
        if (s != da_status_success) return s;
        da_int n_iter = 0;
        int converged = 0;
        double inertia = 0;
        bool empty = false;
        s = run_lloyd(dCcur, dCprev, dLcur, dLprev, n_iter, converged, inertia, empty);
        if (s != da_status_success) return s;
        if (empty) continue;
        valid = true;
        if (inertia < best_inertia || first_valid) {
            first_valid = false;
            best_inertia = inertia;
            best_n_iter = n_iter;
            warn_maxit = converged == 0;
            B200_TRY(download_centres<T>(dCcur, n_clusters, n_features, ld, best_centres,
                                         cuda->stream), "copy");
            // labels stay on the device until they are queried
            if (!dBestL.ensure((size_t)n_samples * sizeof(int)))
                return err->error(da_status_memory_error, "Device memory allocation failed.");
            B200_TRY(cudaMemcpyAsync(dBestL.p, dLcur, n_samples * sizeof(int),
                                     cudaMemcpyDeviceToDevice, cuda->stream), "copy");
            B200_TRY(cudaStreamSynchronize(cuda->stream), "copy");
            best_labels_on_host = false;
        }
    }
    if (!valid)
        return err->error(da_status_empty_clusters,
                          "All " + std::to_string(n_init) +
                              " run(s) of the k-means algorithm resulted in at least one empty "
                              "cluster during the k-means iterations. A better set of initial "
                              "cluster centers is needed.");
    model_trained = true;
    model_sph = sph;
    model_sph_norm = sph_norm;
    if (warn_maxit) return err->warn(da_status_maxit, "The maximum number of iterations was reached.");
    // kmeans.cpp:413-420 only records this warning; compute() still succeeds
    if (warn_status != da_status_success) err->warn(warn_status, warn_msg);
    return da_status_success;
}

// Initial centres of the configured initialisation method (B200 extension).
template <typename T> da_status KMeans<T>::initial_centres(T *C, da_int ldc) {
    if (!initdone)
        return err->error(da_status_no_data,
                          "No data has been passed to the handle. Please call "
                          "da_kmeans_set_data_s or da_kmeans_set_data_d.");
    da_status s = read_options();
    if (s != da_status_success && err->severity == DA_ERROR) return s;
    err->clear();
    if (C == nullptr) return err->error(da_status_invalid_pointer, "The array C is null.");
    const da_order ord = order();
    if ((ord == column_major && ldc < n_clusters) || (ord == row_major && ldc < n_features))
        return err->error(da_status_invalid_leading_dimension, "ldc is too small.");
    s = ensure_device_data();
    if (s != da_status_success) return s;
    s = alloc_work();
    if (s != da_status_success) return s;
    s = prepare_sph();
    if (s != da_status_success) return s;
    if (init_method != INIT_SUPPLIED) {
        if (seed == -1) {
            std::random_device r;
            seed = std::abs((da_int)r());
        }
        mt_gen.seed(seed);
    }
    s = init_centres(dC0.as<T>());
    if (s != da_status_success) return s;
    std::vector<T> Cc;
    B200_TRY(download_centres<T>(dC0.as<T>(), n_clusters, n_features, ld, Cc, cuda->stream), "copy");
    for (da_int i = 0; i < n_clusters; ++i)
        for (da_int j = 0; j < n_features; ++j)
            C[ord == row_major ? (size_t)i * ldc + j : i + (size_t)j * ldc] =
                Cc[i + (size_t)j * n_clusters];
    return da_status_success;
}

// kmeans.cpp:894-993
template <typename T>
da_status KMeans<T>::predict(da_int m, da_int d, const T *Y, da_int ldy, da_int *labels) {
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "The k-means has not been computed. Please call da_kmeans_compute_s or "
                         "da_kmeans_compute_d.");
    if (d != n_features)
        return err->error(da_status_invalid_input,
                          "The function was called with k_features = " + std::to_string(d) +
                              " but the k-means has been computed with " +
                              std::to_string(n_features) + " features.");
    da_status s = check_2d(*err, order(), m, d, Y, ldy, "k_samples", "k_features", "Y", "ldy", 1,
                           1, opts.key("check data") == 1);
    if (s != da_status_success) return s;
    if (labels == nullptr) return err->error(da_status_invalid_pointer, "The array Y_labels is null.");
    s = cuda->init(*err);
    if (s != da_status_success) return s;
    cudaStream_t st = cuda->stream;
    if (!dY.ensure((size_t)m * ld * sizeof(T)) || !dYL.ensure((size_t)m * sizeof(int)) ||
        !dC0.ensure((size_t)n_clusters * ld * sizeof(T)) || !dCn.ensure(n_clusters * sizeof(T)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(upload_matrix<T>(order(), m, d, Y, ldy, dY.as<T>(), ld, dStage, st), "upload");
    B200_TRY(upload_centres<T>(best_centres, n_clusters, n_features, ld, dC0.as<T>(), st), "upload");
    if (model_sph) // -C Y^T (kmeans.cpp:976-981)
        B200_TRY(cudaMemsetAsync(dCn.p, 0, n_clusters * sizeof(T), st), "memset");
    else
        B200_TRY(launch_centre_norms<T>(dC0.as<T>(), ld, n_clusters, n_features, dCn.as<T>(), st),
                 "norms");
    B200_TRY(launch_kmeans_assign<T>(dY.as<T>(), ld, m, n_features, dC0.as<T>(), ld, n_clusters,
                                     dCn.as<T>(), dYL.as<int>(), nullptr, nullptr, nullptr, st),
             "assign");
    std::vector<int> lab(m);
    B200_TRY(cudaMemcpyAsync(lab.data(), dYL.p, m * sizeof(int), cudaMemcpyDeviceToHost, st), "copy");
    B200_TRY(cudaStreamSynchronize(st), "predict");
    for (da_int i = 0; i < m; ++i) labels[i] = lab[i];
    return da_status_success;
}

// kmeans.cpp:786-891: X_transform_ij = |x_i - c_j| (GEMM form, no clamp).
template <typename T>
da_status KMeans<T>::transform(da_int m, da_int d, const T *X, da_int ldx, T *Xt, da_int ldxt) {
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "The k-means has not been computed. Please call da_kmeans_compute_s or "
                         "da_kmeans_compute_d.");
    if (d != n_features)
        return err->error(da_status_invalid_input,
                          "The function was called with m_features = " + std::to_string(d) +
                              " but the k-means has been computed with " +
                              std::to_string(n_features) + " features.");
    da_status s = check_2d(*err, order(), m, d, X, ldx, "m_samples", "m_features", "X", "ldx", 1, 1,
                           opts.key("check data") == 1);
    if (s != da_status_success) return s;
    s = check_2d(*err, order(), m, n_clusters, Xt, ldxt, "m_samples", "n_clusters", "X_transform",
                 "ldx_transform", 1, 1, false);
    if (s != da_status_success) return s;
    s = cuda->init(*err);
    if (s != da_status_success) return s;
    cudaStream_t st = cuda->stream;
    const size_t outn = (size_t)m * n_clusters;
    if (!dY.ensure((size_t)m * ld * sizeof(T)) || !dYL.ensure((size_t)m * sizeof(T)) ||
        !dC0.ensure((size_t)n_clusters * ld * sizeof(T)) || !dCn.ensure(n_clusters * sizeof(T)) ||
        !dKD.ensure(outn * sizeof(T)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(upload_matrix<T>(order(), m, d, X, ldx, dY.as<T>(), ld, dStage, st), "upload");
    B200_TRY(upload_centres<T>(best_centres, n_clusters, n_features, ld, dC0.as<T>(), st), "upload");
    B200_TRY(launch_centre_norms<T>(dC0.as<T>(), ld, n_clusters, n_features, dCn.as<T>(), st), "norms");
    B200_TRY(launch_row_sqnorms<T>(dY.as<T>(), ld, m, n_features, dYL.as<T>(), st), "norms");
    if (model_sph) {
        // 1 - clamp(x.c / |x|) (kmeans.cpp:821-858): -dot, then the post-op
        PairwiseArgs a{ACC_DOT, POST_NEG, 256, 2.0, false, order() == row_major};
        B200_TRY(launch_pairwise<T>(dY.as<T>(), ld, m, dC0.as<T>(), ld, n_clusters, n_features,
                                    dYL.as<T>(), dCn.as<T>(), a, dKD.as<T>(), st), "transform");
        B200_TRY(launch_sph_transform<T>(dKD.as<T>(), m, n_clusters, order() == row_major,
                                         model_sph_norm ? dYL.as<T>() : nullptr, st),
                 "transform");
    } else {
        PairwiseArgs a{ACC_DOT, POST_GEMM_SQRT, 256, 2.0, false, order() == row_major};
        B200_TRY(launch_pairwise<T>(dY.as<T>(), ld, m, dC0.as<T>(), ld, n_clusters, n_features,
                                    dYL.as<T>(), dCn.as<T>(), a, dKD.as<T>(), st), "transform");
    }
    std::vector<T> out(outn);
    B200_TRY(cudaMemcpyAsync(out.data(), dKD.p, outn * sizeof(T), cudaMemcpyDeviceToHost, st), "copy");
    B200_TRY(cudaStreamSynchronize(st), "transform");
    const bool rm = order() == row_major;
    for (da_int i = 0; i < m; ++i)
        for (da_int j = 0; j < n_clusters; ++j)
            Xt[rm ? (size_t)i * ldxt + j : i + (size_t)j * ldxt] =
                out[rm ? (size_t)i * n_clusters + j : i + (size_t)j * m];
    return da_status_success;
}

// kmeans.cpp:146-224
template <typename T> da_status KMeans<T>::get_result_t(da_result q, da_int *dim, T *out) {
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "k-means clustering has not yet been computed. Please call "
                         "da_kmeans_compute_s or da_kmeans_compute_d before extracting results.");
    switch (q) {
    case da_rinfo:
        if (*dim < 6) {
            *dim = 6;
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: 6.");
        }
        out[0] = (T)n_samples;
        out[1] = (T)n_features;
        out[2] = (T)n_clusters;
        out[3] = (T)best_n_iter;
        out[4] = (T)best_inertia;
        out[5] = (T)best_lp_n_iter;
        return da_status_success;
    case da_kmeans_cluster_centres: {
        const da_int need = n_clusters * n_features;
        if (*dim < need) {
            *dim = need;
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: " +
                                 std::to_string(need) + ".");
        }
        const bool rm = order() == row_major;
        for (da_int i = 0; i < n_clusters; ++i)
            for (da_int j = 0; j < n_features; ++j)
                out[rm ? (size_t)i * n_features + j : i + (size_t)j * n_clusters] =
                    best_centres[i + (size_t)j * n_clusters];
        return da_status_success;
    }
    default:
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    }
}
template <typename T> da_status KMeans<T>::get_result(da_result q, da_int *dim, double *out) {
    if constexpr (std::is_same_v<T, double>) return get_result_t(q, dim, (T *)out);
    return err->error(da_status_wrong_type, "Wrong precision type.");
}
template <typename T> da_status KMeans<T>::get_result(da_result q, da_int *dim, float *out) {
    if constexpr (std::is_same_v<T, float>) return get_result_t(q, dim, (T *)out);
    return err->error(da_status_wrong_type, "Wrong precision type.");
}
template <typename T> da_status KMeans<T>::get_result_int(da_result q, da_int *dim, da_int *out) {
    if (q == da_trained) return AlgBase::get_result_int(q, dim, out);
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "k-means clustering has not yet been computed. Please call "
                         "da_kmeans_compute_s or da_kmeans_compute_d before extracting results.");
    if (q == da_kmeans_labels) {
        if (*dim < n_samples) {
            *dim = n_samples;
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: " +
                                 std::to_string(n_samples) + ".");
        }
        if (!best_labels_on_host) {
            std::vector<int> lab(n_samples);
            B200_TRY(cudaMemcpyAsync(lab.data(), dBestL.p, n_samples * sizeof(int),
                                     cudaMemcpyDeviceToHost, cuda->stream), "copy");
            B200_TRY(cudaStreamSynchronize(cuda->stream), "copy");
            best_labels.assign(lab.begin(), lab.end());
            best_labels_on_host = true;
        }
        for (da_int i = 0; i < n_samples; ++i) out[i] = best_labels[i];
        return da_status_success;
    }
    return err->warn(da_status_unknown_query, "The requested result could not be found.");
}

// ------------------------------------------------- sharded Lloyd steps ----
// A data set split over processes, one shard per handle (one GPU each).  The
// caller runs the Lloyd loop of run_lloyd: per iteration shard_partial
// (assignment + the shard's fixed-point centroid sums, counts and
// label-change flag, packed into one int64 device buffer), ONE integer
// all-reduce of that buffer over the processes (exact in any order), then
// shard_finalize (the new centres from the global sums, identical on every
// process, and the shift / norm scalars of the convergence test).  With the
// global column maxima and row count every shard quantises with the scales
// the whole data set would use on one device, so the reduced sums, the
// centres and the convergence decisions equal the single-handle ones bit for
// bit.
template <typename T> da_status KMeans<T>::shard_colmax(float *colmax) {
    if constexpr (!std::is_same_v<T, float>) {
        (void)colmax;
        return err->error(da_status_not_implemented, "Sharded k-means steps are fp32 only.");
    } else {
        if (!initdone)
            return err->error(da_status_no_data, "No data has been passed to the handle.");
        if (!colmax) return err->error(da_status_invalid_pointer, "colmax is null.");
        da_status s = ensure_device_data();
        if (s != da_status_success) return s;
        const int d = n_features;
        if (!dFxScale.ensure((size_t)2 * d * sizeof(double) + (size_t)d * 4 + 16))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        unsigned *cm = reinterpret_cast<unsigned *>(dFxScale.as<double>() + 2 * d);
        int *nonfinite = reinterpret_cast<int *>(cm + d);
        cudaStream_t st = cuda->stream;
        B200_TRY(launch_col_absmax(dX.as<float>(), ld, n_samples, d, cm, nonfinite, st), "maxima");
        std::vector<unsigned> h(d + 1);
        B200_TRY(cudaMemcpyAsync(h.data(), cm, (d + 1) * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                 st), "copy");
        B200_TRY(cudaStreamSynchronize(st), "maxima");
        if (h[d])
            return err->error(da_status_invalid_input, "The data hold inf or NaN values.");
        std::memcpy(colmax, h.data(), d * sizeof(float));
        fx_stale = true; // the scale buffer now holds other values
        return da_status_success;
    }
}

template <typename T>
da_status KMeans<T>::shard_begin(const float *colmax_global, da_int n_global, const float *C) {
    if constexpr (!std::is_same_v<T, float>) {
        (void)colmax_global, (void)n_global, (void)C;
        return err->error(da_status_not_implemented, "Sharded k-means steps are fp32 only.");
    } else {
        shard_ready = false;
        if (!initdone)
            return err->error(da_status_no_data, "No data has been passed to the handle.");
        if (!colmax_global || !C)
            return err->error(da_status_invalid_pointer, "A required array is null.");
        if (n_global < n_samples)
            return err->error(da_status_invalid_input, "n_global is below the shard's rows.");
        da_status s = read_options();
        if (s != da_status_success && err->severity == DA_ERROR) return s;
        err->clear();
        if (sph)
            return err->error(da_status_not_implemented,
                              "Sharded k-means steps use the euclidean distance only.");
        const int k = n_clusters, d = n_features;
        if (!fx_update_supported(k, d))
            return err->error(da_status_not_implemented,
                              "n_clusters * n_features is too large for the sharded update.");
        for (int f = 0; f < d; ++f)
            if (!(colmax_global[f] >= 0.f) || std::isinf(colmax_global[f]))
                return err->error(da_status_invalid_input,
                                  "The column maxima must be finite and non-negative.");
        s = ensure_device_data();
        if (s != da_status_success) return s;
        s = alloc_work();
        if (s != da_status_success) return s;
        s = prepare_tc();
        if (s != da_status_success) return s;
        if (!dFxScale.ensure((size_t)2 * d * sizeof(double) + (size_t)d * 4 + 16) ||
            !dFxAcc.ensure((size_t)k * 4) || !dFxTicket.ensure(16))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        cudaStream_t st = cuda->stream;
        // the scales of prepare_fx, from the whole data set's maxima and rows
        int L = 0;
        while ((1LL << L) < (long long)n_global) ++L;
        std::vector<float> scf(d);
        std::vector<double> inv(d);
        for (int f = 0; f < d; ++f) {
            int E = 0;
            if (colmax_global[f] > 0.f) std::frexp((double)colmax_global[f], &E);
            int sf = std::min(62 - L, 44) - E;
            sf = std::max(-126, std::min(127, sf));
            scf[f] = std::ldexp(1.0f, sf);
            inv[f] = std::ldexp(1.0, -sf);
        }
        double *scale = dFxScale.as<double>();
        B200_TRY(cudaMemcpyAsync(scale, scf.data(), d * sizeof(float), cudaMemcpyHostToDevice, st),
                 "copy");
        B200_TRY(cudaMemcpyAsync(scale + d, inv.data(), d * sizeof(double),
                                 cudaMemcpyHostToDevice, st), "copy");
        B200_TRY(cudaMemsetAsync(dFxTicket.p, 0, 16, st), "memset");
        std::vector<float> Cp((size_t)k * ld, 0.f);
        for (int j = 0; j < k; ++j)
            std::memcpy(&Cp[(size_t)j * ld], C + (size_t)j * d, d * sizeof(float));
        B200_TRY(cudaMemcpyAsync(dC0.p, Cp.data(), Cp.size() * sizeof(float),
                                 cudaMemcpyHostToDevice, st), "copy");
        B200_TRY(cudaStreamSynchronize(st), "sharded start");
        fx_stale = true; // the scales are the whole data set's, not this shard's
        cuda->stats["tensor_core"] = use_tc ? 1.0 : 0.0;
        cuda->stats["fixed_point_update"] = 1.0;
        shard_c = 0;
        shard_l = 0;
        shard_ready = true;
        return da_status_success;
    }
}

// Assignment of the shard's rows to the current centres (labels into the
// other label buffer, flag = any label changed) and the packed sums.
template <typename T> da_status KMeans<T>::shard_partial(long long *acc) {
    if constexpr (!std::is_same_v<T, float>) {
        (void)acc;
        return err->error(da_status_not_implemented, "Sharded k-means steps are fp32 only.");
    } else {
        if (!shard_ready)
            return err->error(da_status_no_data, "da_b200_kmeans_shard_begin_s has not run.");
        if (!acc) return err->error(da_status_invalid_pointer, "acc is null.");
        const int k = n_clusters, d = n_features;
        cudaStream_t st = cuda->stream;
        float *Ccur = (shard_c ? dC1 : dC0).template as<float>();
        shard_l ^= 1;
        int *Lcur = (shard_l ? dL1 : dL0).template as<int>();
        int *Lprev = (shard_l ? dL0 : dL1).template as<int>();
        B200_TRY(launch_centre_norms<float>(Ccur, ld, k, d, dCn.as<float>(), st), "centre norms");
        B200_TRY(cudaMemsetAsync(dFlags.p, 0, 8 * sizeof(int), st), "memset");
        da_status s = assign(Ccur, Lcur, Lprev);
        if (s != da_status_success) return s;
        B200_TRY(cuda->timed("kmeans_update", [&] {
            return launch_kmeans_sums_fx(dX.as<float>(), ld, n_samples, d, k, Lcur,
                                         reinterpret_cast<const float *>(dFxScale.as<double>()),
                                         acc, dFxAcc.as<int>(), dFlags.as<int>(), st);
        }), "sums");
        return da_status_success;
    }
}

template <typename T> da_status KMeans<T>::shard_tc_check() {
    if (!use_tc) return da_status_success;
    int tc_state[3] = {0, 0, 0};
    B200_TRY(cudaMemcpyAsync(tc_state, dTcScal.as<char>() + 16, 3 * sizeof(int),
                             cudaMemcpyDeviceToHost, cuda->stream), "copy");
    B200_TRY(cudaStreamSynchronize(cuda->stream), "copy");
    cuda->stats["relabelled_rows"] = (double)tc_state[0];
    cuda->stats["full_scan_rows"] = (double)tc_state[2];
    if (tc_state[1] != 0)
        return err->error(da_status_internal_error,
                          "The tensor-core assignment kernel timed out waiting on a pipeline "
                          "barrier (code " + std::to_string(tc_state[1]) + ").");
    return da_status_success;
}

template <typename T>
da_status KMeans<T>::shard_finalize(const long long *acc, double *scalars, da_int *flags) {
    if constexpr (!std::is_same_v<T, float>) {
        (void)acc, (void)scalars, (void)flags;
        return err->error(da_status_not_implemented, "Sharded k-means steps are fp32 only.");
    } else {
        if (!shard_ready)
            return err->error(da_status_no_data, "da_b200_kmeans_shard_begin_s has not run.");
        if (!acc || !scalars || !flags)
            return err->error(da_status_invalid_pointer, "A required array is null.");
        const int k = n_clusters, d = n_features;
        cudaStream_t st = cuda->stream;
        float *Ccur = (shard_c ? dC1 : dC0).template as<float>();
        float *Cnew = (shard_c ? dC0 : dC1).template as<float>();
        const double *scale = dFxScale.as<double>();
        B200_TRY(cudaMemsetAsync(dFlags.as<int>() + 1, 0, sizeof(int), st), "memset");
        B200_TRY(launch_kmeans_finalize_shards(k, d, ld, acc, scale + d, Ccur, Cnew,
                                               dScalars.as<double>() + 8, dScalars.as<double>(),
                                               dFlags.as<int>(), dFxTicket.as<unsigned>(), st),
                 "centres");
        double *h_scal = static_cast<double *>(h_small);
        long long *h_chg = reinterpret_cast<long long *>(static_cast<char *>(h_small) + 64);
        int *h_empty = reinterpret_cast<int *>(static_cast<char *>(h_small) + 72);
        B200_TRY(cudaMemcpyAsync(h_scal, dScalars.p, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                 st), "copy");
        B200_TRY(cudaMemcpyAsync(h_chg, acc + (size_t)k * d + k, sizeof(long long),
                                 cudaMemcpyDeviceToHost, st), "copy");
        B200_TRY(cudaMemcpyAsync(h_empty, dFlags.as<int>() + 1, sizeof(int),
                                 cudaMemcpyDeviceToHost, st), "copy");
        B200_TRY(cudaStreamSynchronize(st), "Lloyd iteration");
        shard_c ^= 1;
        scalars[0] = h_scal[0];
        scalars[1] = h_scal[1];
        flags[0] = *h_chg != 0;
        flags[1] = *h_empty;
        return shard_tc_check();
    }
}

template <typename T> da_status KMeans<T>::shard_relabel(double *inertia, bool assign_first) {
    if constexpr (!std::is_same_v<T, float>) {
        (void)inertia, (void)assign_first;
        return err->error(da_status_not_implemented, "Sharded k-means steps are fp32 only.");
    } else {
        if (!shard_ready)
            return err->error(da_status_no_data, "da_b200_kmeans_shard_begin_s has not run.");
        if (!inertia) return err->error(da_status_invalid_pointer, "inertia is null.");
        const int k = n_clusters, d = n_features;
        cudaStream_t st = cuda->stream;
        float *Ccur = (shard_c ? dC1 : dC0).template as<float>();
        if (assign_first) {
            shard_l ^= 1;
            B200_TRY(launch_centre_norms<float>(Ccur, ld, k, d, dCn.as<float>(), st),
                     "centre norms");
            B200_TRY(cudaMemsetAsync(dFlags.p, 0, 8 * sizeof(int), st), "memset");
            da_status s = assign(Ccur, (shard_l ? dL1 : dL0).template as<int>(), nullptr);
            if (s != da_status_success) return s;
        }
        int *Lcur = (shard_l ? dL1 : dL0).template as<int>();
        B200_TRY(launch_kmeans_inertia<float>(dX.as<float>(), ld, n_samples, d, Ccur, ld, Lcur,
                                              dPartials.as<double>(), dScalars.as<double>() + 2,
                                              st), "inertia");
        double *h = static_cast<double *>(h_small) + 2;
        B200_TRY(cudaMemcpyAsync(h, dScalars.as<double>() + 2, sizeof(double),
                                 cudaMemcpyDeviceToHost, st), "copy");
        B200_TRY(cudaStreamSynchronize(st), "inertia");
        *inertia = *h;
        return assign_first ? shard_tc_check() : da_status_success;
    }
}

template <typename T> da_status KMeans<T>::shard_result(float *centres, da_int *labels) {
    if constexpr (!std::is_same_v<T, float>) {
        (void)centres, (void)labels;
        return err->error(da_status_not_implemented, "Sharded k-means steps are fp32 only.");
    } else {
        if (!shard_ready)
            return err->error(da_status_no_data, "da_b200_kmeans_shard_begin_s has not run.");
        const int k = n_clusters, d = n_features;
        cudaStream_t st = cuda->stream;
        std::vector<float> Cp;
        std::vector<int> h;
        if (centres) {
            Cp.resize((size_t)k * ld);
            B200_TRY(cudaMemcpyAsync(Cp.data(), (shard_c ? dC1 : dC0).p, Cp.size() * sizeof(float),
                                     cudaMemcpyDeviceToHost, st), "copy");
        }
        if (labels) {
            h.resize(n_samples);
            B200_TRY(cudaMemcpyAsync(h.data(), (shard_l ? dL1 : dL0).p, h.size() * sizeof(int),
                                     cudaMemcpyDeviceToHost, st), "copy");
        }
        B200_TRY(cudaStreamSynchronize(st), "copy");
        if (centres)
            for (int j = 0; j < k; ++j)
                std::memcpy(centres + (size_t)j * d, &Cp[(size_t)j * ld], d * sizeof(float));
        if (labels)
            for (da_int i = 0; i < n_samples; ++i) labels[i] = (da_int)h[i];
        return da_status_success;
    }
}

// Model persistence: sizes, the run information, the centres (column-major
// k x d) and the labels of the best run.  A loaded handle predicts and
// transforms and answers the result queries; a new fit needs data again.
template <typename T> da_status KMeans<T>::save_state(ByteWriter &w) {
    if (!model_trained)
        return err->error(da_status_no_data,
                          "k-means clustering has not yet been computed. Please call "
                          "da_kmeans_compute_s or da_kmeans_compute_d before saving the model.");
    std::vector<da_int> lab((size_t)n_samples);
    da_int dim = n_samples;
    da_status s = get_result_int(da_kmeans_labels, &dim, lab.data());
    if (s != da_status_success) return s;
    w.put<int64_t>(n_samples);
    w.put<int64_t>(n_features);
    w.put<int64_t>(n_clusters);
    w.put<int32_t>((int32_t)data_order);
    w.put<int64_t>(best_n_iter);
    w.put<int64_t>(best_lp_n_iter);
    w.put<double>(best_inertia);
    w.put<int32_t>(warn_maxit ? 1 : 0);
    w.put_vec(best_centres.data(), best_centres.size());
    w.put_vec(lab.data(), lab.size());
    return da_status_success;
}

template <typename T> da_status KMeans<T>::load_state(ByteReader &r) {
    const int64_t n = r.get<int64_t>(), d = r.get<int64_t>(), k = r.get<int64_t>();
    const int32_t ord = r.get<int32_t>();
    const int64_t nit = r.get<int64_t>(), lpit = r.get<int64_t>();
    const double inertia = r.get<double>();
    const int32_t wm = r.get<int32_t>();
    std::vector<T> cen = r.get_vec<T>();
    std::vector<da_int> lab = r.get_vec<da_int>();
    if (!r.ok || n < 1 || d < 1 || k < 1 || k > n || cen.size() != (size_t)(k * d) ||
        lab.size() != (size_t)n)
        return err->error(da_status_invalid_file_data, "The model file is corrupted.");
    for (da_int v : lab)
        if (v < 0 || v >= k)
            return err->error(da_status_invalid_file_data, "The model file is corrupted.");
    n_samples = (da_int)n;
    n_features = (da_int)d;
    n_clusters = (da_int)k;
    data_order = (da_order)ord;
    best_n_iter = (da_int)nit;
    best_lp_n_iter = (da_int)lpit;
    best_inertia = inertia;
    warn_maxit = wm != 0;
    best_centres = std::move(cen);
    best_labels = std::move(lab);
    best_labels_on_host = true;
    ld = pad4(n_features);
    initdone = false;
    model_trained = true;
    // the options were restored before the state: the model's distance
    model_sph = opts.key("distance") == 1;
    model_sph_norm = opts.key("normalize data") == 1;
    return da_status_success;
}

template struct KMeans<float>;
template struct KMeans<double>;

} // namespace b200
