// IVF-flat approximate-neighbours handle (host side).  Options, argument
// checks, status codes and results follow
// source/core/approximate_neighbors/approximate_neighbors.cpp; the coarse
// k-means, the coarse probe, the assignment of added rows and the list scan
// run on the GPU.
#include "alg.hpp"
#include <limits>

namespace b200 {

// "metric" ids (approximate_neighbors_types.hpp:31) and "algorithm" ids (:30)
enum { AM_EUC = 0, AM_SQEUC = 1, AM_IP = 2, AM_COS = 3 };
enum { AA_IVFFLAT = 0, AA_AUTO = 1 };

template <typename T> IVF<T>::IVF(ErrorRecord *e, CudaCtx *c, bool single) {
    err = e;
    cuda = c;
    opts.single = single;
    register_common_options(opts);
    // approximate_neighbors_options.hpp:45-101
    const da_int imax = std::numeric_limits<da_int>::max();
    opts.add_int("number of neighbors", 1, LB::greaterequal, imax, UB::p_inf, 5);
    opts.add_int("n_list", 1, LB::greaterequal, imax, UB::p_inf, 1);
    opts.add_int("n_probe", 1, LB::greaterequal, imax, UB::p_inf, 1);
    opts.add_int("k-means_iter", 1, LB::greaterequal, imax, UB::p_inf, 10);
    opts.add_int("seed", -1, LB::greaterequal, imax, UB::p_inf, 0);
    opts.add_real("train fraction", 0.0, LB::greaterthan, 1.0, UB::lessequal, 1.0);
    opts.add_string("algorithm", {{"auto", AA_AUTO}, {"ivfflat", AA_IVFFLAT}}, "ivfflat");
    opts.add_string("metric",
                    {{"euclidean", AM_EUC}, {"sqeuclidean", AM_SQEUC},
                     {"inner product", AM_IP}, {"cosine", AM_COS}},
                    "sqeuclidean");
}

// approximate_neighbors.cpp:152-185: n_list, algorithm and metric are fixed
// by train().
template <typename T> da_status IVF<T>::check_options_update() {
    if (opts.i("n_list") != n_list)
        return err->error(da_status_option_locked, "n_list cannot be changed after calling train().");
    if (opts.key("algorithm") != algo)
        return err->error(da_status_option_locked,
                          "algorithm cannot be changed after calling train().");
    if (opts.key("metric") != metric)
        return err->error(da_status_option_locked, "metric cannot be changed after calling train().");
    n_probe = opts.i("n_probe");
    return da_status_success;
}

// approximate_neighbors.cpp:187-231
template <typename T>
da_status IVF<T>::set_training_data(da_int n, da_int d, const T *X, da_int ldx) {
    train_data_set = false;
    model_trained = false;
    data_added = false;
    n_index = 0;
    data_order = order();
    da_status s = check_2d(*err, data_order, n, d, X, ldx, "n_samples", "n_features", "X_train",
                           "ldx_train");
    if (s != da_status_success) return s;
    X_train = X;
    ldx_train = ldx;
    n_samples = n;
    n_features = d;
    train_data_set = true;
    return da_status_success;
}

// Rows scaled to unit length in place (normalize_rows of da_utils.cpp:
// 807-905): the sum of squares accumulated feature by feature in T, factor
// 1 / sqrt (1 for a zero row).  X: rows x d with leading dimension ld in the
// given storage order.
template <typename T>
static void normalise_rows(bool cm, da_int rows, da_int d, T *X, da_int ld) {
    for (da_int i = 0; i < rows; ++i) {
        T s = T(0);
        for (da_int j = 0; j < d; ++j) {
            const T v = X[cm ? i + (size_t)j * ld : (size_t)i * ld + j];
            s += v * v;
        }
        const T nrm = std::sqrt(s);
        const T r = nrm == T(0) ? T(1) : T(1) / nrm;
        for (da_int j = 0; j < d; ++j) X[cm ? i + (size_t)j * ld : (size_t)i * ld + j] *= r;
    }
}

// A normalised copy of rows x d (leading dimension ldx) in the same storage
// order with leading dimension rows (column-major) or d (row-major).
template <typename T>
static std::vector<T> normalised_copy(bool cm, da_int rows, da_int d, const T *X, da_int ldx,
                                      da_int &ld_out) {
    ld_out = cm ? rows : d;
    std::vector<T> out((size_t)rows * d);
    for (da_int i = 0; i < rows; ++i)
        for (da_int j = 0; j < d; ++j)
            out[cm ? i + (size_t)j * ld_out : (size_t)i * ld_out + j] =
                X[cm ? i + (size_t)j * ldx : (size_t)i * ldx + j];
    normalise_rows(cm, rows, d, out.data(), ld_out);
    return out;
}

// The coarse quantiser's kNN handle: the centroids as its training rows,
// squared GEMM-form distances (the reference's euclidean_gemm_distance of the
// coarse step, approximate_neighbors.cpp:660-680, 1098-1104) or, for the
// inner-product and cosine indexes, the key -q.c (the GEMMs with alpha = -1
// of :712-727, 1094-1100), ties to the lower centroid (its first-minimum /
// strict-< heap rules).
template <typename T> da_status IVF<T>::make_coarse() {
    coarse.reset(new NN<T>(err, cuda, opts.single));
    auto &o = coarse->opts;
    const bool sph = metric == AM_IP || metric == AM_COS;
    if (o.set_string("metric", sph ? "inner product" : "sqeuclidean_gemm") != da_status_success ||
        o.set_string("algorithm", "brute") != da_status_success ||
        o.set_string("precision mode", "plain") != da_status_success ||
        o.set_string("storage order", "row-major") != da_status_success)
        return err->error(da_status_internal_error, "Could not configure the coarse quantiser.");
    return coarse->set_data(n_list, n_features, centroids.data(), n_features);
}

// train / train_ivfflat (approximate_neighbors.cpp:233-274, 334-490, 492-523):
// optional subsample (selection sampling on std::mt19937 seeded with "seed"),
// then Lloyd k-means with random-samples initialisation, one run,
// "k-means_iter" iterations at most, tolerance sqrt(eps).
template <typename T> da_status IVF<T>::train() {
    if (!train_data_set)
        return err->error(da_status_no_data,
                          "No data has been passed to the handle. Please call "
                          "da_approx_nn_set_training_data_s or da_approx_nn_set_training_data_d.");
    n_list = opts.i("n_list");
    max_iter = opts.i("k-means_iter");
    seed = opts.i("seed");
    train_fraction = (T)opts.r("train fraction");
    algo = opts.key("algorithm");
    metric = opts.key("metric");
    data_order = order();
    if (n_list > n_samples)
        return err->error(da_status_invalid_array_dimension,
                          "n_samples = " + std::to_string(n_samples) +
                              " must be at least as large as n_list = " + std::to_string(n_list));
    internal_seed = seed;
    if (internal_seed == -1) {
        std::random_device rd;
        internal_seed = (da_int)(rd() & 0x7fffffffu); // non-negative, no abs() overflow
    }
    std::mt19937 mt((unsigned)internal_seed);
    const bool cm = data_order == column_major;
    const T *tp = X_train;
    da_int tld = ldx_train, n_train = n_samples;
    std::vector<T> Xs;
    if (train_fraction < T(1)) {
        n_train = std::max((da_int)((T)n_samples * train_fraction), n_list);
        // selection sampling (da_std.hpp:102-118)
        std::vector<da_int> perm;
        da_int need = std::min(n_train, n_samples), pop = n_samples;
        for (da_int i = 0; need > 0; ++i, --pop) {
            std::uniform_int_distribution<da_int> dd(0, pop - 1);
            if (dd(mt) < need) {
                perm.push_back(i);
                --need;
            }
        }
        tld = cm ? n_train : n_features;
        Xs.assign((size_t)n_train * n_features, T(0));
        for (da_int i = 0; i < n_train; ++i)
            for (da_int j = 0; j < n_features; ++j)
                Xs[cm ? i + (size_t)j * tld : (size_t)i * tld + j] =
                    X_train[cm ? perm[i] + (size_t)j * ldx_train : (size_t)perm[i] * ldx_train + j];
        tp = Xs.data();
    }
    // the inner-product and cosine indexes quantise with spherical k-means on
    // the rows as given, normalised first for cosine (:368-456)
    const bool sph = metric == AM_IP || metric == AM_COS;
    if (metric == AM_COS) {
        if (Xs.empty()) {
            Xs = normalised_copy(cm, n_train, n_features, tp, tld, tld);
        } else {
            normalise_rows(cm, n_train, n_features, Xs.data(), tld);
        }
        tp = Xs.data();
    }
    KMeans<T> km(err, cuda, opts.single);
    auto &o = km.opts;
    if (o.set_int("n_clusters", n_list) != da_status_success ||
        o.set_int("n_init", 1) != da_status_success ||
        o.set_int("max_iter", max_iter) != da_status_success ||
        o.set_int("seed", internal_seed) != da_status_success ||
        o.set_string("initialization method", "random") != da_status_success ||
        o.set_string("algorithm", "lloyd") != da_status_success ||
        o.set_string("storage order", cm ? "column-major" : "row-major") != da_status_success ||
        o.set_real("convergence tolerance", std::sqrt(std::numeric_limits<T>::epsilon())) !=
            da_status_success ||
        (sph && (o.set_string("distance", "cosine") != da_status_success ||
                 o.set_string("normalize data", "no") != da_status_success)))
        return err->error(da_status_internal_error, "Could not configure the coarse k-means.");
    da_status s = km.set_data(n_train, n_features, tp, tld);
    if (s != da_status_success) return s;
    s = km.compute();
    if (s != da_status_success && s != da_status_maxit) return s;
    err->clear();
    kmeans_iter = km.best_n_iter;
    // the centres are column-major k x d; the index keeps them row-major
    centroids.assign((size_t)n_list * n_features, T(0));
    for (da_int c = 0; c < n_list; ++c)
        for (da_int j = 0; j < n_features; ++j)
            centroids[(size_t)c * n_features + j] = km.best_centres[c + (size_t)j * n_list];
    // train() empties the lists; the count of added rows and the "data added"
    // state stay as they were (approximate_neighbors.cpp:345-356)
    list_sizes.assign((size_t)n_list, 0);
    list_rows.assign((size_t)n_list, {});
    list_norms.assign((size_t)n_list, {});
    list_ids.assign((size_t)n_list, {});
    lists_on_device = false;
    s = make_coarse();
    if (s != da_status_success) return s;
    model_trained = true;
    return da_status_success;
}

// add / add_ivfflat (approximate_neighbors.cpp:525-842): every row joins the
// list of its nearest centroid, after the rows already there, with global
// index n_index + its row.
template <typename T> da_status IVF<T>::add(da_int n, da_int d, const T *X, da_int ldx) {
    if (!model_trained)
        return err->error(da_status_no_data,
                          "No index has been trained. Please call da_approx_nn_train_s or "
                          "da_approx_nn_train_d.");
    da_status s = check_options_update();
    if (s != da_status_success) return s;
    const da_order ord = order();
    s = check_2d(*err, ord, n, d, X, ldx, "n_samples", "n_features", "X_add", "ldx_add");
    if (s != da_status_success) return s;
    if (d != n_features)
        return err->error(da_status_invalid_input,
                          "The function was called with n_features = " + std::to_string(d) +
                              " but the index has been trained with " +
                              std::to_string(n_features) + " features.");
    const bool cm = ord == column_major;
    // cosine: the rows are normalised before they are assigned and stored
    // (approximate_neighbors.cpp:577-598)
    std::vector<T> Xn;
    if (metric == AM_COS) {
        Xn = normalised_copy(cm, n, d, X, ldx, ldx);
        X = Xn.data();
    }
    std::vector<da_int> near;
    s = coarse->kneighbors_compute(n, d, X, ldx, ord, 1, near, nullptr);
    if (s != da_status_success) return s;
    for (da_int i = 0; i < n; ++i) {
        const da_int c = near[i];
        auto &rows = list_rows[c];
        T norm = T(0);
        for (da_int j = 0; j < d; ++j) {
            const T v = X[cm ? i + (size_t)j * ldx : (size_t)i * ldx + j];
            rows.push_back(v);
            norm += v * v;
        }
        list_norms[c].push_back(norm);
        list_ids[c].push_back(i + n_index);
        list_sizes[c]++;
    }
    n_index += n;
    data_added = true;
    lists_on_device = false;
    return da_status_success;
}

template <typename T> da_status IVF<T>::train_and_add() {
    da_status s = train();
    if (s != da_status_success) return s;
    return add(n_samples, n_features, X_train, ldx_train);
}

// The lists as one list-ordered device array (rows padded to ld), with the
// squared norms, global indices and list offsets.
template <typename T> da_status IVF<T>::upload_lists() {
    da_status s = cuda->init(*err);
    if (s != da_status_success) return s;
    ld = pad4(n_features);
    const size_t rows = (size_t)std::max<da_int>(n_index, 1);
    std::vector<T> Xh(rows * ld, T(0)), xn(rows, T(0));
    std::vector<int> gid(rows, 0);
    std::vector<long long> off((size_t)n_list + 1, 0);
    size_t r = 0;
    for (da_int c = 0; c < n_list; ++c) {
        off[c] = (long long)r;
        for (size_t i = 0; i < list_ids[c].size(); ++i, ++r) {
            std::copy(list_rows[c].begin() + i * n_features,
                      list_rows[c].begin() + (i + 1) * n_features, Xh.begin() + r * ld);
            xn[r] = list_norms[c][i];
            gid[r] = (int)list_ids[c][i];
        }
    }
    off[n_list] = (long long)r;
    if (!dX.ensure(Xh.size() * sizeof(T)) || !dXn.ensure(xn.size() * sizeof(T)) ||
        !dGid.ensure(gid.size() * sizeof(int)) || !dOff.ensure(off.size() * sizeof(long long)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    cudaStream_t st = cuda->stream;
    B200_TRY(cudaMemcpyAsync(dX.p, Xh.data(), Xh.size() * sizeof(T), cudaMemcpyHostToDevice, st),
             "upload of the lists");
    B200_TRY(cudaMemcpyAsync(dXn.p, xn.data(), xn.size() * sizeof(T), cudaMemcpyHostToDevice, st),
             "upload of the lists");
    B200_TRY(cudaMemcpyAsync(dGid.p, gid.data(), gid.size() * sizeof(int), cudaMemcpyHostToDevice,
                             st),
             "upload of the lists");
    B200_TRY(cudaMemcpyAsync(dOff.p, off.data(), off.size() * sizeof(long long),
                             cudaMemcpyHostToDevice, st),
             "upload of the lists");
    B200_TRY(cudaStreamSynchronize(st), "upload of the lists");
    lists_on_device = true;
    return da_status_success;
}

// kneighbors / ivf_search (approximate_neighbors.cpp:858-942, 1193-1344):
// the n_probe nearest centroids of every query, then the k nearest rows of
// those lists; results in the storage order, index -1 and distance +inf
// where the probed lists hold fewer than k rows.
template <typename T>
da_status IVF<T>::kneighbors(da_int nq, da_int d, const T *Xt, da_int ldt, da_int *n_ind,
                             T *n_dist, da_int k, da_int return_distance) {
    if (!model_trained)
        return err->error(da_status_no_data,
                          "No index has been trained. Please call da_approx_nn_train_s or "
                          "da_approx_nn_train_d.");
    if (!data_added)
        return err->error(da_status_no_data,
                          "No data has been added. Please call da_approx_nn_add_s or "
                          "da_approx_nn_add_d");
    da_status s = check_options_update();
    if (s != da_status_success) return s;
    if (k <= 0) k = opts.i("number of neighbors");
    if (k > n_index)
        return err->error(da_status_invalid_input,
                          std::to_string(k) + " neighbors were requested but only " +
                              std::to_string(n_index) + " samples have been added to the index");
    if (n_probe > n_list)
        return err->error(da_status_invalid_input,
                          "n_probe=" + std::to_string(n_probe) +
                              " must be no larger than n_list=" + std::to_string(n_list));
    if (n_ind == nullptr) return err->error(da_status_invalid_pointer, "n_ind is not a valid pointer.");
    if (return_distance && n_dist == nullptr)
        return err->error(da_status_invalid_pointer, "n_dist is not a valid pointer.");
    const da_order ord = order();
    s = check_2d(*err, ord, nq, d, Xt, ldt, "n_samples", "n_features", "X_test", "ldx_test");
    if (s != da_status_success) return s;
    if (d != n_features)
        return err->error(da_status_invalid_input,
                          "The function was called with n_features = " + std::to_string(d) +
                              " but the index has been trained with " +
                              std::to_string(n_features) + " features.");
    const bool fp64 = sizeof(T) == 8;
    if (ivf_scan_smem((int)k, fp64) > (size_t)200 * 1024)
        return err->error(da_status_not_implemented,
                          "k = " + std::to_string(k) +
                              " exceeds the on-chip top-k of the B200 IVF-flat search.");
    // cosine: the queries are normalised first (approximate_neighbors.cpp:1066-1080)
    std::vector<T> Qn;
    if (metric == AM_COS) {
        Qn = normalised_copy(ord == column_major, nq, d, Xt, ldt, ldt);
        Xt = Qn.data();
    }
    std::vector<da_int> probe;
    s = coarse->kneighbors_compute(nq, d, Xt, ldt, ord, n_probe, probe, nullptr);
    if (s != da_status_success) return s;
    if (!lists_on_device) {
        s = upload_lists();
        if (s != da_status_success) return s;
    }
    cudaStream_t st = cuda->stream;
    std::vector<int> pr(probe.begin(), probe.end());
    const size_t nk = (size_t)nq * k;
    if (!dQ.ensure((size_t)nq * ld * sizeof(T)) || !dQn.ensure((size_t)nq * sizeof(T)) ||
        !dProbe.ensure(pr.size() * sizeof(int)) || !dOutD.ensure(nk * sizeof(T)) ||
        !dOutI.ensure(nk * sizeof(int)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(upload_matrix<T>(ord, nq, d, Xt, ldt, dQ.as<T>(), ld, dStage, st), "upload of X_test");
    B200_TRY(launch_row_sqnorms<T>(dQ.as<T>(), ld, nq, d, dQn.as<T>(), st), "query norms");
    B200_TRY(cudaMemcpyAsync(dProbe.p, pr.data(), pr.size() * sizeof(int), cudaMemcpyHostToDevice,
                             st),
             "upload of the probes");
    B200_TRY(cuda->timed("ivf_scan", [&] {
        return launch_ivf_scan<T>(dQ.as<T>(), dQn.as<T>(), ld, (int)nq, dProbe.as<int>(),
                                  (int)n_probe, dOff.as<long long>(), dX.as<T>(), dXn.as<T>(),
                                  dGid.as<int>(), (int)k,
                                  metric == AM_EUC   ? IVF_OUT_SQRT
                                  : metric == AM_IP  ? IVF_OUT_IP
                                  : metric == AM_COS ? IVF_OUT_COS
                                                     : IVF_OUT_SQ,
                                  dOutD.as<T>(), dOutI.as<int>(), st);
    }), "list scan");
    std::vector<int> oi(nk);
    std::vector<T> od(nk);
    B200_TRY(cudaMemcpyAsync(oi.data(), dOutI.p, nk * sizeof(int), cudaMemcpyDeviceToHost, st),
             "download");
    if (return_distance)
        B200_TRY(cudaMemcpyAsync(od.data(), dOutD.p, nk * sizeof(T), cudaMemcpyDeviceToHost, st),
                 "download");
    B200_TRY(cudaStreamSynchronize(st), "IVF-flat search");
    const bool cm = ord == column_major;
    for (da_int q = 0; q < nq; ++q)
        for (da_int r = 0; r < k; ++r) {
            const size_t src = (size_t)q * k + r, dst = cm ? q + (size_t)r * nq : src;
            n_ind[dst] = (da_int)oi[src];
            if (return_distance) n_dist[dst] = od[src];
        }
    return da_status_success;
}

// get_result (approximate_neighbors.cpp:62-150)
template <typename T> da_status IVF<T>::result_values(da_result q, da_int *dim, T *out) {
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "Index has not yet been trained. Please call da_approx_nn_train_d or "
                         "da_approx_nn_train_s before extracting results.");
    switch (q) {
    case da_rinfo:
        if (*dim < 4) {
            *dim = 4;
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: 4.");
        }
        out[0] = (T)n_list;
        out[1] = (T)n_index;
        out[2] = (T)n_features;
        out[3] = (T)kmeans_iter;
        return da_status_success;
    case da_approx_nn_cluster_centroids: {
        const da_int need = n_list * n_features;
        if (*dim < need) {
            *dim = need;
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: " +
                                 std::to_string(need) + ".");
        }
        const bool cm = data_order == column_major;
        for (da_int c = 0; c < n_list; ++c)
            for (da_int j = 0; j < n_features; ++j)
                out[cm ? c + (size_t)j * n_list : (size_t)c * n_features + j] =
                    centroids[(size_t)c * n_features + j];
        return da_status_success;
    }
    default:
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    }
}

template <typename T> da_status IVF<T>::get_result(da_result q, da_int *dim, double *out) {
    if constexpr (std::is_same_v<T, double>) return result_values(q, dim, out);
    (void)q, (void)dim, (void)out;
    return err->error(da_status_wrong_type, "Wrong precision type.");
}
template <typename T> da_status IVF<T>::get_result(da_result q, da_int *dim, float *out) {
    if constexpr (std::is_same_v<T, float>) return result_values(q, dim, out);
    (void)q, (void)dim, (void)out;
    return err->error(da_status_wrong_type, "Wrong precision type.");
}

template <typename T> da_status IVF<T>::get_result_int(da_result q, da_int *dim, da_int *out) {
    if (q == da_trained) return AlgBase::get_result_int(q, dim, out);
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "Index has not yet been trained. Please call da_approx_nn_train_d or "
                         "da_approx_nn_train_s before extracting results.");
    if (q != da_approx_nn_list_sizes)
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    if (*dim < n_list) {
        *dim = n_list;
        return err->warn(da_status_invalid_array_dimension,
                         "The array is too small. Please provide an array of at least size: " +
                             std::to_string(n_list) + ".");
    }
    for (da_int c = 0; c < n_list; ++c) out[c] = list_sizes[c];
    return da_status_success;
}

// Model persistence (approximate_neighbors.cpp:1346-1432 keeps the same
// state): the trained index -- centroids, run information and the lists in
// insertion order.  A loaded handle searches and accepts adds like the saved
// one; train() needs set_training_data again.
template <typename T> da_status IVF<T>::save_state(ByteWriter &w) {
    if (!model_trained)
        return err->error(da_status_no_data,
                          "No index has been trained. Please call da_approx_nn_train_s or "
                          "da_approx_nn_train_d before saving the model.");
    w.put<int64_t>(n_list);
    w.put<int64_t>(n_features);
    w.put<int64_t>(n_index);
    w.put<int64_t>(kmeans_iter);
    w.put<int32_t>((int32_t)algo);
    w.put<int32_t>((int32_t)metric);
    w.put<int32_t>((int32_t)data_order);
    w.put<int32_t>(data_added ? 1 : 0);
    w.put_vec(centroids.data(), centroids.size());
    std::vector<T> rows, norms;
    std::vector<int64_t> ids, sizes;
    for (da_int c = 0; c < n_list; ++c) {
        rows.insert(rows.end(), list_rows[c].begin(), list_rows[c].end());
        norms.insert(norms.end(), list_norms[c].begin(), list_norms[c].end());
        ids.insert(ids.end(), list_ids[c].begin(), list_ids[c].end());
        sizes.push_back(list_sizes[c]);
    }
    w.put_vec(sizes.data(), sizes.size());
    w.put_vec(ids.data(), ids.size());
    w.put_vec(norms.data(), norms.size());
    w.put_vec(rows.data(), rows.size());
    return da_status_success;
}

template <typename T> da_status IVF<T>::load_state(ByteReader &r) {
    const int64_t nl = r.get<int64_t>(), d = r.get<int64_t>(), ni = r.get<int64_t>(),
                  it = r.get<int64_t>();
    const int32_t al = r.get<int32_t>(), me = r.get<int32_t>(), ord = r.get<int32_t>(),
                  added = r.get<int32_t>();
    std::vector<T> cen = r.get_vec<T>();
    std::vector<int64_t> sizes = r.get_vec<int64_t>(), ids = r.get_vec<int64_t>();
    std::vector<T> norms = r.get_vec<T>(), rows = r.get_vec<T>();
    const auto bad = [&] {
        return err->error(da_status_invalid_file_data, "The model file is corrupted.");
    };
    // every size must fit da_int before the narrowing casts below, and the
    // products are formed only once both factors are in range
    const int64_t imax = (int64_t)std::numeric_limits<da_int>::max();
    if (!r.ok || nl < 1 || d < 1 || ni < 0 || nl > imax || d > imax || ni > imax ||
        sizes.size() != (size_t)nl || cen.size() / (size_t)nl != (size_t)d ||
        cen.size() != (size_t)nl * (size_t)d || ids.size() != norms.size() ||
        rows.size() / (size_t)d != ids.size() || rows.size() != ids.size() * (size_t)d ||
        me < AM_EUC || me > AM_COS)
        return bad();
    // list sizes: each within the listed rows before it is added (no overflow)
    int64_t total = 0;
    for (int64_t v : sizes) {
        if (v < 0 || v > (int64_t)ids.size() - total) return bad();
        total += v;
    }
    if (total != (int64_t)ids.size() || total > ni) return bad();
    for (int64_t v : ids)
        if (v < 0 || v >= ni) return bad();
    n_list = (da_int)nl;
    n_features = (da_int)d;
    n_index = (da_int)ni;
    kmeans_iter = (da_int)it;
    algo = al;
    metric = me;
    data_order = (da_order)ord;
    data_added = added != 0;
    centroids = std::move(cen);
    list_sizes.assign((size_t)nl, 0);
    list_rows.assign((size_t)nl, {});
    list_norms.assign((size_t)nl, {});
    list_ids.assign((size_t)nl, {});
    size_t o = 0;
    for (da_int c = 0; c < n_list; ++c) {
        const size_t m = (size_t)sizes[c];
        list_sizes[c] = (da_int)m;
        list_rows[c].assign(rows.begin() + o * d, rows.begin() + (o + m) * d);
        list_norms[c].assign(norms.begin() + o, norms.begin() + o + m);
        for (size_t i = 0; i < m; ++i) list_ids[c].push_back((da_int)ids[o + i]);
        o += m;
    }
    train_data_set = false;
    lists_on_device = false;
    model_trained = true;
    return make_coarse();
}

template struct IVF<float>;
template struct IVF<double>;

} // namespace b200
