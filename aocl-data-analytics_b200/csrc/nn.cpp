// Brute-force k-nearest-neighbours handle (host side).  Argument checks,
// option semantics and status codes follow
// source/core/nearest_neighbors/nearest_neighbors.cpp; the distance tile and
// the top-k selection run on the GPU (dist_simt.cu).
#include "alg.hpp"
#include <cstdlib>
#include <map>

namespace b200 {

// metric ids of the "metric" option (aoclda_metrics.h:44-59)
enum { M_EUC = 0, M_SQEUC = 1, M_MINK = 2, M_MANH = 3, M_COS = 4, M_EUC_GEMM = 5,
       M_SQEUC_GEMM = 6, M_IP = 7 };
// algorithm ids (nearest_neighbors_types.hpp:29)
enum { A_BRUTE = 0, A_KD = 1, A_BALL = 2, A_AUTO = 3 };
// "outlier handling" ids (nearest_neighbors_types.hpp)
enum { OH_NONE = 0, OH_MANUAL = 1, OH_MOST_FREQUENT = 2 };

template <typename T>
NN<T>::NN(ErrorRecord *e, CudaCtx *c, bool single) {
    err = e;
    cuda = c;
    opts.single = single;
    register_common_options(opts);
    // nearest_neighbors_options.hpp:52-124
    const da_int imax = std::numeric_limits<da_int>::max();
    const da_int imin = std::numeric_limits<da_int>::min();
    const double fmax = (double)std::numeric_limits<T>::max();
    const double flow = (double)std::numeric_limits<T>::lowest();
    opts.add_int("number of neighbors", 1, LB::greaterequal, imax, UB::p_inf, 5);
    opts.add_int("leaf size", 1, LB::greaterequal, imax, UB::p_inf, 30);
    opts.add_int("outlier label", imin, LB::m_inf, imax, UB::p_inf, 0);
    opts.add_real("minkowski parameter", 0.0, LB::greaterthan, fmax, UB::p_inf, 2.0);
    opts.add_real("radius", 0.0, LB::greaterequal, fmax, UB::p_inf, 1.0);
    opts.add_real("outlier target", flow, LB::m_inf, fmax, UB::p_inf, 0.0);
    opts.add_string("algorithm",
                    {{"auto", A_AUTO}, {"brute", A_BRUTE}, {"kd tree", A_KD}, {"ball tree", A_BALL}},
                    "auto");
    opts.add_string("metric",
                    {{"euclidean", M_EUC},
                     {"l2", M_EUC},
                     {"sqeuclidean", M_SQEUC},
                     {"manhattan", M_MANH},
                     {"l1", M_MANH},
                     {"cityblock", M_MANH},
                     {"cosine", M_COS},
                     {"minkowski", M_MINK},
                     {"sqeuclidean_gemm", M_SQEUC_GEMM},
                     {"euclidean_gemm", M_EUC_GEMM},
                     {"inner product", M_IP}},
                    "euclidean");
    opts.add_string("weights", {{"uniform", 0}, {"distance", 1}}, "uniform");
    opts.add_string("outlier handling",
                    {{"none", OH_NONE}, {"manual", OH_MANUAL}, {"most frequent", OH_MOST_FREQUENT}},
                    "none");
    // B200 options (no counterpart in the reference):
    //   "reference isa": which AOCL-DA build's KC blocking the squared-euclidean
    //   summation order reproduces (avx512: KC=256/512, avx2: KC=64/32).
    opts.add_string("reference isa", {{"avx512", 0}, {"avx2", 1}}, "avx512");
    //   "precision mode": "bf16x3" lets large fp32 euclidean searches run a
    //   tensor-core candidate pass with an exact re-score (same neighbours and
    //   distances as "plain", the SIMT fp32 path).
    opts.add_string("precision mode", {{"plain", 0}, {"bf16x3", 3}}, "bf16x3");
}

template <typename T> da_status NN<T>::set_params() {
    n_neighbors = opts.i("number of neighbors");
    algo = opts.key("algorithm");
    metric = opts.key("metric");
    weights = opts.key("weights");
    p = (T)opts.r("minkowski parameter");
    // Tree algorithms reject non-metric distances (nearest_neighbors.cpp:313-330).
    if (algo == A_KD || algo == A_BALL) {
        if (metric == M_COS || metric == M_SQEUC || metric == M_SQEUC_GEMM || metric == M_IP)
            return err->error(da_status_incompatible_options,
                              "The tree algorithms are not compatible with the cosine, squared "
                              "Euclidean, or inner product distances.");
        if (metric == M_MINK && p < T(1))
            return err->error(da_status_incompatible_options,
                              "Tree algorithms are not compatible with the Minkowski metric when "
                              "0 < p < 1.");
    }
    up_to_date = true;
    return da_status_success;
}

// nearest_neighbors.cpp:398-466: after set_data the tree-related options are
// locked.  As in the reference, "number of neighbors", "metric", "weights" and
// "minkowski parameter" are read when the training data are set
// (set_params, nearest_neighbors.cpp:497-499) and not re-read afterwards.
template <typename T> da_status NN<T>::check_options_update() {
    const da_int a = opts.key("algorithm");
    if (a == A_AUTO || a == A_KD || a == A_BALL) {
        if (a != locked_algo || opts.i("leaf size") != locked_leaf)
            return err->error(da_status_option_locked,
                              "Options need to be set before calling set_training_data().");
        if (a == A_AUTO &&
            (opts.key("metric") != locked_metric || (T)opts.r("minkowski parameter") != locked_p))
            return err->error(da_status_option_locked,
                              "Options need to be set before calling set_training_data().");
    }
    return da_status_success;
}

template <typename T>
da_status NN<T>::set_data(da_int n, da_int d, const T *X, da_int ldx) {
    if (n_samples > 0 && n != n_samples)
        return err->error(da_status_invalid_array_dimension,
                          "n_samples = " + std::to_string(n) +
                              " doesn't match the training data size " +
                              std::to_string(n_samples) + ".");
    const da_order ord = order();
    da_status s = check_2d(*err, ord, n, d, X, ldx, "n_samples", "n_features", "X_train",
                           "ldx_train", 1, 1, opts.key("check data") == 1);
    if (s != da_status_success) return s;
    n_samples = n;
    n_features = d;
    X_host = X;
    ldx_host = ldx;
    data_order = ord;
    have_X = true;
    X_on_device = false;
    xn_kind = -1;
    s = set_params();
    if (s != da_status_success) return s;
    locked_algo = algo;
    locked_leaf = opts.i("leaf size");
    locked_metric = metric;
    locked_p = p;
    // Upload now when a device is present (the reference keeps the user's
    // pointer; an eager device copy is a safe superset of that contract).
    if (cuda->init(*err) == da_status_success) {
        s = ensure_device_data();
        if (s != da_status_success) return s;
    } else {
        err->clear();
    }
    return da_status_success;
}

// The training data of `src` (same precision and storage order, same device):
// this handle takes its host pointers (rows, labels, targets) as set_data /
// set_labels / set_targets would, and holds the same device copies of the
// rows -- fp32/fp64 rows, and the tensor-core bf16 pair and norms when src
// has built them -- instead of uploading its own.  Neither handle writes into
// a shared copy: a later set_data on either gives that handle new buffers.
template <typename T> da_status NN<T>::share_data(NN<T> &src) {
    if (!src.have_X)
        return err->error(da_status_no_data, "The source handle holds no training data.");
    if (src.order() != order())
        return err->error(da_status_invalid_input,
                          "The two handles have different storage orders.");
    if (n_samples > 0 && src.n_samples != n_samples)
        return err->error(da_status_invalid_array_dimension,
                          "n_samples = " + std::to_string(src.n_samples) +
                              " doesn't match the training data size " +
                              std::to_string(n_samples) + ".");
    da_status s = cuda->init(*err);
    if (s != da_status_success) return s;
    if (src.cuda->init(*src.err) != da_status_success || src.ensure_device_data() != da_status_success)
        return err->error(da_status_memory_error,
                          "The source handle's training data are not on the device: " +
                              src.err->message);
    if (src.cuda->device != cuda->device)
        return err->error(da_status_invalid_input, "The two handles use different devices.");
    // the source's uploads are complete before this handle's stream reads them
    B200_TRY(cudaStreamSynchronize(src.cuda->stream), "synchronisation with the source handle");
    n_samples = src.n_samples;
    n_features = src.n_features;
    X_host = src.X_host;
    if (!src.X_own.empty()) { // a loaded source owns its rows: keep a copy
        X_own = src.X_own;
        X_host = X_own.data();
    }
    ldx_host = src.ldx_host;
    data_order = src.data_order;
    have_X = true;
    s = set_params();
    if (s != da_status_success) return s;
    locked_algo = algo;
    locked_leaf = opts.i("leaf size");
    locked_metric = metric;
    locked_p = p;
    ld = src.ld;
    dX.share(src.dX);
    X_on_device = true;
    xn_kind = -1;
    tc_train_ready = false;
    if (src.tc_train_ready) {
        // max |x| is the first scalar of the tensor-core state; the rest of
        // that buffer is per call
        if (!dTkScal.ensure(64))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        B200_TRY(cudaMemcpyAsync(dTkScal.p, src.dTkScal.p, 16, cudaMemcpyDeviceToDevice,
                                 cuda->stream),
                 "copy");
        dXh.share(src.dXh);
        dXl.share(src.dXl);
        dXsq.share(src.dXsq);
        tc_ldbf = src.tc_ldbf;
        tc_train_ready = true;
    }
    if (src.have_labels) {
        const da_int *y = src.y_class;
        if (!src.y_own.empty()) {
            y_own = src.y_own;
            y = y_own.data();
        }
        s = set_labels(src.n_samples, y);
        if (s != da_status_success) return s;
    }
    if (src.have_targets) {
        const T *y = src.y_reg;
        if (!src.t_own.empty()) {
            t_own = src.t_own;
            y = t_own.data();
        }
        s = set_targets(src.n_samples, y);
        if (s != da_status_success) return s;
    }
    return da_status_success;
}

// Model persistence: the training rows in their storage order (dense), then
// the labels and targets when set.  Loading replays set_data / set_labels /
// set_targets on the handle's own copies (the options were loaded first).
template <typename T> da_status NN<T>::save_state(ByteWriter &w) {
    if (!have_X)
        return err->error(da_status_no_data,
                          "No training data have been set. Please call da_nn_set_data_s or "
                          "da_nn_set_data_d before saving the model.");
    const bool rm = data_order == row_major;
    std::vector<T> X((size_t)n_samples * n_features);
    for (da_int i = 0; i < n_samples; ++i)
        for (da_int j = 0; j < n_features; ++j)
            X[rm ? (size_t)i * n_features + j : i + (size_t)j * n_samples] =
                X_host[rm ? (size_t)i * ldx_host + j : i + (size_t)j * ldx_host];
    w.put<int64_t>(n_samples);
    w.put<int64_t>(n_features);
    w.put<int32_t>((int32_t)data_order);
    w.put_vec(X.data(), X.size());
    w.put<int32_t>(have_labels ? 1 : 0);
    if (have_labels) w.put_vec(y_class, (size_t)n_samples);
    w.put<int32_t>(have_targets ? 1 : 0);
    if (have_targets) w.put_vec(y_reg, (size_t)n_samples);
    return da_status_success;
}

template <typename T> da_status NN<T>::load_state(ByteReader &r) {
    const int64_t n = r.get<int64_t>(), d = r.get<int64_t>();
    const int32_t ord = r.get<int32_t>();
    X_own = r.get_vec<T>();
    if (!r.ok || n < 1 || d < 1 || X_own.size() != (size_t)(n * d) || ord != (int32_t)order())
        return err->error(da_status_invalid_file_data, "The model file is corrupted.");
    da_status s = set_data((da_int)n, (da_int)d, X_own.data(),
                           ord == row_major ? (da_int)d : (da_int)n);
    if (s != da_status_success) return s;
    if (r.get<int32_t>()) {
        y_own = r.get_vec<da_int>();
        if (!r.ok || y_own.size() != (size_t)n)
            return err->error(da_status_invalid_file_data, "The model file is corrupted.");
        s = set_labels((da_int)n, y_own.data());
        if (s != da_status_success) return s;
    }
    if (r.get<int32_t>()) {
        t_own = r.get_vec<T>();
        if (!r.ok || t_own.size() != (size_t)n)
            return err->error(da_status_invalid_file_data, "The model file is corrupted.");
        s = set_targets((da_int)n, t_own.data());
        if (s != da_status_success) return s;
    }
    if (!r.ok) return err->error(da_status_invalid_file_data, "The model file is corrupted.");
    return da_status_success;
}

template <typename T> da_status NN<T>::ensure_device_data() {
    da_status s = cuda->init(*err);
    if (s != da_status_success) return s;
    if (X_on_device) return da_status_success;
    ld = pad4(n_features);
    if (!dX.ensure((size_t)n_samples * ld * sizeof(T)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(upload_matrix<T>(data_order, n_samples, n_features, X_host, ldx_host, dX.as<T>(),
                              ld, dStage, cuda->stream),
             "upload of X_train");
    X_on_device = true;
    xn_kind = -1;
    tc_train_ready = false;
    return da_status_success;
}

// Tensor-core candidate pass + exact re-score (knn_tc.cu) into dOutK / dOutI,
// in query batches that bound the candidate lists' memory.  Any query the
// pass could not certify sends the whole call to the plain path (done =
// false).
template <typename T>
da_status NN<T>::kneighbors_tc(da_int nq, da_int d, da_int k, int kc, bool take_sqrt,
                                bool cosine, bool &done) {
    done = false;
    if constexpr (std::is_same_v<T, float>) {
        cudaStream_t st = cuda->stream;
        if (cosine) {
            // the plain path's norms of the training rows and queries, and the
            // reciprocals of the former
            if (!dQn.ensure((size_t)nq * sizeof(T)) || !dXn.ensure((size_t)n_samples * sizeof(T)) ||
                !dXinv.ensure((size_t)n_samples * sizeof(float)))
                return err->error(da_status_memory_error, "Device memory allocation failed.");
            B200_TRY(launch_row_norms_eps1<float>(dQ.as<float>(), ld, (int)nq, (int)d,
                                                  dQn.as<float>(), st), "norms");
            if (xn_kind != 1)
                B200_TRY(launch_row_norms_eps1<float>(dX.as<float>(), ld, (int)n_samples, (int)d,
                                                      dXn.as<float>(), st), "norms");
            xn_kind = 1;
            B200_TRY(launch_recip(dXn.as<float>(), (int)n_samples, dXinv.as<float>(), st),
                     "norms");
        }
        // bf16 rows of d rounded up to 8 (at least 64): no padded K block is
        // stored or read (the tensor maps zero-fill past the row)
        const int ldbf = d <= 64 ? 64 : (int)((d + 7) / 8 * 8);
        if (!tc_train_ready || tc_ldbf != ldbf) {
            tc_ldbf = ldbf;
            const size_t xb = (size_t)n_samples * tc_ldbf * 2;
            if (!dXh.ensure(xb) || !dXl.ensure(xb) || !dXsq.ensure((size_t)n_samples * 4) ||
                !dTkScal.ensure(64))
                return err->error(da_status_memory_error, "Device memory allocation failed.");
            B200_TRY(launch_knn_tc_train_prep(dX.as<float>(), ld, (int)n_samples, (int)d, dXh.p,
                                              dXl.p, tc_ldbf, dXsq.as<float>(),
                                              dTkScal.as<float>(), st),
                     "tensor-core training copies");
            tc_train_ready = true;
        }
        const da_int QB = 16384;
        const da_int qb = std::min(nq, QB);
        if (!dTkQ.ensure(knn_tc_query_bytes((int)qb, (int)d)) ||
            !dTkList.ensure((size_t)qb * knn_tc_list_cap() * 8) ||
            !dTkFlag.ensure((size_t)qb * sizeof(int)) ||
            !dOutK.ensure((size_t)nq * k * sizeof(float)) ||
            !dOutI.ensure((size_t)nq * k * sizeof(int)))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        int *n_fb = reinterpret_cast<int *>(dTkScal.as<char>() + 16);
        int *errf = n_fb + 1;
        int h_state[5] = {0, 0, 0, 0, 0};
        for (da_int q0 = 0; q0 < nq; q0 += QB) {
            const da_int nb = std::min(QB, nq - q0);
            const KnnTcCosine cs{dXn.as<float>(), dXinv.as<float>(),
                                 cosine ? dQn.as<float>() + q0 : nullptr};
            B200_TRY(cuda->timed("knn_tc", [&] {
                return launch_knn_tc(dX.as<float>(), dXh.p, dXl.p, dXsq.as<float>(),
                                     dTkScal.as<float>(), (int)n_samples, ld, tc_ldbf, (int)d,
                                     dQ.as<float>() + (size_t)q0 * ld, (int)nb, (int)k, kc,
                                     take_sqrt ? 1 : 0, dTkQ.p, dTkList.p, dTkFlag.as<int>(),
                                     n_fb, errf, dOutK.as<float>() + (size_t)q0 * k,
                                     dOutI.as<int>() + (size_t)q0 * k, st,
                                     cosine ? &cs : nullptr);
            }), "kNN tensor-core pass");
            B200_TRY(cudaMemcpyAsync(h_state, n_fb, 5 * sizeof(int), cudaMemcpyDeviceToHost, st),
                     "copy");
            std::vector<int> lens((size_t)nb);
            B200_TRY(cudaMemcpyAsync(lens.data(), knn_tc_counts(dTkQ.p, (int)nb, (int)d),
                                     lens.size() * sizeof(int), cudaMemcpyDeviceToHost, st),
                     "copy");
            B200_TRY(cudaStreamSynchronize(st), "kNN tensor-core pass");
            double mx = 0, sum = 0;
            for (int v : lens) {
                mx = std::max(mx, (double)v);
                sum += v;
            }
            cuda->stats["knn_tc_max_list"] = std::max(cuda->stats["knn_tc_max_list"], mx);
            cuda->stats["knn_tc_mean_list"] = sum / std::max<double>(1.0, (double)nb);
            if (h_state[1] != 0)
                return err->error(da_status_internal_error,
                                  "The tensor-core kNN kernel timed out waiting on a pipeline "
                                  "barrier (code " + std::to_string(h_state[1]) + ").");
            cuda->stats["knn_tc_fallback_queries"] += (double)h_state[0];
            cuda->stats["knn_tc_fallback_list_overflow"] += (double)h_state[2];
            cuda->stats["knn_tc_fallback_many_survivors"] += (double)h_state[3];
            cuda->stats["knn_tc_fallback_few_survivors"] += (double)h_state[4];
            if (h_state[0] != 0) {
                // the queries the pass could not certify: the plain path on
                // just those rows (gathered, searched, scattered back)
                std::vector<int> flags((size_t)nb), idx;
                B200_TRY(cudaMemcpyAsync(flags.data(), dTkFlag.p, flags.size() * sizeof(int),
                                         cudaMemcpyDeviceToHost, st), "copy");
                B200_TRY(cudaStreamSynchronize(st), "copy");
                for (int i = 0; i < (int)nb; ++i)
                    if (flags[i]) idx.push_back(i);
                const int m = (int)idx.size();
                const int BN = knn_tile_rows_train(false);
                const int q_tiles = (m + 63) / 64;
                const int max_chunks = std::max(1, (int)((n_samples + BN - 1) / BN));
                // enough CTAs to fill the GPU, but at most ~16K partial entries per query
                // (the merge ranks every entry against every chunk list)
                int n_chunks = std::max(1, std::min({max_chunks, (148 * 8 + q_tiles - 1) / q_tiles,
                                                     std::max(8, 16384 / (int)k)}));
                int chunk_rows = (int)((n_samples + n_chunks - 1) / n_chunks);
                chunk_rows = ((chunk_rows + BN - 1) / BN) * BN;
                n_chunks = (int)((n_samples + chunk_rows - 1) / chunk_rows);
                // scratch inside the (now free) candidate-list buffer
                const size_t parts = (size_t)m * n_chunks * k;
                const size_t need = (size_t)m * 4 + (size_t)m * ld * 4 + parts * 8 +
                                    (size_t)m * k * 8 + (size_t)m * 4 + 1280;
                if (!dTkList.ensure(need))
                    return err->error(da_status_memory_error, "Device memory allocation failed.");
                char *p = dTkList.as<char>();
                int *didx = reinterpret_cast<int *>(p);
                float *qsub = reinterpret_cast<float *>(p + ((size_t)m * 4 + 255) / 256 * 256);
                float *pk = qsub + (size_t)m * ld;
                int *pi = reinterpret_cast<int *>(pk + parts);
                float *ok = reinterpret_cast<float *>(pi + parts);
                int *oi = reinterpret_cast<int *>(ok + (size_t)m * k);
                float *qnsub = reinterpret_cast<float *>(oi + (size_t)m * k);
                KnnArgs pa{cosine ? ACC_DOT : ACC_SQEUC, cosine ? POST_COSINE : POST_NONE, kc, 2.0,
                           (int)k, chunk_rows, n_chunks};
                B200_TRY(cudaMemcpyAsync(didx, idx.data(), (size_t)m * 4, cudaMemcpyHostToDevice,
                                         st), "copy");
                B200_TRY(launch_rows_gather(dQ.as<float>() + (size_t)q0 * ld, ld, didx, m, qsub,
                                            st), "gather");
                if (cosine)
                    B200_TRY(launch_rows_gather(dQn.as<float>() + q0, 1, didx, m, qnsub, st),
                             "gather");
                B200_TRY(launch_knn_chunks<float>(qsub, ld, m, dX.as<float>(), ld,
                                                  (int)n_samples, (int)d,
                                                  cosine ? qnsub : nullptr,
                                                  cosine ? dXn.as<float>() : nullptr, pa, pk,
                                                  pi, nullptr, st), "kNN distance kernel");
                B200_TRY(launch_knn_merge<float>(pk, pi, m, n_chunks, (int)k,
                                                 take_sqrt && !cosine ? 1 : 0, ok, oi, st),
                         "kNN merge kernel");
                B200_TRY(launch_results_scatter(ok, oi, didx, m, (int)k,
                                                dOutK.as<float>() + (size_t)q0 * k,
                                                dOutI.as<int>() + (size_t)q0 * k, st), "scatter");
                B200_TRY(cudaStreamSynchronize(st), "kNN fallback");
            }
        }
        cuda->stats["tensor_core"] = 1.0;
        done = true;
    } else {
        (void)nq;
        (void)d;
        (void)k;
        (void)kc;
        (void)take_sqrt;
        (void)cosine;
    }
    return da_status_success;
}

template <typename T> da_status NN<T>::set_labels(da_int n, const da_int *y) {
    if (n_samples > 0 && n != n_samples)
        return err->error(da_status_invalid_array_dimension,
                          "n_samples = " + std::to_string(n) +
                              " doesn't match the training data size " +
                              std::to_string(n_samples) + ".");
    if (n < 1)
        return err->error(da_status_invalid_array_dimension,
                          "The function was called with n_samples = " + std::to_string(n) +
                              ". Constraint: n_samples >= 1.");
    if (y == nullptr) return err->error(da_status_invalid_pointer, "The array y_train_class is null.");
    n_samples = n;
    y_class = y;
    have_labels = true;
    classes_done = false;
    return da_status_success;
}

template <typename T> da_status NN<T>::set_targets(da_int n, const T *y) {
    if (n_samples > 0 && n != n_samples)
        return err->error(da_status_invalid_array_dimension,
                          "n_samples = " + std::to_string(n) +
                              " doesn't match the training data size " +
                              std::to_string(n_samples) + ".");
    if (n < 1)
        return err->error(da_status_invalid_array_dimension,
                          "The function was called with n_samples = " + std::to_string(n) +
                              ". Constraint: n_samples >= 1.");
    if (y == nullptr) return err->error(da_status_invalid_pointer, "The array y_train_reg is null.");
    n_samples = n;
    y_reg = y;
    have_targets = true;
    return da_status_success;
}

template <typename T>
da_status NN<T>::validate_queries(da_int nq, da_int d, const T *Xt, da_int ldt) {
    if (Xt == nullptr) return err->error(da_status_invalid_pointer, "X_test is not a valid pointer.");
    if (d != n_features)
        return err->error(da_status_invalid_array_dimension,
                          "n_features = " + std::to_string(d) +
                              " doesn't match the expected value " +
                              std::to_string(n_features) + ".");
    return check_2d(*err, order(), nq, d, Xt, ldt, "n_queries", "n_features", "X_test",
                    "ldx_test", 1, 1, opts.key("check data") == 1);
}

// Run the fused distance + top-k kernels; ind/dist are q-major (q*k + r).
template <typename T>
da_status NN<T>::kneighbors_compute(da_int nq, da_int d, const T *Xt, da_int ldt, da_order ord,
                                    da_int k, std::vector<da_int> &ind, std::vector<T> *dist) {
    da_status s = ensure_device_data();
    if (s != da_status_success) return s;
    cudaStream_t st = cuda->stream;
    // metric -> accumulation family, selection key and output transform
    int acc = ACC_SQEUC, post = POST_NONE, tf = 0, norm_kind = -1;
    switch (metric) {
    case M_EUC: acc = ACC_SQEUC; post = POST_NONE; tf = 1; break;
    case M_SQEUC: acc = ACC_SQEUC; post = POST_NONE; break;
    case M_EUC_GEMM: acc = ACC_DOT; post = POST_GEMM_SQ_CLAMP; tf = 1; norm_kind = 0; break;
    case M_SQEUC_GEMM: acc = ACC_DOT; post = POST_GEMM_SQ_CLAMP; norm_kind = 0; break;
    case M_MANH: acc = ACC_MANHATTAN; break;
    case M_COS: acc = ACC_DOT; post = POST_COSINE; norm_kind = 1; break;
    case M_IP: acc = ACC_DOT; post = POST_NEG; tf = 2; break;
    case M_MINK:
        if (p == T(2)) { acc = ACC_SQEUC; tf = 1; }
        else if (p == T(1)) { acc = ACC_MANHATTAN; }
        else { acc = ACC_MINKOWSKI; post = POST_POW; }
        break;
    }
    const bool fp64 = sizeof(T) == 8;
    const int kc = opts.key("reference isa") == 1 ? (fp64 ? 32 : 64) : (fp64 ? 512 : 256);
    // queries -> device
    if (!dQ.ensure((size_t)nq * ld * sizeof(T)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(upload_matrix<T>(ord, nq, d, Xt, ldt, dQ.as<T>(), ld, dStage, st), "upload of X_test");
    cuda->stats["tensor_core"] = 0.0;
    cuda->stats["knn_tc_fallback_queries"] = 0.0;
    cuda->stats["knn_tc_fallback_list_overflow"] = 0.0;
    cuda->stats["knn_tc_fallback_many_survivors"] = 0.0;
    cuda->stats["knn_tc_fallback_few_survivors"] = 0.0;
    bool tc_done = false;
    const bool tc_metric = metric == M_EUC || metric == M_SQEUC || metric == M_COS ||
                           (metric == M_MINK && p == T(2));
    if (!fp64 && tc_metric && opts.key("precision mode") != 0 &&
        knn_tc_supported((int)n_samples, (int)d, (int)k) && n_samples >= 65536 &&
        (double)n_samples * (double)std::max<da_int>(nq, 256) * (double)d >= 4.0e9) {
        s = kneighbors_tc(nq, d, k, kc, metric != M_SQEUC && metric != M_COS, metric == M_COS,
                          tc_done);
        if (s != da_status_success) return s;
    }
    if (!tc_done) {
        const T *qn = nullptr, *xn = nullptr;
        if (norm_kind >= 0) {
            if (!dQn.ensure((size_t)nq * sizeof(T)) || !dXn.ensure((size_t)n_samples * sizeof(T)))
                return err->error(da_status_memory_error, "Device memory allocation failed.");
            if (norm_kind == 0) {
                B200_TRY(launch_row_sqnorms<T>(dQ.as<T>(), ld, nq, d, dQn.as<T>(), st), "norms");
                if (xn_kind != 0)
                    B200_TRY(launch_row_sqnorms<T>(dX.as<T>(), ld, n_samples, d, dXn.as<T>(), st), "norms");
            } else {
                B200_TRY(launch_row_norms_eps1<T>(dQ.as<T>(), ld, nq, d, dQn.as<T>(), st), "norms");
                if (xn_kind != 1)
                    B200_TRY(launch_row_norms_eps1<T>(dX.as<T>(), ld, n_samples, d, dXn.as<T>(), st), "norms");
            }
            xn_kind = norm_kind;
            qn = dQn.as<T>();
            xn = dXn.as<T>();
        }
        if (k > knn_max_k(fp64))
            return err->error(da_status_not_implemented,
                              "k = " + std::to_string(k) + " exceeds the largest supported number "
                              "of neighbours per query (" + std::to_string(knn_max_k(fp64)) + ").");
        // chunking of the training rows: enough CTAs to fill 148 SMs several times
        const int BN = knn_tile_rows_train(fp64);
        const int q_tiles = (int)((nq + 63) / 64);
        const int max_chunks = std::max(1, (int)((n_samples + BN - 1) / BN));
        // enough CTAs to fill the GPU, but at most ~16K partial entries per query
        // (the merge ranks every entry against every chunk list)
        int n_chunks = std::max(1, std::min({max_chunks, (148 * 8 + q_tiles - 1) / q_tiles,
                                             std::max(8, 16384 / (int)k)}));
        int chunk_rows = (int)((n_samples + n_chunks - 1) / n_chunks);
        chunk_rows = ((chunk_rows + BN - 1) / BN) * BN;
        n_chunks = (int)((n_samples + chunk_rows - 1) / chunk_rows);
        KnnArgs a{acc, post, kc, (double)p, (int)k, chunk_rows, n_chunks};
        const size_t parts = (size_t)nq * n_chunks * k;
        if (!dPartK.ensure(parts * sizeof(T)) || !dPartI.ensure(parts * sizeof(int)) ||
            !dOutK.ensure((size_t)nq * k * sizeof(T)) || !dOutI.ensure((size_t)nq * k * sizeof(int)))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        B200_TRY(cuda->timed("knn_chunks", [&] {
            return launch_knn_chunks<T>(dQ.as<T>(), ld, (int)nq, dX.as<T>(), ld, (int)n_samples,
                                        (int)d, qn, xn, a, dPartK.as<T>(), dPartI.as<int>(), nullptr,
                                        st);
        }), "kNN distance kernel");
        B200_TRY(cuda->timed("knn_merge", [&] {
            return launch_knn_merge<T>(dPartK.as<T>(), dPartI.as<int>(), (int)nq, n_chunks, (int)k,
                                       tf, dOutK.as<T>(), dOutI.as<int>(), st);
        }), "kNN merge kernel");
    }
    ind.resize((size_t)nq * k);
    std::vector<int> tmp((size_t)nq * k);
    B200_TRY(cudaMemcpyAsync(tmp.data(), dOutI.p, tmp.size() * sizeof(int), cudaMemcpyDeviceToHost, st),
             "download");
    if (dist) {
        dist->resize((size_t)nq * k);
        B200_TRY(cudaMemcpyAsync(dist->data(), dOutK.p, dist->size() * sizeof(T),
                                 cudaMemcpyDeviceToHost, st), "download");
    }
    B200_TRY(cudaStreamSynchronize(st), "kNN");
    for (size_t i = 0; i < tmp.size(); ++i) ind[i] = (da_int)tmp[i];
    return da_status_success;
}

// Core of the radius search (radius_neighbors_compute, nearest_neighbors.cpp:
// 1983-2068): per query its count and start in the flat index / value arrays,
// rows in index order; values (only when want_val) as computed, squared for
// euclidean (`squares`).  Options and queries are validated by the caller.
template <typename T>
da_status NN<T>::radius_compute(da_int nq, da_int d, const T *Xt, da_int ldt, T r, bool want_val,
                                std::vector<da_int> &cnt_out, std::vector<long long> &start_out,
                                std::vector<da_int> &idx_out, std::vector<T> &val_out,
                                bool &squares) {
    da_status s;
    cnt_out.assign((size_t)nq, 0);
    start_out.assign((size_t)nq, 0);
    idx_out.clear();
    val_out.clear();
    s = ensure_device_data();
    if (s != da_status_success) return s;
    cudaStream_t st = cuda->stream;
    int acc = ACC_SQEUC, post = POST_NONE, tf = 0, norm_kind = -1;
    switch (metric) {
    case M_EUC: acc = ACC_SQEUC; tf = 1; break;
    case M_SQEUC: acc = ACC_SQEUC; break;
    case M_EUC_GEMM: acc = ACC_DOT; post = POST_GEMM_SQ_CLAMP; tf = 1; norm_kind = 0; break;
    case M_SQEUC_GEMM: acc = ACC_DOT; post = POST_GEMM_SQ_CLAMP; norm_kind = 0; break;
    case M_MANH: acc = ACC_MANHATTAN; break;
    case M_COS: acc = ACC_DOT; post = POST_COSINE; norm_kind = 1; break;
    case M_IP: acc = ACC_DOT; break; // radius predict only: rows with dot <= r
    case M_MINK:
        if (p == T(2)) { acc = ACC_SQEUC; tf = 1; }
        else if (p == T(1)) { acc = ACC_MANHATTAN; }
        else { acc = ACC_MINKOWSKI; post = POST_POW; }
        break;
    }
    squares = tf == 1;
    const T thr = squares ? r * r : r;
    const bool fp64 = sizeof(T) == 8;
    const int kc = opts.key("reference isa") == 1 ? (fp64 ? 32 : 64) : (fp64 ? 512 : 256);
    if (!dQ.ensure((size_t)nq * ld * sizeof(T)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    B200_TRY(upload_matrix<T>(order(), nq, d, Xt, ldt, dQ.as<T>(), ld, dStage, st), "upload of X_test");
    const T *qn = nullptr, *xn = nullptr;
    if (norm_kind >= 0) {
        if (!dQn.ensure((size_t)nq * sizeof(T)) || !dXn.ensure((size_t)n_samples * sizeof(T)))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        if (norm_kind == 0) {
            B200_TRY(launch_row_sqnorms<T>(dQ.as<T>(), ld, nq, d, dQn.as<T>(), st), "norms");
            if (xn_kind != 0)
                B200_TRY(launch_row_sqnorms<T>(dX.as<T>(), ld, n_samples, d, dXn.as<T>(), st), "norms");
        } else {
            B200_TRY(launch_row_norms_eps1<T>(dQ.as<T>(), ld, nq, d, dQn.as<T>(), st), "norms");
            if (xn_kind != 1)
                B200_TRY(launch_row_norms_eps1<T>(dX.as<T>(), ld, n_samples, d, dXn.as<T>(), st), "norms");
        }
        xn_kind = norm_kind;
        qn = dQn.as<T>();
        xn = dXn.as<T>();
    }
    // query blocks whose distance rows fit in 256 MB
    const size_t n = (size_t)n_samples;
    // (at most 65,535 rows: the count / compaction grids put the rows on y)
    // (and a whole number of the distance kernel's 64-row tiles when there
    // are more queries: a partial last tile row costs a full one)
    da_int B = (da_int)std::max<size_t>(
        1, std::min<size_t>({(size_t)nq, (256u << 20) / (n * sizeof(T)), (size_t)65535}));
    if (B < nq && B > 64) B -= B % 64;
    const int nch = radius_chunks((int)n);
    if (!dD.ensure((size_t)B * n * sizeof(T)) ||
        !dRc.ensure(radius_scan_work_bytes((int)B, (int)n) + 64) ||
        !dRs.ensure((size_t)B * nch * sizeof(long long)) ||
        !dRh.ensure((size_t)B * nch * sizeof(int)))
        return err->error(da_status_memory_error, "Device memory allocation failed.");
    // testing hook: the offsets' waits run out (AOCLDA_B200_TEST_RADIUS_WAIT=1)
    const char *tw = std::getenv("AOCLDA_B200_TEST_RADIUS_WAIT");
    const int test_wait = (tw && tw[0] == '1') ? 1 : 0;
    std::vector<long long> start((size_t)B * nch + 2);
    // the distance kernel also counts each (row, chunk) piece's hits
    PairwiseArgs pa{acc, post, kc, (double)p, false, true};
    pa.thr = (double)thr;
    pa.hits = dRh.as<int>();
    long long *d_total = reinterpret_cast<long long *>(dRc.as<char>() +
                                                       radius_scan_work_bytes((int)B, (int)n));
    int *d_err = reinterpret_cast<int *>(d_total + 1);
    for (da_int q0 = 0; q0 < nq; q0 += B) {
        const int b = (int)std::min<da_int>(B, nq - q0);
        B200_TRY(cudaMemsetAsync(dRh.p, 0, (size_t)b * nch * sizeof(int), st), "memset");
        B200_TRY(cuda->timed("radius_distances", [&] {
            return launch_pairwise<T>(dQ.as<T>() + (size_t)q0 * ld, ld, b, dX.as<T>(), ld, (int)n,
                                      (int)d, qn ? qn + q0 : nullptr, xn, pa, dD.as<T>(), st);
        }), "distance kernel");
        // counts and offsets in (row, chunk) order on the device: every row's
        // hits stay in index order
        B200_TRY(cuda->timed("radius_count", [&] {
            return launch_radius_count_scan<T>(dD.as<T>(), b, (int)n, n, thr, dRc.p,
                                               dRs.as<long long>(), d_total, d_err, test_wait, st,
                                               dRh.as<int>());
        }), "count");
        B200_TRY(cudaMemcpyAsync(start.data(), dRs.p, (size_t)b * nch * sizeof(long long),
                                 cudaMemcpyDeviceToHost, st), "copy");
        B200_TRY(cudaMemcpyAsync(start.data() + (size_t)b * nch, d_total, 2 * sizeof(long long),
                                 cudaMemcpyDeviceToHost, st), "copy");
        B200_TRY(cudaStreamSynchronize(st), "radius search");
        int scan_err = 0;
        std::memcpy(&scan_err, start.data() + (size_t)b * nch + 1, sizeof(int));
        if (scan_err != 0)
            return err->error(da_status_internal_error,
                              "The radius search's offset scan timed out waiting for another "
                              "block of the GPU.");
        const long long tot = start[(size_t)b * nch];
        const size_t base = idx_out.size();
        for (int i = 0; i < b; ++i) {
            const long long s0 = start[(size_t)i * nch];
            const long long s1 = i + 1 < b ? start[(size_t)(i + 1) * nch] : tot;
            start_out[(size_t)q0 + i] = (long long)base + s0;
            cnt_out[(size_t)q0 + i] = (da_int)(s1 - s0);
        }
        if (tot == 0) continue;
        if (!dRi.ensure((size_t)tot * sizeof(int)) || !dRv.ensure((size_t)tot * sizeof(T)))
            return err->error(da_status_memory_error, "Device memory allocation failed.");
        B200_TRY(cuda->timed("radius_emit", [&] {
            return launch_radius_emit<T>(dD.as<T>(), b, (int)n, n, thr, dRs.as<long long>(),
                                         dRi.as<int>(), dRv.as<T>(), st);
        }), "compaction");
        idx_out.resize(base + (size_t)tot);
        if (want_val) val_out.resize(base + (size_t)tot);
        std::vector<int> ii((size_t)tot);
        B200_TRY(cudaMemcpyAsync(ii.data(), dRi.p, (size_t)tot * sizeof(int),
                                 cudaMemcpyDeviceToHost, st), "copy");
        if (want_val)
            B200_TRY(cudaMemcpyAsync(val_out.data() + base, dRv.p, (size_t)tot * sizeof(T),
                                     cudaMemcpyDeviceToHost, st), "copy");
        B200_TRY(cudaStreamSynchronize(st), "radius search");
        for (size_t i = 0; i < (size_t)tot; ++i) idx_out[base + i] = (da_int)ii[i];
    }
    return da_status_success;
}

// nearest_neighbors.cpp:940-1015
// Radius neighbours, brute force (nearest_neighbors.cpp:1915-2068 and the
// brute-force search :2070-2247): the distance block of the kNN path's
// metric plan (squared for euclidean, compared with radius^2), the rows
// within the radius in index order per query, then (sort_results) a stable
// sort by distance as sorted_n_dist_n_ind (nearest_neighbors_utils.hpp:73-101).
template <typename T>
da_status NN<T>::radius_neighbors(da_int nq, da_int d, const T *Xt, da_int ldt, T r,
                                  da_int return_distance, da_int sort_results) {
    if (!return_distance && sort_results)
        return err->error(da_status_invalid_input,
                          "Cannot sort results if distances are not returned.");
    if (!have_X)
        return err->error(da_status_no_data,
                          "No training data have been set. Please call da_nn_set_data_s or "
                          "da_nn_set_data_d.");
    da_status s = check_options_update();
    if (s != da_status_success) return s;
    if (metric == M_IP)
        return err->error(da_status_incompatible_options,
                          "The inner product metric is not compatible with radius neighbors. "
                          "Use da_nn_kneighbors to find the k most similar training vectors by "
                          "inner product.");
    s = validate_queries(nq, d, Xt, ldt);
    if (s != da_status_success) return s;
    if (r < T(0)) r = (T)opts.r("radius");
    model_trained = false;
    s = radius_compute(nq, d, Xt, ldt, r, return_distance || sort_results, rnn_count, rnn_start,
                       rnn_idx, rnn_val, rnn_squares);
    if (s != da_status_success) return s;
    rnn_dist = return_distance != 0;
    if (sort_results) {
        std::vector<da_int> perm, ti;
        std::vector<T> tv;
        for (da_int q = 0; q < nq; ++q) {
            const size_t o = (size_t)rnn_start[q], m = (size_t)rnn_count[q];
            perm.resize(m);
            for (size_t i = 0; i < m; ++i) perm[i] = (da_int)i;
            std::stable_sort(perm.begin(), perm.end(), [&](da_int a, da_int b) {
                return rnn_val[o + a] < rnn_val[o + b];
            });
            ti.assign(rnn_idx.begin() + o, rnn_idx.begin() + o + m);
            tv.assign(rnn_val.begin() + o, rnn_val.begin() + o + m);
            for (size_t i = 0; i < m; ++i) {
                rnn_idx[o + i] = ti[perm[i]];
                rnn_val[o + i] = tv[perm[i]];
            }
        }
    }
    model_trained = true;
    return da_status_success;
}

// Result queries of the radius search (nearest_neighbors.cpp:118-260).
template <typename T> da_status NN<T>::radius_values(da_result q, da_int *dim, T *out) {
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "Radius neighbors have not been computed. Please call "
                         "da_nn_radius_neighbors_s or da_nn_radius_neighbors_d first.");
    if (q != da_nn_radius_neighbors_distances && q != da_nn_radius_neighbors_distances_index)
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    if (!rnn_dist)
        return err->warn(da_status_no_data,
                         "Distances were not requested during radius neighbors computation. "
                         "Please set return_distance to true in da_nn_radius_neighbors_s or "
                         "da_nn_radius_neighbors_d call.");
    const da_int nq = (da_int)rnn_count.size();
    auto put = [&](da_int qi, T *dst) {
        const size_t o = (size_t)rnn_start[qi];
        for (da_int i = 0; i < rnn_count[qi]; ++i)
            dst[i] = rnn_squares ? std::sqrt(rnn_val[o + i]) : rnn_val[o + i];
    };
    if (q == da_nn_radius_neighbors_distances_index) {
        const da_int qi = (da_int)out[0];
        if (qi < 0 || qi >= nq)
            return err->warn(da_status_invalid_input,
                             "The provided index is out of bounds. It should be in the range [0, " +
                                 std::to_string(nq - 1) + "].");
        if (rnn_count[qi] > *dim) {
            *dim = rnn_count[qi];
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: " +
                                 std::to_string(rnn_count[qi]) + ".");
        }
        put(qi, out);
        return da_status_success;
    }
    const da_int total = (da_int)rnn_val.size();
    if (total > *dim) {
        *dim = total;
        return err->warn(da_status_invalid_array_dimension,
                         "The array is too small. Please provide an array of at least size: " +
                             std::to_string(total) + ".");
    }
    da_int a = 0;
    for (da_int qi = 0; qi < nq; ++qi) {
        put(qi, out + a);
        a += rnn_count[qi];
    }
    return da_status_success;
}
template <typename T> da_status NN<T>::get_result(da_result q, da_int *dim, double *out) {
    if constexpr (std::is_same_v<T, double>) return radius_values(q, dim, out);
    (void)q, (void)dim, (void)out;
    return err->error(da_status_wrong_type, "Wrong precision type.");
}
template <typename T> da_status NN<T>::get_result(da_result q, da_int *dim, float *out) {
    if constexpr (std::is_same_v<T, float>) return radius_values(q, dim, out);
    (void)q, (void)dim, (void)out;
    return err->error(da_status_wrong_type, "Wrong precision type.");
}
template <typename T> da_status NN<T>::get_result_int(da_result q, da_int *dim, da_int *out) {
    if (q == da_trained) return AlgBase::get_result_int(q, dim, out);
    if (!model_trained)
        return err->warn(da_status_no_data,
                         "Radius neighbors have not been computed. Please call "
                         "da_nn_radius_neighbors first.");
    const da_int nq = (da_int)rnn_count.size();
    const da_int total = (da_int)rnn_idx.size();
    switch (q) {
    case da_nn_radius_neighbors_count:
    case da_nn_radius_neighbors_offsets: {
        if (nq + 1 > *dim) {
            *dim = nq + 1;
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: " +
                                 std::to_string(nq + 1) + ".");
        }
        da_int off = 0;
        for (da_int i = 0; i < nq; ++i) {
            if (q == da_nn_radius_neighbors_count) out[i] = rnn_count[i];
            else out[i] = rnn_count[i] > 0 ? off : -1;
            off += rnn_count[i];
        }
        out[nq] = off;
        return da_status_success;
    }
    case da_nn_radius_neighbors_indices_index: {
        const da_int qi = out[0];
        if (qi < 0 || qi >= nq)
            return err->warn(da_status_invalid_input,
                             "The provided index is out of bounds. It should be in the range [0, " +
                                 std::to_string(nq - 1) + "].");
        if (rnn_count[qi] > *dim) {
            *dim = rnn_count[qi];
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: " +
                                 std::to_string(rnn_count[qi]) + ".");
        }
        for (da_int i = 0; i < rnn_count[qi]; ++i) out[i] = rnn_idx[(size_t)rnn_start[qi] + i];
        return da_status_success;
    }
    case da_nn_radius_neighbors_indices: {
        if (total > *dim) {
            *dim = total;
            return err->warn(da_status_invalid_array_dimension,
                             "The array is too small. Please provide an array of at least size: " +
                                 std::to_string(total) + ".");
        }
        da_int a = 0;
        for (da_int qi = 0; qi < nq; ++qi)
            for (da_int i = 0; i < rnn_count[qi]; ++i) out[a++] = rnn_idx[(size_t)rnn_start[qi] + i];
        return da_status_success;
    }
    default:
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    }
}

template <typename T>
da_status NN<T>::kneighbors(da_int nq, da_int d, const T *Xt, da_int ldt, da_int *n_ind,
                            T *n_dist, da_int k, da_int return_distance) {
    if (!have_X)
        return err->error(da_status_no_data,
                          "No training data have been set. Please call da_nn_set_data_s or "
                          "da_nn_set_data_d.");
    da_status s = check_options_update();
    if (s != da_status_success) return s;
    if (n_ind == nullptr) return err->error(da_status_invalid_pointer, "n_ind is not a valid pointer.");
    s = validate_queries(nq, d, Xt, ldt);
    if (s != da_status_success) return s;
    if (k <= 0 && n_neighbors <= 0)
        return err->error(da_status_invalid_input, "Number of requested neighbors must be positive.");
    if (k <= 0) k = n_neighbors;
    if (k > n_samples)
        return err->error(da_status_invalid_input,
                          "Number of requested neighbors must be at least as big as the number "
                          "of samples.");
    if (return_distance && n_dist == nullptr)
        return err->error(da_status_invalid_pointer, "n_dist is not a valid pointer.");
    std::vector<da_int> ind;
    std::vector<T> dist;
    s = kneighbors_compute(nq, d, Xt, ldt, order(), k, ind, return_distance ? &dist : nullptr);
    if (s != da_status_success) return s;
    // outputs: q-major for row-major storage, n_queries x k column-major otherwise
    const bool cm = order() == column_major;
    for (da_int q = 0; q < nq; ++q)
        for (da_int r = 0; r < k; ++r) {
            const size_t src = (size_t)q * k + r;
            const size_t dst = cm ? (size_t)r * nq + q : src;
            n_ind[dst] = ind[src];
            if (return_distance) n_dist[dst] = dist[src];
        }
    return da_status_success;
}

template <typename T> da_status NN<T>::available_classes() {
    if (!have_X)
        return err->error(da_status_no_data,
                          "No training data have been set. Please call da_nn_set_data_s or "
                          "da_nn_set_data_d.");
    if (!have_labels)
        return err->error(da_status_no_data,
                          "No classification labels have been set. Please call "
                          "da_nn_set_labels_s or da_nn_set_labels_d.");
    std::set<da_int> s(y_class, y_class + n_samples);
    classes.assign(s.begin(), s.end());
    classes_done = true;
    return da_status_success;
}

template <typename T> da_status NN<T>::classes_api(da_int *n_classes, da_int *cls) {
    if (n_classes == nullptr)
        return err->error(da_status_invalid_pointer, "n_classes is not a valid pointer.");
    if (!classes_done) {
        da_status s = available_classes();
        if (s != da_status_success) return s;
    }
    const da_int nc = (da_int)classes.size();
    if (*n_classes <= 0 || cls == nullptr) {
        *n_classes = nc;
        return da_status_success;
    }
    if (*n_classes < nc) {
        *n_classes = nc;
        return err->error(da_status_invalid_array_dimension,
                          "The classes array is too small, it must be at least " +
                              std::to_string(nc) + ".");
    }
    for (da_int i = 0; i < nc; ++i) cls[i] = classes[i];
    *n_classes = nc;
    return da_status_success;
}

// Vote of predict_proba_compute_knn (nearest_neighbors.cpp:1166-1272):
// proba is q-major (q * n_classes + c).
template <typename T>
da_status NN<T>::compute_proba(da_int nq, da_int d, const T *Xt, da_int ldt,
                               std::vector<T> &proba) {
    if (metric == M_IP && weights == 1)
        return err->error(da_status_incompatible_options,
                          "The inner product metric is not compatible with "
                          "weights=\"distance\". Use weights=\"uniform\" instead.");
    if (!classes_done) {
        da_status s = available_classes();
        if (s != da_status_success) return s;
    }
    const da_int k = n_neighbors;
    if (k > n_samples)
        return err->error(da_status_invalid_input,
                          "Number of requested neighbors must be at least as big as the number "
                          "of samples.");
    std::vector<da_int> ind;
    std::vector<T> dist;
    da_status s = kneighbors_compute(nq, d, Xt, ldt, order(), k, ind, weights == 1 ? &dist : nullptr);
    if (s != da_status_success) return s;
    const da_int nc = (da_int)classes.size();
    proba.assign((size_t)nq * nc, T(0));
    for (da_int q = 0; q < nq; ++q) {
        T den = T(0);
        for (da_int c = 0; c < nc; ++c) {
            T v = T(0);
            for (da_int r = 0; r < k; ++r) {
                const da_int lbl = y_class[ind[(size_t)q * k + r]];
                if (lbl != classes[c]) continue;
                if (weights == 0) v += T(1);
                else {
                    const T w = dist[(size_t)q * k + r];
                    v += (w <= std::numeric_limits<T>::epsilon()) ? T(1) : T(1) / w;
                }
            }
            proba[(size_t)q * nc + c] = v;
            den += v;
        }
        for (da_int c = 0; c < nc; ++c) proba[(size_t)q * nc + c] /= den;
    }
    return da_status_success;
}

// Radius-mode vote (predict_proba_compute_rnn, nearest_neighbors.cpp:1280-1479):
// the rows within the "radius" option of each query vote for their labels,
// with weight 1 (uniform) or 1 / distance (distance; 1 at distance <= eps).
// A query with no row within the radius is an error under outlier handling
// "none"; "manual" gives it probability 1 for the "outlier label" (all zero
// and a warning when that label is not a training label), "most frequent"
// probability 1 for the most frequent training label.  proba is q-major.
template <typename T>
da_status NN<T>::compute_proba_rnn(da_int nq, da_int d, const T *Xt, da_int ldt,
                                   std::vector<T> &proba) {
    if (metric == M_IP && weights == 1)
        return err->error(da_status_incompatible_options,
                          "The inner product metric is not compatible with "
                          "weights=\"distance\". Use weights=\"uniform\" instead.");
    if (!classes_done) {
        da_status s = available_classes();
        if (s != da_status_success) return s;
    }
    const da_int oh = opts.key("outlier handling");
    const da_int nc = (da_int)classes.size();
    const da_int mf = oh == OH_MOST_FREQUENT ? most_frequent_label() : 0;
    da_int manual_idx = -1;
    if (oh == OH_MANUAL) {
        auto it = std::lower_bound(classes.begin(), classes.end(), (da_int)opts.i("outlier label"));
        if (it != classes.end() && *it == (da_int)opts.i("outlier label"))
            manual_idx = (da_int)(it - classes.begin());
    }
    std::vector<da_int> cnt, idx;
    std::vector<long long> start;
    std::vector<T> val;
    bool squares = false;
    da_status s = radius_compute(nq, d, Xt, ldt, (T)opts.r("radius"), weights == 1, cnt, start,
                                 idx, val, squares);
    if (s != da_status_success) return s;
    proba.assign((size_t)nq * nc, T(0));
    bool outliers = false;
    for (da_int q = 0; q < nq; ++q) {
        T *pq = proba.data() + (size_t)q * nc;
        const size_t o = (size_t)start[q], m = (size_t)cnt[q];
        if (m == 0) {
            if (oh == OH_NONE)
                return err->error(da_status_operation_failed,
                                  "Failed to compute probabilities for query " + std::to_string(q) +
                                      " since it does not have any neighbors within the "
                                      "specified radius.");
            if (oh == OH_MANUAL) {
                outliers = true;
                if (manual_idx != -1) pq[manual_idx] = T(1);
            } else {
                for (da_int c = 0; c < nc; ++c) pq[c] = classes[c] == mf ? T(1) : T(0);
            }
            continue;
        }
        // per class, the neighbours' weights in neighbour order
        for (size_t i = 0; i < m; ++i) {
            const da_int c = (da_int)(std::lower_bound(classes.begin(), classes.end(),
                                                       y_class[idx[o + i]]) - classes.begin());
            pq[c] += weights == 0 ? T(1) : radius_weight(val[o + i], squares);
        }
        T den = T(0);
        for (da_int c = 0; c < nc; ++c) den += pq[c];
        for (da_int c = 0; c < nc; ++c) pq[c] /= den;
    }
    if (oh == OH_MANUAL && outliers && manual_idx == -1)
        return err->warn(da_status_outlier_warning,
                         "The manually set outlier label is not present in the training labels. "
                         "Setting probabilities to 0.0.");
    return da_status_success;
}

// most_frequent_element (nearest_neighbors.cpp:1037-1058): the most frequent
// training label, the smallest of equally frequent ones.
template <typename T> da_int NN<T>::most_frequent_label() {
    std::map<da_int, da_int> freq;
    for (da_int i = 0; i < n_samples; ++i) freq[y_class[i]]++;
    da_int best = y_class[0], top = 0;
    for (const auto &f : freq)
        if (f.second > top) {
            top = f.second;
            best = f.first;
        }
    return best;
}

// get_weights (nearest_neighbors.cpp:1021-1033) of one radius neighbour; the
// stored value is squared for euclidean.
template <typename T> T NN<T>::radius_weight(T v, bool squares) {
    const T w = squares ? std::sqrt(v) : v;
    return w <= std::numeric_limits<T>::epsilon() ? T(1) : T(1) / w;
}

template <typename T>
da_status NN<T>::predict_proba(da_int nq, da_int d, const T *Xt, da_int ldt, T *proba,
                               da_nn_search_mode mode) {
    if (!have_X)
        return err->error(da_status_no_data,
                          "No training data have been set. Please call da_nn_set_data_s or "
                          "da_nn_set_data_d.");
    if (!have_labels)
        return err->error(da_status_no_data,
                          "No classification labels have been set. Please call "
                          "da_nn_set_labels_s or da_nn_set_labels_d.");
    da_status s = check_options_update();
    if (s != da_status_success) return s;
    if (proba == nullptr) return err->error(da_status_invalid_pointer, "proba is not a valid pointer.");
    if (nq < 1)
        return err->error(da_status_invalid_array_dimension,
                          "Number of queries must be greater than zero.");
    if (d < 1)
        return err->error(da_status_invalid_array_dimension,
                          "Number of features must be greater than zero.");
    s = validate_queries(nq, d, Xt, ldt);
    if (s != da_status_success) return s;
    if (mode != knn_search_mode && mode != radius_search_mode)
        return err->error(da_status_invalid_input,
                          "Unknown search mode: " + std::to_string((int)mode) + ".");
    std::vector<T> pr;
    s = mode == knn_search_mode ? compute_proba(nq, d, Xt, ldt, pr)
                                : compute_proba_rnn(nq, d, Xt, ldt, pr);
    if (s != da_status_success && s != da_status_outlier_warning) return s;
    const da_int nc = (da_int)classes.size();
    const bool cm = order() == column_major;
    for (da_int q = 0; q < nq; ++q)
        for (da_int c = 0; c < nc; ++c)
            proba[cm ? (size_t)c * nq + q : (size_t)q * nc + c] = pr[(size_t)q * nc + c];
    return s;
}

template <typename T>
da_status NN<T>::predict(da_int nq, da_int d, const T *Xt, da_int ldt, da_int *y,
                         da_nn_search_mode mode) {
    da_status s = check_options_update();
    if (s != da_status_success) return s;
    if (!have_X)
        return err->error(da_status_no_data,
                          "No training data have been set. Please call da_nn_set_data_s or "
                          "da_nn_set_data_d.");
    if (!have_labels)
        return err->error(da_status_no_data,
                          "No classification labels have been set. Please call "
                          "da_nn_set_labels_s or da_nn_set_labels_d.");
    if (y == nullptr) return err->error(da_status_invalid_pointer, "y_test is not a valid pointer.");
    if (nq < 1)
        return err->error(da_status_invalid_array_dimension, "n_queries must be greater than 0.");
    s = validate_queries(nq, d, Xt, ldt);
    if (s != da_status_success) return s;
    if (mode != knn_search_mode && mode != radius_search_mode)
        return err->error(da_status_invalid_input,
                          "Unknown search mode: " + std::to_string((int)mode) + ".");
    std::vector<T> pr;
    s = mode == knn_search_mode ? compute_proba(nq, d, Xt, ldt, pr)
                                : compute_proba_rnn(nq, d, Xt, ldt, pr);
    if (s != da_status_success && s != da_status_outlier_warning) return s;
    const da_int nc = (da_int)classes.size();
    // radius mode with outlier handling: an all-zero row (a query without
    // neighbours) takes the outlier label or the most frequent label
    // (nearest_neighbors.cpp:1566-1599)
    const da_int oh = mode == knn_search_mode ? OH_NONE : opts.key("outlier handling");
    const da_int fill = oh == OH_MANUAL ? (da_int)opts.i("outlier label")
                        : oh == OH_MOST_FREQUENT ? most_frequent_label() : 0;
    for (da_int q = 0; q < nq; ++q) {
        // first maximum (cblas_iamax semantics, nearest_neighbors.cpp:1566-1573)
        da_int best = 0;
        T bv = std::fabs(pr[(size_t)q * nc]);
        for (da_int c = 1; c < nc; ++c) {
            const T v = std::fabs(pr[(size_t)q * nc + c]);
            if (v > bv) {
                bv = v;
                best = c;
            }
        }
        y[q] = (oh != OH_NONE && pr[(size_t)q * nc + best] == T(0)) ? fill : classes[best];
    }
    return s;
}

template <typename T>
da_status NN<T>::predict_reg(da_int nq, da_int d, const T *Xt, da_int ldt, T *y,
                             da_nn_search_mode mode) {
    if (!have_X)
        return err->error(da_status_no_data,
                          "No training data have been set. Please call da_nn_set_data_s or "
                          "da_nn_set_data_d.");
    if (!have_targets)
        return err->error(da_status_no_data,
                          "No regression targets have been set. Please call "
                          "da_nn_set_targets_s or da_nn_set_targets_d.");
    da_status s = check_options_update();
    if (s != da_status_success) return s;
    if (y == nullptr) return err->error(da_status_invalid_pointer, "y_test is not a valid pointer.");
    if (nq < 1)
        return err->error(da_status_invalid_array_dimension, "n_queries must be greater than 0.");
    s = validate_queries(nq, d, Xt, ldt);
    if (s != da_status_success) return s;
    if (mode != knn_search_mode && mode != radius_search_mode)
        return err->error(da_status_invalid_input,
                          "Unknown search mode: " + std::to_string((int)mode) + ".");
    if (metric == M_IP && weights == 1)
        return err->error(da_status_incompatible_options,
                          "The inner product metric is not compatible with "
                          "weights=\"distance\". Use weights=\"uniform\" instead.");
    if (mode == radius_search_mode) return predict_reg_rnn(nq, d, Xt, ldt, y);
    const da_int k = n_neighbors;
    if (k > n_samples)
        return err->error(da_status_invalid_input,
                          "Number of requested neighbors must be at least as big as the number "
                          "of samples.");
    std::vector<da_int> ind;
    std::vector<T> dist;
    s = kneighbors_compute(nq, d, Xt, ldt, order(), k, ind, weights == 1 ? &dist : nullptr);
    if (s != da_status_success) return s;
    // nearest_neighbors.cpp:1707-1747
    for (da_int q = 0; q < nq; ++q) {
        if (weights == 0) {
            T sum = T(0);
            for (da_int r = 0; r < k; ++r) sum += y_reg[ind[(size_t)q * k + r]];
            y[q] = sum / T(k);
        } else {
            T num = T(0), den = T(0);
            for (da_int r = 0; r < k; ++r) {
                const T dv = dist[(size_t)q * k + r];
                const T w = (dv <= std::numeric_limits<T>::epsilon()) ? T(1) : T(1) / dv;
                num += y_reg[ind[(size_t)q * k + r]] * w;
                den += w;
            }
            y[q] = num / den;
        }
    }
    return da_status_success;
}

// Radius-mode regression (predict_targets_rnn, nearest_neighbors.cpp:1763-1909):
// the mean target of the rows within the radius (uniform) or their
// 1 / distance weighted mean (distance).  A query without neighbours is an
// error under outlier handling "none"; it takes the mean training target
// under "most frequent" and the "outlier target" (with a warning) under
// "manual".
template <typename T>
da_status NN<T>::predict_reg_rnn(da_int nq, da_int d, const T *Xt, da_int ldt, T *y) {
    const da_int oh = opts.key("outlier handling");
    T mean_target = T(0);
    if (oh == OH_MOST_FREQUENT) {
        for (da_int i = 0; i < n_samples; ++i) mean_target += y_reg[i];
        mean_target /= T(n_samples);
    }
    const T manual_target = (T)opts.r("outlier target");
    std::vector<da_int> cnt, idx;
    std::vector<long long> start;
    std::vector<T> val;
    bool squares = false;
    da_status s = radius_compute(nq, d, Xt, ldt, (T)opts.r("radius"), weights == 1, cnt, start,
                                 idx, val, squares);
    if (s != da_status_success) return s;
    bool outliers = false;
    for (da_int q = 0; q < nq; ++q) {
        const size_t o = (size_t)start[q], m = (size_t)cnt[q];
        if (m == 0) {
            if (oh == OH_NONE)
                return err->error(da_status_operation_failed,
                                  std::string(weights == 0 ? "Failed to compute targets for query "
                                                           : "Failed to predict targets for query ") +
                                      std::to_string(q) +
                                      " since it does not have any neighbors within the "
                                      "specified radius.");
            if (oh == OH_MOST_FREQUENT) {
                y[q] = mean_target;
            } else {
                outliers = true;
                y[q] = manual_target;
            }
            continue;
        }
        if (weights == 0) {
            T sum = T(0);
            for (size_t i = 0; i < m; ++i) sum += y_reg[idx[o + i]];
            y[q] = sum / T(m);
        } else {
            T num = T(0), den = T(0);
            for (size_t i = 0; i < m; ++i) {
                const T w = radius_weight(val[o + i], squares);
                num += y_reg[idx[o + i]] * w;
                den += w;
            }
            y[q] = num / den;
        }
    }
    if (oh == OH_MANUAL && outliers)
        return err->warn(da_status_outlier_warning,
                         "One or more samples have no neighbors within the specified radius. "
                         "Setting the corresponding targets to " + std::to_string(manual_target) +
                             ".");
    return da_status_success;
}

template struct NN<float>;
template struct NN<double>;

} // namespace b200
