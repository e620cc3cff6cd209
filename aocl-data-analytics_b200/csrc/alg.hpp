// Algorithm handles behind the C ABI: the kNN handle and the k-means handle,
// both templated on the working precision (float / double) like the
// reference's basic_handle<T> family (source/core/utilities/basic_handle.hpp).
#pragma once
#include "b200_kernels.hpp"
#include "host_common.hpp"
#include <memory>
#include <random>
#include <set>

namespace b200 {

struct AlgBase {
    Registry opts;
    ErrorRecord *err = nullptr;
    CudaCtx *cuda = nullptr;
    bool model_trained = false;
    virtual ~AlgBase() = default;
    virtual void refresh() {}
    virtual da_status get_result(da_result q, da_int *dim, double *out) {
        (void)q, (void)dim, (void)out;
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    }
    virtual da_status get_result(da_result q, da_int *dim, float *out) {
        (void)q, (void)dim, (void)out;
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    }
    virtual da_status get_result_int(da_result q, da_int *dim, da_int *out) {
        if (q == da_trained) {
            if (*dim < 1) {
                *dim = 1;
                return err->warn(da_status_invalid_array_dimension,
                                 "Size of the result array is too small, provide an array of "
                                 "at least size: 1.");
            }
            out[0] = da_int(model_trained);
            return da_status_success;
        }
        return err->warn(da_status_unknown_query, "The requested result could not be found.");
    }
    da_order order() { return da_order(opts.key("storage order")); }
    // model persistence: the algorithm's state after its options
    virtual da_status save_state(ByteWriter &w) {
        (void)w;
        return err->error(da_status_not_implemented, "This handle cannot be saved.");
    }
    virtual da_status load_state(ByteReader &r) {
        (void)r;
        return err->error(da_status_not_implemented, "This handle cannot be loaded.");
    }
};

// ------------------------------------------------------------------ kNN ----
// Reference: source/core/nearest_neighbors/nearest_neighbors.{hpp,cpp}
template <typename T> struct NN : public AlgBase {
    // option-derived state (nearest_neighbors.cpp:295-352)
    da_int n_neighbors = 5, algo = 3, metric = 0, weights = 0;
    T p = 2;
    bool up_to_date = false;
    da_int locked_algo = -1, locked_metric = -1, locked_leaf = -1;
    T locked_p = 0;
    // data
    da_int n_samples = 0, n_features = 0;
    const T *X_host = nullptr;
    da_int ldx_host = 0;
    da_order data_order = column_major;
    bool have_X = false, X_on_device = false;
    const da_int *y_class = nullptr;
    const T *y_reg = nullptr;
    bool have_labels = false, have_targets = false;
    std::vector<da_int> classes;
    bool classes_done = false;
    // device
    int ld = 0;
    DevBuf dX, dXn, dQ, dQn, dPartK, dPartI, dOutK, dOutI, dStage;
    int xn_kind = -1; // which norms dXn holds: 0 squared, 1 eps1-norm
    // tensor-core candidate pass (fp32 euclidean, cosine): bf16 hi/lo copies
    // of the training rows, their fp32 |x|^2 and max |x|, 1 / |x| (cosine);
    // per-call query buffers
    DevBuf dXh, dXl, dXsq, dTkScal, dTkQ, dTkList, dTkFlag, dXinv;
    bool tc_train_ready = false;
    int tc_ldbf = 0;

    NN(ErrorRecord *e, CudaCtx *c, bool single);
    da_status set_params();
    da_status check_options_update();
    da_status set_data(da_int n, da_int d, const T *X, da_int ldx);
    da_status set_labels(da_int n, const da_int *y);
    da_status set_targets(da_int n, const T *y);
    // training data of another handle, with its device copies shared
    da_status share_data(NN<T> &src);
    da_status kneighbors(da_int nq, da_int d, const T *Xt, da_int ldt, da_int *n_ind, T *n_dist,
                         da_int k, da_int return_distance);
    da_status classes_api(da_int *n_classes, da_int *cls);
    da_status predict_proba(da_int nq, da_int d, const T *Xt, da_int ldt, T *proba,
                            da_nn_search_mode mode);
    da_status predict(da_int nq, da_int d, const T *Xt, da_int ldt, da_int *y,
                      da_nn_search_mode mode);
    da_status predict_reg(da_int nq, da_int d, const T *Xt, da_int ldt, T *y,
                          da_nn_search_mode mode);
    void refresh() override { up_to_date = false; }
    // model persistence: the training rows (and labels / targets) are copied
    // into the file; a loaded handle owns them (X_own, y_own, t_own)
    std::vector<T> X_own, t_own;
    std::vector<da_int> y_own;
    // radius search (nearest_neighbors.cpp:1915-2068, 2070-2247): per query
    // its count and start in the flat index / value arrays; values as
    // computed (squared for euclidean), the square root taken on extraction
    std::vector<da_int> rnn_count, rnn_idx;
    std::vector<long long> rnn_start;
    std::vector<T> rnn_val;
    bool rnn_dist = false, rnn_squares = false;
    DevBuf dD, dRc, dRs, dRi, dRv, dRh;
    da_status radius_neighbors(da_int nq, da_int d, const T *Xt, da_int ldt, T radius,
                               da_int return_distance, da_int sort_results);
    da_status get_result(da_result q, da_int *dim, double *out) override;
    da_status get_result(da_result q, da_int *dim, float *out) override;
    da_status get_result_int(da_result q, da_int *dim, da_int *out) override;
    da_status radius_values(da_result q, da_int *dim, T *out);
    da_status save_state(ByteWriter &w) override;
    da_status load_state(ByteReader &r) override;

    // core: q-major results (n_ind[q*k + r]) on the host
    da_status kneighbors_compute(da_int nq, da_int d, const T *Xt, da_int ldt, da_order ord,
                                 da_int k, std::vector<da_int> &ind, std::vector<T> *dist);
    da_status ensure_device_data();
    da_status validate_queries(da_int nq, da_int d, const T *Xt, da_int ldt);
    // tensor-core path; `done` false when the plain path must run instead
    da_status kneighbors_tc(da_int nq, da_int d, da_int k, int kc, bool take_sqrt, bool cosine,
                            bool &done);
    da_status compute_proba(da_int nq, da_int d, const T *Xt, da_int ldt, std::vector<T> &proba);
    // radius mode of predict / predict_proba (outlier handling as the reference)
    da_status radius_compute(da_int nq, da_int d, const T *Xt, da_int ldt, T r, bool want_val,
                             std::vector<da_int> &cnt, std::vector<long long> &start,
                             std::vector<da_int> &idx, std::vector<T> &val, bool &squares);
    da_status compute_proba_rnn(da_int nq, da_int d, const T *Xt, da_int ldt,
                                std::vector<T> &proba);
    da_status predict_reg_rnn(da_int nq, da_int d, const T *Xt, da_int ldt, T *y);
    da_int most_frequent_label();
    static T radius_weight(T v, bool squares);
    da_status available_classes();
};

// --------------------------------------------------------------- k-means ---
// Reference: source/core/clustering/kmeans/kmeans.{hpp,cpp}, kmeans_lloyd.hpp
template <typename T> struct KMeans : public AlgBase {
    da_int n_samples = 0, n_features = 0;
    const T *A_host = nullptr;
    da_int lda_host = 0;
    da_order data_order = column_major;
    bool initdone = false, centres_supplied = false;
    std::vector<T> C_supplied; // column-major n_clusters x d
    // options read at compute
    da_int n_clusters = 1, n_init = 10, max_iter = 300, seed = 0, init_method = 1;
    da_int algorithm = 0, empty_mode = 0, afk_samples = 50;
    double tol = 1e-4;
    std::mt19937_64 mt_gen;
    // results
    std::vector<T> best_centres; // column-major k x d
    std::vector<da_int> best_labels;
    bool best_labels_on_host = false;
    double best_inertia = 0;
    da_int best_n_iter = 0, best_lp_n_iter = 0;
    bool warn_maxit = false;
    // device
    int ld = 0;
    DevBuf dX, dXn, dC0, dC1, dCn, dL0, dL1, dCounts, dBlockCounts, dOffsets, dSorted,
        dChunkSums, dSegStart, dScalars, dFlags, dPartials, dW, dKD, dCand, dStage, dY, dYL,
        dBestL, dXh, dXl, dXnrm, dBh, dBl, dBaug, dAaug, dCtmp, dTcScal, dAmb, dFxScale,
        dFxAcc, dFxTicket, dKppU, dKppBs, dChg;
    // changed-row list of the graph loop's assignments (incremental update)
    int chg_cap = 0;
    bool chg_capture = false;
    int tc_split = 0;     // bf16 terms of the resident X copies (0: none)
    bool use_tc = false; // bf16 tensor-core assignment active for this compute
    bool dXbf_stale = true;
    bool dx_loaded = false; // dX holds the current data set
    bool aaug_ready = false;
    bool fx_stale = true;  // fixed-point scales need recomputing (new data)
    bool fx_data_ok = false; // data finite (scales valid)
    bool use_fx = false;   // fixed-point centroid update active for this compute
    int fx_parity = 0;
    int ldbf = 0;
    da_int amb_last = 0;  // rows relabelled exactly in the last tensor-core pass
    // spherical (cosine) k-means (kmeans.cpp:396-405): the options of the
    // current compute, those the fitted model was computed with, the rows'
    // inverse norms (dXinv) and normalised rows (dXs) of the data set
    bool sph = false, sph_norm = true, model_sph = false, model_sph_norm = true;
    DevBuf dXinv, dXs;
    int sph_ready = 0; // bit 0: dXinv, bit 1: dXs hold the current data set
    const void *fx_src = nullptr; // rows the fixed-point scales were computed from
    T *h_pin = nullptr;
    void *h_small = nullptr; // pinned: flags + scalars
    // Lloyd iterations 1.. as one CUDA graph (a WHILE node whose body is one
    // iteration in place); rebuilt when a pointer or size it holds changes
    cudaGraph_t loop_graph = nullptr;
    cudaGraphExec_t loop_exec = nullptr;
    std::vector<uintptr_t> loop_key;
    DevBuf dLoop;

    KMeans(ErrorRecord *e, CudaCtx *c, bool single);
    // model persistence: the fitted centres, labels and run information
    da_status save_state(ByteWriter &w) override;
    da_status load_state(ByteReader &r) override;
    ~KMeans() override;
    void refresh() override;
    da_status set_data(da_int n, da_int d, const T *A, da_int lda);
    da_status set_init_centres(const T *C, da_int ldc);
    da_status compute();
    da_status read_options();
    da_status initial_centres(T *C, da_int ldc);
    da_status predict(da_int m, da_int d, const T *Y, da_int ldy, da_int *labels);
    da_status transform(da_int m, da_int d, const T *X, da_int ldx, T *Xt, da_int ldxt);
    da_status get_result_t(da_result q, da_int *dim, T *out);
    da_status get_result(da_result q, da_int *dim, double *out) override;
    da_status get_result(da_result q, da_int *dim, float *out) override;
    da_status get_result_int(da_result q, da_int *dim, da_int *out) override;

    // internals
    da_status ensure_device_data();
    da_status alloc_work();
    da_status init_centres(T *dC);
    da_status init_centres_raw(T *dC);
    da_status prepare_sph();
    // rows the centroid update sums: the normalised copy for spherical
    // k-means on normalised data, else the data set
    T *update_rows() { return (sph && sph_norm) ? dXs.as<T>() : dX.as<T>(); }
    da_status kmeans_plusplus(T *dC);
    da_status afk_mcmc(std::vector<T> &Cc);
    da_status run_lloyd(T *&dCcur, T *&dCprev, int *&dLcur, int *&dLprev, da_int &n_iter,
                        int &converged, double &inertia, bool &empty_found);
    da_status lloyd_step(const T *dCprev, T *dCnew, int *dL, const int *dLprev, bool update,
                         double *h_scal, int *h_flags);
    da_status split_empty(T *dC, int *dL, bool &split);
    da_status lloyd_graph(T *dC, int *dL, da_int &n_iter, int &converged, bool &ran);
    bool build_loop_graph(T *dC, int *dL);
    void drop_loop_graph();
    da_status prepare_tc();
    da_status prepare_fx();
    // Lloyd steps of a shard of a data set split across processes: the
    // current centres are dC0 / dC1 by shard_c, the current labels dL0 / dL1
    // by shard_l
    int shard_c = 0, shard_l = 0;
    bool shard_ready = false;
    da_status shard_colmax(float *colmax);
    da_status shard_begin(const float *colmax_global, da_int n_global, const float *C);
    da_status shard_partial(long long *acc);
    da_status shard_finalize(const long long *acc, double *scalars, da_int *flags);
    da_status shard_relabel(double *inertia, bool assign_first);
    da_status shard_result(float *centres, da_int *labels);
    da_status shard_tc_check();
    da_status assign(const T *dC, int *dL, const int *dLprev);
};

// ---------------------------------------------------- IVF-flat (approx) ---
// Reference: source/core/approximate_neighbors/approximate_neighbors.{hpp,cpp}
// The coarse quantiser is this library's k-means (Lloyd, random-samples
// initialisation, one run) on the GPU; the coarse probe and the assignment of
// added rows are GPU kNN searches over the centroids (squared GEMM-form
// distances); the inverted lists are one list-ordered device array scanned by
// launch_ivf_scan.
template <typename T> struct IVF : public AlgBase {
    // options read at train (approximate_neighbors.cpp:233-274)
    da_int n_list = 1, n_probe = 1, max_iter = 10, seed = 0, algo = 0, metric = 1;
    da_int internal_seed = 0, kmeans_iter = 0;
    T train_fraction = T(1);
    bool train_data_set = false, data_added = false;
    // training data (user memory)
    da_int n_samples = 0, n_features = 0, ldx_train = 0;
    const T *X_train = nullptr;
    da_order data_order = column_major;
    // the index: centroids (row-major n_list x d), per-list rows (row-major),
    // their squared norms and global indices, in insertion order
    std::vector<T> centroids;
    std::vector<std::vector<T>> list_rows, list_norms;
    std::vector<std::vector<da_int>> list_ids;
    std::vector<da_int> list_sizes;
    da_int n_index = 0;
    std::unique_ptr<NN<T>> coarse; // kNN over the centroids
    // device copy of the lists (rebuilt after every add)
    int ld = 0;
    bool lists_on_device = false;
    DevBuf dX, dXn, dGid, dOff, dQ, dQn, dProbe, dOutD, dOutI, dStage;

    IVF(ErrorRecord *e, CudaCtx *c, bool single);
    void refresh() override {}
    da_status check_options_update();
    da_status set_training_data(da_int n, da_int d, const T *X, da_int ldx);
    da_status train();
    da_status add(da_int n, da_int d, const T *X, da_int ldx);
    da_status train_and_add();
    da_status kneighbors(da_int nq, da_int d, const T *Xt, da_int ldt, da_int *n_ind, T *n_dist,
                         da_int k, da_int return_distance);
    da_status get_result(da_result q, da_int *dim, double *out) override;
    da_status get_result(da_result q, da_int *dim, float *out) override;
    da_status get_result_int(da_result q, da_int *dim, da_int *out) override;
    da_status result_values(da_result q, da_int *dim, T *out);
    da_status make_coarse();
    da_status upload_lists();
    // model persistence: the trained index (centroids, lists); the training
    // array is the user's and is not saved
    da_status save_state(ByteWriter &w) override;
    da_status load_state(ByteReader &r) override;
};

} // namespace b200

namespace b200 {
// Model files of AOCL-DA's own da_handle_save_model (ref_model.cpp): the
// test for its keyword, and a new handle of the file's type and precision
// (created by handle_init) holding its options and trained state.
bool is_reference_model(const char *p, size_t n);
da_status load_reference_model(const char *p, size_t n, da_handle *out,
                               da_status (*handle_init)(da_handle *, da_handle_type,
                                                        da_precision));
} // namespace b200

// The opaque handle of the C ABI (source/include/aoclda_handle.h:98).
struct _da_handle {
    da_precision precision = da_unknown;
    da_handle_type type = da_handle_uninitialized;
    b200::ErrorRecord err;
    b200::CudaCtx cuda;
    std::unique_ptr<b200::AlgBase> alg;
};
