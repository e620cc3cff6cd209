/*
 * aoclda_b200.h -- C ABI of the B200 (sm_100a) distance / kNN / k-means library.
 *
 * The library is a drop-in for the AOCL-DA entry points of one hot path: the
 * blocked pairwise-distance kernel and its two consumers, brute-force
 * k-nearest neighbours and k-means (Lloyd).  Every symbol below keeps the
 * name, argument meaning, enum values and status codes of the AOCL-DA C API,
 * so a program written against that API links against libaoclda_b200.so
 * unchanged.  Each declaration cites the AOCL-DA header line it replaces
 * (paths relative to the AOCL-DA source tree).
 *
 * Plain C types only: pointers are HOST pointers, sizes are da_int.  Device
 * memory, streams and kernels are internal to the handle.
 */
#ifndef AOCLDA_B200_H
#define AOCLDA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- basic types: source/include/aoclda_types.h:42-92 ------------------- */
#if defined(AOCLDA_ILP64)
typedef int64_t da_int;
#else
typedef int32_t da_int;
#endif

enum da_precision_ { da_unknown = 255, da_double = 0, da_single = 1 };
typedef enum da_precision_ da_precision;

enum da_order_ { row_major = 0, column_major = 1 };
typedef enum da_order_ da_order;

/* ---- status codes: source/include/aoclda_error.h:38-110 ----------------- */
enum da_status_ {
    da_status_success = 0,
    da_status_internal_error = 1,
    da_status_memory_error = 2,
    da_status_invalid_pointer = 3,
    da_status_invalid_input = 4,
    da_status_not_implemented = 5,
    da_status_out_of_date = 6,
    da_status_wrong_type = 7,
    da_status_overflow = 8,
    da_status_invalid_handle_type = 9,
    da_status_handle_not_initialized = 10,
    da_status_store_not_initialized = 11,
    da_status_invalid_option = 12,
    da_status_incompatible_options = 13,
    da_status_operation_failed = 14,
    da_status_invalid_leading_dimension = 15,
    da_status_negative_data = 16,
    da_status_invalid_array_dimension = 17,
    da_status_unknown_query = 18,
    da_status_incorrect_output = 19,
    da_status_no_data = 20,
    da_status_maxit = 21,
    da_status_maxtime = 22,
    da_status_numerical_difficulties = 23,
    da_status_bad_derivatives = 24,
    da_status_arch_not_supported = 25,
    da_status_io_error = 26,
    da_status_file_reading_error = 100,
    da_status_parsing_error = 101,
    da_status_missing_data = 102,
    da_status_option_not_found = 400,
    da_status_option_locked = 401,
    da_status_option_wrong_type = 402,
    da_status_option_invalid_bounds = 403,
    da_status_option_invalid_value = 404,
    da_status_outlier_warning = 700,
    da_status_serialization_error = 800,
    da_status_invalid_file_data = 801,
    da_status_version_mismatch = 802,
    da_status_empty_clusters = 900
};
typedef enum da_status_ da_status;

/* source/include/aoclda_error.h:112-116 */
typedef enum da_severity_ { DA_NOTSET = 0, DA_WARNING = 1, DA_ERROR = 2 } da_severity;

/* ---- handles: source/include/aoclda_handle.h:45-98 ---------------------- */
enum da_handle_type_ {
    da_handle_uninitialized = 0,
    da_handle_linmod = 1,
    da_handle_pca = 2,
    da_handle_kmeans = 3,
    da_handle_dbscan = 4,
    da_handle_decision_tree = 5,
    da_handle_decision_forest = 6,
    da_handle_nlls = 7,
    da_handle_nn = 8,
    da_handle_svm = 9,
    da_handle_interpolation = 10,
    da_handle_approx_nn = 11,
    da_handle_kernel_pca = 12,
    da_handle_tsne = 13
};
typedef enum da_handle_type_ da_handle_type;

typedef struct _da_handle *da_handle;

/* ---- results: source/include/aoclda_result.h:43-111 --------------------- */
enum da_result_ {
    da_rinfo = 1,
    da_trained = 2,
    da_kmeans_cluster_centres = 501,
    da_kmeans_labels = 502,
    da_nn_radius_neighbors_count = 601,
    da_nn_radius_neighbors_offsets = 602,
    da_nn_radius_neighbors_indices = 603,
    da_nn_radius_neighbors_distances = 604,
    da_nn_radius_neighbors_indices_index = 605,
    da_nn_radius_neighbors_distances_index = 606,
    da_approx_nn_cluster_centroids = 801,
    da_approx_nn_list_sizes = 802
};
typedef enum da_result_ da_result;

/* ---- metrics: source/include/aoclda_metrics.h:44-59 --------------------- */
enum da_metric_ {
    da_euclidean = 0,
    da_l2 = da_euclidean,
    da_sqeuclidean = 1,
    da_minkowski = 2,
    da_manhattan = 3,
    da_l1 = da_manhattan,
    da_cityblock = da_manhattan,
    da_cosine = 4,
    da_euclidean_gemm = 5,
    da_sqeuclidean_gemm = 6,
    da_inner_product = 7
};
typedef enum da_metric_ da_metric;

/* ---- kNN search mode: source/include/aoclda_nearest_neighbors.h:45-51 --- */
enum da_nn_search_mode_ { knn_search_mode = 0, radius_search_mode = 1 };
typedef enum da_nn_search_mode_ da_nn_search_mode;

/* ======================================================================== */
/* Handle lifecycle and diagnostics                                          */
/* ======================================================================== */
/* source/include/aoclda_handle.h:118 */
da_status da_handle_init_d(da_handle *handle, da_handle_type handle_type);
/* source/include/aoclda_handle.h:119 */
da_status da_handle_init_s(da_handle *handle, da_handle_type handle_type);
/* source/include/aoclda_handle.h:133 */
da_status da_handle_print_error_message(da_handle handle);
/* source/include/aoclda_handle.h:146 */
void da_handle_destroy(da_handle *handle);
/* source/include/aoclda_handle.h:149 (the caller frees *message with free()) */
da_status da_handle_get_error_message(da_handle handle, char **message);
/* source/include/aoclda_handle.h:150 */
da_status da_handle_get_error_severity(da_handle handle, da_severity *severity);
/* source/include/aoclda_handle.h:153 */
void da_handle_refresh(da_handle handle);
/* source/include/aoclda_handle.h:177 -- a trained kNN (training data set),
 * k-means (computed) or IVF-flat (trained) handle to a file: its options and
 * its state (kNN: the training rows and labels / targets; k-means: centres,
 * labels, run information; IVF-flat: centroids, run information and the
 * inverted lists).  The file format is this library's own (a magic string,
 * format version 1, handle type, precision, options, state, FNV-1a
 * checksum), not the reference's. */
da_status da_handle_save_model(da_handle handle, const char *file_name);
/* source/include/aoclda_handle.h:201 -- a new handle (*handle must be null)
 * from a file written by da_handle_save_model -- this library's, or
 * AOCL-DA's own format (utilities/model_persistence.cpp) for k-means, kNN and
 * IVF-flat models: da_status_io_error when it cannot be read,
 * da_status_invalid_file_data when it is not a model file or is corrupted,
 * da_status_version_mismatch for another format version,
 * da_status_not_implemented for an AOCL-DA model of another handle type. */
da_status da_handle_load_model(da_handle *handle, const char *file_name);

/* ======================================================================== */
/* Options                                                                   */
/* ======================================================================== */
/* source/include/aoclda_options.h:48 */
da_status da_options_set_int(da_handle handle, const char *option, da_int value);
/* source/include/aoclda_options.h:49 */
da_status da_options_set_string(da_handle handle, const char *option, const char *value);
/* source/include/aoclda_options.h:67 */
da_status da_options_set_real_s(da_handle handle, const char *option, float value);
/* source/include/aoclda_options.h:68 */
da_status da_options_set_real_d(da_handle handle, const char *option, double value);
/* source/include/aoclda_options.h:82 */
da_status da_options_get_int(da_handle handle, const char *option, da_int *value);
/* source/include/aoclda_options.h:96 */
da_status da_options_get_real_s(da_handle handle, const char *option, float *value);
/* source/include/aoclda_options.h:97 */
da_status da_options_get_real_d(da_handle handle, const char *option, double *value);
/* source/include/aoclda_options.h:113 */
da_status da_options_get_string(da_handle handle, const char *option, char *value,
                                da_int *lvalue);
/* source/include/aoclda_options.h:130 */
da_status da_options_get_string_key(da_handle handle, const char *option, char *value,
                                    da_int *lvalue, da_int *key);
/* source/include/aoclda_options.h:140 */
da_status da_options_print(da_handle handle);

/* ======================================================================== */
/* Results                                                                   */
/* ======================================================================== */
/* source/include/aoclda_result.h:139 */
da_status da_handle_get_result_d(const da_handle handle, da_result query, da_int *dim,
                                 double *result);
/* source/include/aoclda_result.h:142 */
da_status da_handle_get_result_s(const da_handle handle, da_result query, da_int *dim,
                                 float *result);
/* source/include/aoclda_result.h:145 */
da_status da_handle_get_result_int(const da_handle handle, da_result query, da_int *dim,
                                   da_int *result);

/* ======================================================================== */
/* Brute-force k-nearest neighbours                                          */
/* ======================================================================== */
/* source/include/aoclda_nearest_neighbors.h:75 */
da_status da_nn_set_data_d(da_handle handle, da_int n_samples, da_int n_features,
                           const double *X_train, da_int ldx_train);
/* source/include/aoclda_nearest_neighbors.h:77 */
da_status da_nn_set_data_s(da_handle handle, da_int n_samples, da_int n_features,
                           const float *X_train, da_int ldx_train);
/* source/include/aoclda_nearest_neighbors.h:96 */
da_status da_nn_set_labels_s(da_handle handle, da_int n_samples, const da_int *y_train);
/* source/include/aoclda_nearest_neighbors.h:97 */
da_status da_nn_set_labels_d(da_handle handle, da_int n_samples, const da_int *y_train);
/* source/include/aoclda_nearest_neighbors.h:115 */
da_status da_nn_set_targets_d(da_handle handle, da_int n_samples, const double *y_train);
/* source/include/aoclda_nearest_neighbors.h:116 */
da_status da_nn_set_targets_s(da_handle handle, da_int n_samples, const float *y_train);
/* source/include/aoclda_nearest_neighbors.h:144 */
da_status da_nn_kneighbors_d(da_handle handle, da_int n_queries, da_int n_features,
                             const double *X_test, da_int ldx_test, da_int *n_ind,
                             double *n_dist, da_int k, da_int return_distance);
/* source/include/aoclda_nearest_neighbors.h:147 */
da_status da_nn_kneighbors_s(da_handle handle, da_int n_queries, da_int n_features,
                             const float *X_test, da_int ldx_test, da_int *n_ind,
                             float *n_dist, da_int k, da_int return_distance);
/* source/include/aoclda_nearest_neighbors.h:188 -- brute force on the GPU;
 * per query the training rows within `radius` in index order (sort_results:
 * stable by distance); the results through da_handle_get_result_? /
 * _int with the da_nn_radius_neighbors_* queries */
da_status da_nn_radius_neighbors_d(da_handle handle, da_int n_queries, da_int n_features,
                                   const double *X_test, da_int ldx_test, double radius,
                                   da_int return_distance, da_int sort_results);
/* source/include/aoclda_nearest_neighbors.h:191 */
da_status da_nn_radius_neighbors_s(da_handle handle, da_int n_queries, da_int n_features,
                                   const float *X_test, da_int ldx_test, float radius,
                                   da_int return_distance, da_int sort_results);
/* source/include/aoclda_nearest_neighbors.h:214 */
da_status da_nn_classes_d(da_handle handle, da_int *n_classes, da_int *classes);
/* source/include/aoclda_nearest_neighbors.h:215 */
da_status da_nn_classes_s(da_handle handle, da_int *n_classes, da_int *classes);
/* source/include/aoclda_nearest_neighbors.h:249 */
da_status da_nn_classifier_predict_proba_d(da_handle handle, da_int n_queries,
                                           da_int n_features, const double *X_test,
                                           da_int ldx_test, double *proba,
                                           da_nn_search_mode search_mode);
/* source/include/aoclda_nearest_neighbors.h:253 */
da_status da_nn_classifier_predict_proba_s(da_handle handle, da_int n_queries,
                                           da_int n_features, const float *X_test,
                                           da_int ldx_test, float *proba,
                                           da_nn_search_mode search_mode);
/* source/include/aoclda_nearest_neighbors.h:290 */
da_status da_nn_classifier_predict_d(da_handle handle, da_int n_queries,
                                     da_int n_features, const double *X_test,
                                     da_int ldx_test, da_int *y_test,
                                     da_nn_search_mode search_mode);
/* source/include/aoclda_nearest_neighbors.h:294 */
da_status da_nn_classifier_predict_s(da_handle handle, da_int n_queries,
                                     da_int n_features, const float *X_test,
                                     da_int ldx_test, da_int *y_test,
                                     da_nn_search_mode search_mode);
/* source/include/aoclda_nearest_neighbors.h:330 */
da_status da_nn_regressor_predict_d(da_handle handle, da_int n_queries, da_int n_features,
                                    const double *X_test, da_int ldx_test, double *y_test,
                                    da_nn_search_mode search_mode);
/* source/include/aoclda_nearest_neighbors.h:333 */
da_status da_nn_regressor_predict_s(da_handle handle, da_int n_queries, da_int n_features,
                                    const float *X_test, da_int ldx_test, float *y_test,
                                    da_nn_search_mode search_mode);

/* ======================================================================== */
/* IVF-flat approximate neighbours (handle type da_handle_approx_nn; options  */
/* "n_list", "n_probe", "k-means_iter", "seed", "train fraction",            */
/* "number of neighbors", "algorithm", "metric": euclidean / sqeuclidean)    */
/* ======================================================================== */
/* source/include/aoclda_approximate_neighbors.h:64 */
da_status da_approx_nn_set_training_data_d(da_handle handle, da_int n_samples,
                                           da_int n_features, const double *X_train,
                                           da_int ldx_train);
/* source/include/aoclda_approximate_neighbors.h:68 */
da_status da_approx_nn_set_training_data_s(da_handle handle, da_int n_samples,
                                           da_int n_features, const float *X_train,
                                           da_int ldx_train);
/* source/include/aoclda_approximate_neighbors.h:98 */
da_status da_approx_nn_train_d(da_handle handle);
/* source/include/aoclda_approximate_neighbors.h:100 */
da_status da_approx_nn_train_s(da_handle handle);
/* source/include/aoclda_approximate_neighbors.h:127 */
da_status da_approx_nn_add_d(da_handle handle, da_int n_samples_add, da_int n_features,
                             const double *X_add, da_int ldx_add);
/* source/include/aoclda_approximate_neighbors.h:130 */
da_status da_approx_nn_add_s(da_handle handle, da_int n_samples_add, da_int n_features,
                             const float *X_add, da_int ldx_add);
/* source/include/aoclda_approximate_neighbors.h:152 */
da_status da_approx_nn_train_and_add_d(da_handle handle);
/* source/include/aoclda_approximate_neighbors.h:154 */
da_status da_approx_nn_train_and_add_s(da_handle handle);
/* source/include/aoclda_approximate_neighbors.h:184 */
da_status da_approx_nn_kneighbors_d(da_handle handle, da_int n_queries, da_int n_features,
                                    const double *X_test, da_int ldx_test, da_int *n_ind,
                                    double *n_dist, da_int k, da_int return_distance);
/* source/include/aoclda_approximate_neighbors.h:188 */
da_status da_approx_nn_kneighbors_s(da_handle handle, da_int n_queries, da_int n_features,
                                    const float *X_test, da_int ldx_test, da_int *n_ind,
                                    float *n_dist, da_int k, da_int return_distance);

/* ======================================================================== */
/* k-means (Lloyd)                                                           */
/* ======================================================================== */
/* source/include/aoclda_kmeans.h:56 */
da_status da_kmeans_set_data_d(da_handle handle, da_int n_samples, da_int n_features,
                               const double *A, da_int lda);
/* source/include/aoclda_kmeans.h:59 */
da_status da_kmeans_set_data_s(da_handle handle, da_int n_samples, da_int n_features,
                               const float *A, da_int lda);
/* source/include/aoclda_kmeans.h:85 */
da_status da_kmeans_set_init_centres_d(da_handle handle, const double *C, da_int ldc);
/* source/include/aoclda_kmeans.h:87 */
da_status da_kmeans_set_init_centres_s(da_handle handle, const float *C, da_int ldc);
/* source/include/aoclda_kmeans.h:119 */
da_status da_kmeans_compute_d(da_handle handle);
/* source/include/aoclda_kmeans.h:121 */
da_status da_kmeans_compute_s(da_handle handle);
/* source/include/aoclda_kmeans.h:145 */
da_status da_kmeans_transform_d(da_handle handle, da_int m_samples, da_int m_features,
                                const double *X, da_int ldx, double *X_transform,
                                da_int ldx_transform);
/* source/include/aoclda_kmeans.h:149 */
da_status da_kmeans_transform_s(da_handle handle, da_int m_samples, da_int m_features,
                                const float *X, da_int ldx, float *X_transform,
                                da_int ldx_transform);
/* source/include/aoclda_kmeans.h:174 */
da_status da_kmeans_predict_d(da_handle handle, da_int k_samples, da_int k_features,
                              const double *Y, da_int ldy, da_int *Y_labels);
/* source/include/aoclda_kmeans.h:177 */
da_status da_kmeans_predict_s(da_handle handle, da_int k_samples, da_int k_features,
                              const float *Y, da_int ldy, da_int *Y_labels);

/* ======================================================================== */
/* Pairwise distances                                                        */
/* ======================================================================== */
/* source/include/aoclda_metrics.h:99 */
da_status da_pairwise_distances_d(da_order order, da_int m, da_int n, da_int k,
                                  const double *X, da_int ldx, const double *Y,
                                  da_int ldy, double *D, da_int ldd, double p,
                                  da_metric metric);
/* source/include/aoclda_metrics.h:104 */
da_status da_pairwise_distances_s(da_order order, da_int m, da_int n, da_int k,
                                  const float *X, da_int ldx, const float *Y, da_int ldy,
                                  float *D, da_int ldd, float p, da_metric metric);

#ifdef __cplusplus
}
#endif

#endif /* AOCLDA_B200_H */
