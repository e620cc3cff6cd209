// extern "C" entry points of libaoclda_b200.so.  Names, argument meaning and
// status codes are those of the AOCL-DA C API; each function cites the
// reference implementation whose behaviour it reproduces.
#include "alg.hpp"
#include "../../include/aoclda_b200_ext.h"
#include <algorithm>

using namespace b200;

namespace b200 {

template <typename T>
cudaError_t upload_matrix(da_order order, da_int rows, da_int cols, const T *host, da_int ld,
                          T *dst, int ldo, DevBuf &stage, cudaStream_t s) {
    cudaError_t e;
    if (order == row_major) {
        e = cudaMemcpy2DAsync(dst, (size_t)ldo * sizeof(T), host, (size_t)ld * sizeof(T),
                              (size_t)cols * sizeof(T), rows, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        if (ldo > cols)
            e = cudaMemset2DAsync(dst + cols, (size_t)ldo * sizeof(T), 0,
                                  (size_t)(ldo - cols) * sizeof(T), rows, s);
        return e;
    }
    if (!stage.ensure((size_t)rows * cols * sizeof(T))) return cudaErrorMemoryAllocation;
    e = cudaMemcpy2DAsync(stage.p, (size_t)rows * sizeof(T), host, (size_t)ld * sizeof(T),
                          (size_t)rows * sizeof(T), cols, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return launch_colmajor_to_rowmajor<T>(stage.as<T>(), rows, cols, dst, ldo, s);
}

template <typename T>
cudaError_t download_matrix(da_order order, da_int rows, da_int cols, const T *dev, int ldi,
                            T *host, da_int ld, DevBuf &stage, cudaStream_t s) {
    if (order == row_major)
        return cudaMemcpy2DAsync(host, (size_t)ld * sizeof(T), dev, (size_t)ldi * sizeof(T),
                                 (size_t)cols * sizeof(T), rows, cudaMemcpyDeviceToHost, s);
    if (!stage.ensure((size_t)rows * cols * sizeof(T))) return cudaErrorMemoryAllocation;
    cudaError_t e = launch_rowmajor_to_colmajor<T>(dev, rows, cols, ldi, stage.as<T>(), rows, s);
    if (e != cudaSuccess) return e;
    return cudaMemcpy2DAsync(host, (size_t)ld * sizeof(T), stage.p, (size_t)rows * sizeof(T),
                             (size_t)rows * sizeof(T), cols, cudaMemcpyDeviceToHost, s);
}

template cudaError_t upload_matrix<float>(da_order, da_int, da_int, const float *, da_int, float *,
                                          int, DevBuf &, cudaStream_t);
template cudaError_t upload_matrix<double>(da_order, da_int, da_int, const double *, da_int,
                                           double *, int, DevBuf &, cudaStream_t);
template cudaError_t download_matrix<float>(da_order, da_int, da_int, const float *, int, float *,
                                            da_int, DevBuf &, cudaStream_t);
template cudaError_t download_matrix<double>(da_order, da_int, da_int, const double *, int,
                                             double *, da_int, DevBuf &, cudaStream_t);

} // namespace b200

namespace {

template <typename T> constexpr da_precision prec_of() {
    return std::is_same_v<T, double> ? da_double : da_single;
}

// check_precision<T> (da_handle.hpp:89)
template <typename T> da_status check_precision(da_handle h) {
    if (h->precision != prec_of<T>())
        return h->err.error(da_status_wrong_type,
                            "The handle was initialized with a different precision type than "
                            "the one used in this call.");
    return da_status_success;
}

template <typename T> NN<T> *as_nn(da_handle h) {
    return dynamic_cast<NN<T> *>(h->alg.get());
}
template <typename T> KMeans<T> *as_km(da_handle h) {
    return dynamic_cast<KMeans<T> *>(h->alg.get());
}
template <typename T> IVF<T> *as_ivf(da_handle h) {
    return dynamic_cast<IVF<T> *>(h->alg.get());
}

// da_handle_init (da_handle_public.cpp:34-197): only the handle types of
// this library's path (kNN, k-means, IVF-flat) are accepted.
da_status handle_init(da_handle *handle, da_handle_type type, da_precision prec) {
    if (handle == nullptr) return da_status_invalid_input;
    *handle = nullptr;
    std::unique_ptr<_da_handle> h;
    try {
        h.reset(new _da_handle());
    } catch (std::bad_alloc &) {
        return da_status_memory_error;
    }
    h->precision = prec;
    h->type = type;
    const bool single = prec == da_single;
    try {
        switch (type) {
        case da_handle_nn:
            if (single) h->alg.reset(new NN<float>(&h->err, &h->cuda, true));
            else h->alg.reset(new NN<double>(&h->err, &h->cuda, false));
            break;
        case da_handle_kmeans:
            if (single) h->alg.reset(new KMeans<float>(&h->err, &h->cuda, true));
            else h->alg.reset(new KMeans<double>(&h->err, &h->cuda, false));
            break;
        case da_handle_approx_nn:
            if (single) h->alg.reset(new IVF<float>(&h->err, &h->cuda, true));
            else h->alg.reset(new IVF<double>(&h->err, &h->cuda, false));
            break;
        case da_handle_uninitialized:
            break;
        default:
            return da_status_not_implemented;
        }
    } catch (std::bad_alloc &) {
        return da_status_memory_error;
    }
    *handle = h.release();
    return da_status_success;
}

#define NN_CALL(T, h, call)                                                                   \
    do {                                                                                      \
        if (!(h)) return da_status_handle_not_initialized;                                    \
        (h)->err.clear();                                                                     \
        da_status _s = check_precision<T>(h);                                                 \
        if (_s != da_status_success) return _s;                                               \
        auto *_a = as_nn<T>(h);                                                               \
        if (!_a)                                                                              \
            return (h)->err.error(da_status_invalid_handle_type,                              \
                                  "handle was not initialized with handle_type=da_handle_nn " \
                                  "or handle is invalid.");                                   \
        return _a->call;                                                                      \
    } while (0)

#define KM_CALL(T, h, call)                                                                   \
    do {                                                                                      \
        if (!(h)) return da_status_handle_not_initialized;                                    \
        (h)->err.clear();                                                                     \
        da_status _s = check_precision<T>(h);                                                 \
        if (_s != da_status_success) return _s;                                               \
        auto *_a = as_km<T>(h);                                                               \
        if (!_a)                                                                              \
            return (h)->err.error(da_status_invalid_handle_type,                              \
                                  "handle was not initialized with "                          \
                                  "handle_type=da_handle_kmeans or handle is invalid.");      \
        return _a->call;                                                                      \
    } while (0)

#define IVF_CALL(T, h, call)                                                                  \
    do {                                                                                      \
        if (!(h)) return da_status_handle_not_initialized;                                    \
        (h)->err.clear();                                                                     \
        da_status _s = check_precision<T>(h);                                                 \
        if (_s != da_status_success) return _s;                                               \
        auto *_a = as_ivf<T>(h);                                                              \
        if (!_a)                                                                              \
            return (h)->err.error(da_status_invalid_handle_type,                              \
                                  "handle was not initialized with "                          \
                                  "handle_type=da_handle_approx_nn or handle is invalid.");   \
        return _a->call;                                                                      \
    } while (0)

Registry *opts_of(da_handle h) {
    if (!h->alg) return nullptr;
    return &h->alg->opts;
}

// ------------------------------------------------------- pairwise distances --
ErrorRecord g_err;
CudaCtx g_cuda;
DevBuf g_X, g_Y, g_D, g_xn, g_yn, g_stage;

// pairwise_distances.cpp:37-114
template <typename T>
da_status pairwise(da_order order, da_int m, da_int n, da_int k, const T *X, da_int ldx,
                   const T *Y, da_int ldy, T *D, da_int ldd, T p, da_metric metric) {
    if (m < 1 || k < 1) return da_status_invalid_array_dimension;
    if (order == column_major && ldx < m) return da_status_invalid_leading_dimension;
    if (order == row_major && ldx < k) return da_status_invalid_leading_dimension;
    if (X == nullptr || D == nullptr) return da_status_invalid_pointer;
    if (Y != nullptr) {
        if (n < 1) return da_status_invalid_array_dimension;
        if (order == column_major) {
            if (ldy < n || ldd < m) return da_status_invalid_leading_dimension;
        } else {
            if (ldy < k || ldd < n) return da_status_invalid_leading_dimension;
        }
    } else {
        if (ldd < m) return da_status_invalid_leading_dimension;
    }
    if (metric == da_minkowski && p <= 0) return da_status_invalid_input;
    int acc = ACC_SQEUC, post = POST_NONE, norms = -1;
    switch (metric) {
    case da_euclidean: post = POST_SQRT; break;
    case da_sqeuclidean: break;
    case da_manhattan: acc = ACC_MANHATTAN; break;
    case da_cosine: acc = ACC_DOT; post = POST_COSINE; norms = 1; break;
    case da_minkowski:
        if (p == T(2)) post = POST_SQRT;
        else if (p == T(1)) acc = ACC_MANHATTAN;
        else { acc = ACC_MINKOWSKI; post = POST_POW; }
        break;
    case da_euclidean_gemm: acc = ACC_DOT; post = POST_GEMM_SQRT; norms = 0; break;
    case da_sqeuclidean_gemm: acc = ACC_DOT; post = POST_GEMM_SQ; norms = 0; break;
    case da_inner_product: acc = ACC_DOT; break;
    default: return da_status_not_implemented;
    }
    g_err.clear();
    da_status s = g_cuda.init(g_err);
    if (s != da_status_success) return s;
    const bool x_is_y = (Y == nullptr);
    if (x_is_y) {
        n = m;
        Y = X;
        ldy = ldx;
    }
    const int ld = pad4((int)k);
    cudaStream_t st = g_cuda.stream;
    if (!g_X.ensure((size_t)m * ld * sizeof(T)) || !g_Y.ensure((size_t)n * ld * sizeof(T)) ||
        !g_D.ensure((size_t)m * n * sizeof(T)) || !g_xn.ensure((size_t)m * sizeof(T)) ||
        !g_yn.ensure((size_t)n * sizeof(T)))
        return da_status_memory_error;
    auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    if (!ok(upload_matrix<T>(order, m, k, X, ldx, g_X.as<T>(), ld, g_stage, st)) ||
        !ok(upload_matrix<T>(order, n, k, Y, ldy, g_Y.as<T>(), ld, g_stage, st)))
        return da_status_internal_error;
    const T *xn = nullptr, *yn = nullptr;
    if (norms == 0) {
        if (!ok(launch_row_sqnorms<T>(g_X.as<T>(), ld, m, k, g_xn.as<T>(), st)) ||
            !ok(launch_row_sqnorms<T>(g_Y.as<T>(), ld, n, k, g_yn.as<T>(), st)))
            return da_status_internal_error;
    } else if (norms == 1) {
        if (!ok(launch_row_norms_eps1<T>(g_X.as<T>(), ld, m, k, g_xn.as<T>(), st)) ||
            !ok(launch_row_norms_eps1<T>(g_Y.as<T>(), ld, n, k, g_yn.as<T>(), st)))
            return da_status_internal_error;
    }
    if (norms >= 0) {
        xn = g_xn.as<T>();
        yn = g_yn.as<T>();
    }
    const int kc = sizeof(T) == 8 ? 512 : 256;
    PairwiseArgs a{acc, post, kc, (double)p, x_is_y, order == row_major};
    if (!ok(launch_pairwise<T>(g_X.as<T>(), ld, m, g_Y.as<T>(), ld, n, k, xn, yn, a, g_D.as<T>(), st)))
        return da_status_internal_error;
    cudaError_t e;
    if (order == row_major)
        e = cudaMemcpy2DAsync(D, (size_t)ldd * sizeof(T), g_D.p, (size_t)n * sizeof(T),
                              (size_t)n * sizeof(T), m, cudaMemcpyDeviceToHost, st);
    else
        e = cudaMemcpy2DAsync(D, (size_t)ldd * sizeof(T), g_D.p, (size_t)m * sizeof(T),
                              (size_t)m * sizeof(T), n, cudaMemcpyDeviceToHost, st);
    if (!ok(e) || !ok(cudaStreamSynchronize(st))) return da_status_internal_error;
    return da_status_success;
}

} // namespace

extern "C" {

// ---------------------------------------------------------------- handles --
da_status da_handle_init_d(da_handle *handle, da_handle_type t) {
    return handle_init(handle, t, da_double);
}
da_status da_handle_init_s(da_handle *handle, da_handle_type t) {
    return handle_init(handle, t, da_single);
}
void da_handle_destroy(da_handle *handle) {
    if (handle) {
        delete *handle;
        *handle = nullptr;
    }
}
da_status da_handle_print_error_message(da_handle handle) {
    if (!handle) return da_status_invalid_input;
    if (!handle->err.message.empty()) std::printf("%s\n", handle->err.message.c_str());
    return da_status_success;
}
da_status da_handle_get_error_message(da_handle handle, char **message) {
    if (!handle || !message) return da_status_invalid_input;
    const std::string &m = handle->err.message;
    *message = static_cast<char *>(std::malloc(m.size() + 1));
    if (!*message) return da_status_memory_error;
    std::memcpy(*message, m.c_str(), m.size() + 1);
    return da_status_success;
}
da_status da_handle_get_error_severity(da_handle handle, da_severity *severity) {
    if (!handle || !severity) return da_status_invalid_input;
    *severity = handle->err.severity;
    return da_status_success;
}
void da_handle_refresh(da_handle handle) {
    if (handle && handle->alg) handle->alg->refresh();
}

// ------------------------------------------------------ model persistence --
// da_handle_public.cpp:295-345 (file forms).  Layout: the 12-byte magic,
// uint32 format version, int32 handle type, int32 precision, the options
// (Registry::save), the algorithm's state (save_state), and the 64-bit
// FNV-1a hash of everything before it.
static const char kModelMagic[12] = {'A', 'O', 'C', 'L', 'D', 'A', '-', 'B', '2', '0', '0', '\n'};
static const uint32_t kModelVersion = 1;
static uint64_t fnv1a(const char *p, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= (unsigned char)p[i];
        h *= 1099511628211ull;
    }
    return h;
}

da_status da_handle_save_model(da_handle h, const char *file_name) {
    if (!h) return da_status_invalid_pointer;
    h->err.clear();
    if (!file_name) return h->err.error(da_status_invalid_pointer, "file_name cannot be null.");
    if (!h->alg) return h->err.error(da_status_invalid_input, "The handle is not initialized.");
    ByteWriter w;
    w.b.insert(w.b.end(), kModelMagic, kModelMagic + sizeof(kModelMagic));
    w.put<uint32_t>(kModelVersion);
    w.put<int32_t>((int32_t)h->type);
    w.put<int32_t>((int32_t)h->precision);
    h->alg->opts.save(w);
    da_status s = h->alg->save_state(w);
    if (s != da_status_success) return s;
    w.put<uint64_t>(fnv1a(w.b.data(), w.b.size()));
    std::FILE *f = std::fopen(file_name, "wb");
    if (!f) return h->err.error(da_status_io_error, "Cannot open the file for writing.");
    const size_t wrote = std::fwrite(w.b.data(), 1, w.b.size(), f);
    const int closed = std::fclose(f);
    if (wrote != w.b.size() || closed != 0)
        return h->err.error(da_status_io_error, "Writing the model file failed.");
    return da_status_success;
}

da_status da_handle_load_model(da_handle *handle, const char *file_name) {
    if (!handle || *handle || !file_name) return da_status_invalid_pointer;
    std::vector<char> buf;
    {
        std::FILE *f = std::fopen(file_name, "rb");
        if (!f) return da_status_io_error;
        char tmp[1 << 16];
        size_t got;
        while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
        const bool bad = std::ferror(f) != 0;
        std::fclose(f);
        if (bad) return da_status_io_error;
    }
    // a file of AOCL-DA's own da_handle_save_model (ref_model.cpp)
    if (is_reference_model(buf.data(), buf.size()))
        return load_reference_model(buf.data(), buf.size(), handle, handle_init);
    const size_t head = sizeof(kModelMagic) + 4 + 4 + 4;
    if (buf.size() < head + 8 || std::memcmp(buf.data(), kModelMagic, sizeof(kModelMagic)) != 0)
        return da_status_invalid_file_data;
    uint64_t sum;
    std::memcpy(&sum, buf.data() + buf.size() - 8, 8);
    if (sum != fnv1a(buf.data(), buf.size() - 8)) return da_status_invalid_file_data;
    ByteReader r;
    r.p = buf.data();
    r.n = buf.size() - 8;
    r.pos = sizeof(kModelMagic);
    if (r.get<uint32_t>() != kModelVersion) return da_status_version_mismatch;
    const int32_t type = r.get<int32_t>(), prec = r.get<int32_t>();
    if ((type != (int32_t)da_handle_nn && type != (int32_t)da_handle_kmeans &&
         type != (int32_t)da_handle_approx_nn) ||
        (prec != (int32_t)da_single && prec != (int32_t)da_double))
        return da_status_invalid_file_data;
    da_handle h = nullptr;
    da_status s = handle_init(&h, (da_handle_type)type, (da_precision)prec);
    if (s != da_status_success) return s;
    if (!h->alg->opts.load(r)) {
        delete h;
        return da_status_invalid_file_data;
    }
    s = h->alg->load_state(r);
    if (s == da_status_success && (!r.ok || r.pos != r.n)) s = da_status_invalid_file_data;
    if (s != da_status_success) {
        delete h;
        return s;
    }
    *handle = h;
    return da_status_success;
}

// ---------------------------------------------------------------- options --
// options_public.cpp:32-123
da_status da_options_set_int(da_handle h, const char *option, da_int value) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    Registry *r = opts_of(h);
    if (!r) return h->err.error(da_status_invalid_pointer, "handle seems to be corrupted.");
    h->alg->refresh();
    da_status s = r->set_int(option ? option : "", value);
    return s == da_status_success ? s : h->err.error(s, r->errmsg);
}
da_status da_options_set_string(da_handle h, const char *option, const char *value) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    Registry *r = opts_of(h);
    if (!r) return h->err.error(da_status_invalid_pointer, "handle seems to be corrupted.");
    h->alg->refresh();
    da_status s = r->set_string(option ? option : "", value ? value : "");
    return s == da_status_success ? s : h->err.error(s, r->errmsg);
}
extern "C++" template <typename T> da_status options_set_real(da_handle h, const char *option, T value) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    da_status s = check_precision<T>(h);
    if (s != da_status_success) return s;
    Registry *r = opts_of(h);
    if (!r) return h->err.error(da_status_invalid_pointer, "handle seems to be corrupted.");
    h->alg->refresh();
    s = r->set_real(option ? option : "", (double)value);
    return s == da_status_success ? s : h->err.error(s, r->errmsg);
}
da_status da_options_set_real_s(da_handle h, const char *option, float value) {
    return options_set_real<float>(h, option, value);
}
da_status da_options_set_real_d(da_handle h, const char *option, double value) {
    return options_set_real<double>(h, option, value);
}
da_status da_options_get_int(da_handle h, const char *option, da_int *value) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    Registry *r = opts_of(h);
    if (!r) return h->err.error(da_status_invalid_pointer, "handle seems to be corrupted.");
    if (!value) return h->err.error(da_status_invalid_input, "value is null.");
    da_status s = r->get_int(option ? option : "", *value);
    return s == da_status_success ? s : h->err.error(s, r->errmsg);
}
extern "C++" template <typename T> da_status options_get_real(da_handle h, const char *option, T *value) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    da_status s = check_precision<T>(h);
    if (s != da_status_success) return s;
    Registry *r = opts_of(h);
    if (!r) return h->err.error(da_status_invalid_pointer, "handle seems to be corrupted.");
    if (!value) return h->err.error(da_status_invalid_input, "value is null.");
    double v = 0;
    s = r->get_real(option ? option : "", v);
    if (s != da_status_success) return h->err.error(s, r->errmsg);
    *value = (T)v;
    return da_status_success;
}
da_status da_options_get_real_s(da_handle h, const char *option, float *value) {
    return options_get_real<float>(h, option, value);
}
da_status da_options_get_real_d(da_handle h, const char *option, double *value) {
    return options_get_real<double>(h, option, value);
}
static da_status options_get_str(da_handle h, const char *option, char *value, da_int *lvalue,
                                 da_int *key) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    Registry *r = opts_of(h);
    if (!r) return h->err.error(da_status_invalid_pointer, "handle seems to be corrupted.");
    if (!lvalue) return h->err.error(da_status_invalid_input, "lvalue is null.");
    std::string sv;
    da_status s = r->get_string(option ? option : "", sv, key);
    if (s != da_status_success) return h->err.error(s, r->errmsg);
    const size_t n = sv.size();
    if (value == nullptr || n >= (size_t)(*lvalue)) {
        *lvalue = (da_int)(n + 1);
        return h->err.error(da_status_invalid_input,
                            "target storage where to store option string value is too small, "
                            "make it at least " + std::to_string(n + 1) + " characters long");
    }
    std::memcpy(value, sv.c_str(), n + 1);
    return da_status_success;
}
da_status da_options_get_string(da_handle h, const char *option, char *value, da_int *lvalue) {
    return options_get_str(h, option, value, lvalue, nullptr);
}
da_status da_options_get_string_key(da_handle h, const char *option, char *value,
                                    da_int *lvalue, da_int *key) {
    return options_get_str(h, option, value, lvalue, key);
}
da_status da_options_print(da_handle h) {
    if (!h) return da_status_handle_not_initialized;
    Registry *r = opts_of(h);
    if (!r) return da_status_invalid_pointer;
    r->print();
    return da_status_success;
}

// ---------------------------------------------------------------- results --
// da_handle_public.cpp:233-262
extern "C++" template <typename T>
da_status get_result_impl(da_handle h, da_result q, da_int *dim, T *out) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    if (dim == nullptr) return h->err.error(da_status_invalid_input, "dim has not been defined");
    if (out == nullptr)
        return h->err.error(da_status_invalid_input, "The result array has not been allocated");
    if constexpr (std::is_same_v<T, da_int>) {
        if (!h->alg) return h->err.error(da_status_handle_not_initialized, "handle not initialized");
        return h->alg->get_result_int(q, dim, out);
    } else {
        da_status s = check_precision<T>(h);
        if (s != da_status_success) return s;
        if (!h->alg) return h->err.error(da_status_handle_not_initialized, "handle not initialized");
        return h->alg->get_result(q, dim, out);
    }
}
da_status da_handle_get_result_d(const da_handle h, da_result q, da_int *dim, double *out) {
    return get_result_impl<double>(h, q, dim, out);
}
da_status da_handle_get_result_s(const da_handle h, da_result q, da_int *dim, float *out) {
    return get_result_impl<float>(h, q, dim, out);
}
da_status da_handle_get_result_int(const da_handle h, da_result q, da_int *dim, da_int *out) {
    return get_result_impl<da_int>(h, q, dim, out);
}

// -------------------------------------------------------------------- kNN --
// nearest_neighbors_public.cpp / aoclda_c_wrapper.cpp:833-930
da_status da_nn_set_data_d(da_handle h, da_int n, da_int d, const double *X, da_int ldx) {
    NN_CALL(double, h, set_data(n, d, X, ldx));
}
da_status da_nn_set_data_s(da_handle h, da_int n, da_int d, const float *X, da_int ldx) {
    NN_CALL(float, h, set_data(n, d, X, ldx));
}
da_status da_nn_set_labels_d(da_handle h, da_int n, const da_int *y) { NN_CALL(double, h, set_labels(n, y)); }
da_status da_nn_set_labels_s(da_handle h, da_int n, const da_int *y) { NN_CALL(float, h, set_labels(n, y)); }
da_status da_nn_set_targets_d(da_handle h, da_int n, const double *y) { NN_CALL(double, h, set_targets(n, y)); }
da_status da_nn_set_targets_s(da_handle h, da_int n, const float *y) { NN_CALL(float, h, set_targets(n, y)); }
da_status da_nn_kneighbors_d(da_handle h, da_int nq, da_int d, const double *X, da_int ldx,
                             da_int *n_ind, double *n_dist, da_int k, da_int rd) {
    NN_CALL(double, h, kneighbors(nq, d, X, ldx, n_ind, n_dist, k, rd));
}
da_status da_nn_kneighbors_s(da_handle h, da_int nq, da_int d, const float *X, da_int ldx,
                             da_int *n_ind, float *n_dist, da_int k, da_int rd) {
    NN_CALL(float, h, kneighbors(nq, d, X, ldx, n_ind, n_dist, k, rd));
}
da_status da_nn_radius_neighbors_d(da_handle h, da_int nq, da_int d, const double *X, da_int ldx,
                                   double radius, da_int rd, da_int sort) {
    NN_CALL(double, h, radius_neighbors(nq, d, X, ldx, radius, rd, sort));
}
da_status da_nn_radius_neighbors_s(da_handle h, da_int nq, da_int d, const float *X, da_int ldx,
                                   float radius, da_int rd, da_int sort) {
    NN_CALL(float, h, radius_neighbors(nq, d, X, ldx, radius, rd, sort));
}

// IVF-flat (approximate_neighbors_public.cpp:30-127)
da_status da_approx_nn_set_training_data_d(da_handle h, da_int n, da_int d, const double *X,
                                           da_int ldx) {
    IVF_CALL(double, h, set_training_data(n, d, X, ldx));
}
da_status da_approx_nn_set_training_data_s(da_handle h, da_int n, da_int d, const float *X,
                                           da_int ldx) {
    IVF_CALL(float, h, set_training_data(n, d, X, ldx));
}
da_status da_approx_nn_train_d(da_handle h) { IVF_CALL(double, h, train()); }
da_status da_approx_nn_train_s(da_handle h) { IVF_CALL(float, h, train()); }
da_status da_approx_nn_add_d(da_handle h, da_int n, da_int d, const double *X, da_int ldx) {
    IVF_CALL(double, h, add(n, d, X, ldx));
}
da_status da_approx_nn_add_s(da_handle h, da_int n, da_int d, const float *X, da_int ldx) {
    IVF_CALL(float, h, add(n, d, X, ldx));
}
da_status da_approx_nn_train_and_add_d(da_handle h) { IVF_CALL(double, h, train_and_add()); }
da_status da_approx_nn_train_and_add_s(da_handle h) { IVF_CALL(float, h, train_and_add()); }
da_status da_approx_nn_kneighbors_d(da_handle h, da_int nq, da_int d, const double *X,
                                    da_int ldx, da_int *n_ind, double *n_dist, da_int k,
                                    da_int rd) {
    IVF_CALL(double, h, kneighbors(nq, d, X, ldx, n_ind, n_dist, k, rd));
}
da_status da_approx_nn_kneighbors_s(da_handle h, da_int nq, da_int d, const float *X,
                                    da_int ldx, da_int *n_ind, float *n_dist, da_int k,
                                    da_int rd) {
    IVF_CALL(float, h, kneighbors(nq, d, X, ldx, n_ind, n_dist, k, rd));
}
da_status da_nn_classes_d(da_handle h, da_int *nc, da_int *c) { NN_CALL(double, h, classes_api(nc, c)); }
da_status da_nn_classes_s(da_handle h, da_int *nc, da_int *c) { NN_CALL(float, h, classes_api(nc, c)); }
da_status da_nn_classifier_predict_proba_d(da_handle h, da_int nq, da_int d, const double *X,
                                           da_int ldx, double *proba, da_nn_search_mode m) {
    NN_CALL(double, h, predict_proba(nq, d, X, ldx, proba, m));
}
da_status da_nn_classifier_predict_proba_s(da_handle h, da_int nq, da_int d, const float *X,
                                           da_int ldx, float *proba, da_nn_search_mode m) {
    NN_CALL(float, h, predict_proba(nq, d, X, ldx, proba, m));
}
da_status da_nn_classifier_predict_d(da_handle h, da_int nq, da_int d, const double *X, da_int ldx,
                                     da_int *y, da_nn_search_mode m) {
    NN_CALL(double, h, predict(nq, d, X, ldx, y, m));
}
da_status da_nn_classifier_predict_s(da_handle h, da_int nq, da_int d, const float *X, da_int ldx,
                                     da_int *y, da_nn_search_mode m) {
    NN_CALL(float, h, predict(nq, d, X, ldx, y, m));
}
da_status da_nn_regressor_predict_d(da_handle h, da_int nq, da_int d, const double *X, da_int ldx,
                                    double *y, da_nn_search_mode m) {
    NN_CALL(double, h, predict_reg(nq, d, X, ldx, y, m));
}
da_status da_nn_regressor_predict_s(da_handle h, da_int nq, da_int d, const float *X, da_int ldx,
                                    float *y, da_nn_search_mode m) {
    NN_CALL(float, h, predict_reg(nq, d, X, ldx, y, m));
}

// ---------------------------------------------------------------- k-means --
// kmeans_public.cpp:32-104 / aoclda_c_wrapper.cpp:570-613
da_status da_kmeans_set_data_d(da_handle h, da_int n, da_int d, const double *A, da_int lda) {
    KM_CALL(double, h, set_data(n, d, A, lda));
}
da_status da_kmeans_set_data_s(da_handle h, da_int n, da_int d, const float *A, da_int lda) {
    KM_CALL(float, h, set_data(n, d, A, lda));
}
da_status da_kmeans_set_init_centres_d(da_handle h, const double *C, da_int ldc) {
    KM_CALL(double, h, set_init_centres(C, ldc));
}
da_status da_kmeans_set_init_centres_s(da_handle h, const float *C, da_int ldc) {
    KM_CALL(float, h, set_init_centres(C, ldc));
}
da_status da_kmeans_compute_d(da_handle h) { KM_CALL(double, h, compute()); }
da_status da_kmeans_compute_s(da_handle h) { KM_CALL(float, h, compute()); }
da_status da_kmeans_transform_d(da_handle h, da_int m, da_int d, const double *X, da_int ldx,
                                double *Xt, da_int ldxt) {
    KM_CALL(double, h, transform(m, d, X, ldx, Xt, ldxt));
}
da_status da_kmeans_transform_s(da_handle h, da_int m, da_int d, const float *X, da_int ldx,
                                float *Xt, da_int ldxt) {
    KM_CALL(float, h, transform(m, d, X, ldx, Xt, ldxt));
}
da_status da_kmeans_predict_d(da_handle h, da_int m, da_int d, const double *Y, da_int ldy,
                              da_int *labels) {
    KM_CALL(double, h, predict(m, d, Y, ldy, labels));
}
da_status da_kmeans_predict_s(da_handle h, da_int m, da_int d, const float *Y, da_int ldy,
                              da_int *labels) {
    KM_CALL(float, h, predict(m, d, Y, ldy, labels));
}

// ---------------------------------------------------- pairwise distances --
da_status da_pairwise_distances_d(da_order order, da_int m, da_int n, da_int k, const double *X,
                                  da_int ldx, const double *Y, da_int ldy, double *D, da_int ldd,
                                  double p, da_metric metric) {
    return pairwise<double>(order, m, n, k, X, ldx, Y, ldy, D, ldd, p, metric);
}
da_status da_pairwise_distances_s(da_order order, da_int m, da_int n, da_int k, const float *X,
                                  da_int ldx, const float *Y, da_int ldy, float *D, da_int ldd,
                                  float p, da_metric metric) {
    return pairwise<float>(order, m, n, k, X, ldx, Y, ldy, D, ldd, p, metric);
}

} // extern "C"

// ------------------------------------------------------- B200 extensions --
// include/aoclda_b200_ext.h: no counterpart in the reference API.
extern "C" {

da_status da_b200_set_stream(da_handle h, void *stream) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    da_status s = h->cuda.init(h->err);
    if (s != da_status_success) return s;
    h->cuda.stream = stream ? static_cast<cudaStream_t>(stream) : h->cuda.own_stream;
    return da_status_success;
}
da_status da_b200_set_stream_priority(da_handle h, da_int priority) {
    if (!h) return da_status_handle_not_initialized;
    h->err.clear();
    da_status s = h->cuda.init(h->err);
    if (s != da_status_success) return s;
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    const int p = std::max(greatest, std::min(least, (int)priority));
    cudaStream_t ns = nullptr;
    if (cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, p) != cudaSuccess) {
        cudaGetLastError();
        return h->err.error(da_status_internal_error, "cudaStreamCreateWithPriority failed.");
    }
    // the work in flight on the old stream completes first
    cudaStreamSynchronize(h->cuda.own_stream);
    const bool bound_own = h->cuda.stream == h->cuda.own_stream;
    cudaStreamDestroy(h->cuda.own_stream);
    h->cuda.own_stream = ns;
    if (bound_own) h->cuda.stream = ns;
    return da_status_success;
}
da_status da_b200_set_kernel_timing(da_handle h, da_int enable) {
    if (!h) return da_status_handle_not_initialized;
    if (!enable) h->cuda.flush_timing();
    h->cuda.timing = enable != 0;
    return da_status_success;
}
da_status da_b200_get_kernel_time(da_handle h, const char *kernel, double *total_ms,
                                  da_int *launches) {
    if (!h) return da_status_handle_not_initialized;
    if (!kernel || !total_ms || !launches) return da_status_invalid_pointer;
    h->cuda.flush_timing();
    auto it = h->cuda.ktime.find(kernel);
    if (it == h->cuda.ktime.end()) {
        *total_ms = 0;
        *launches = 0;
        return da_status_success;
    }
    *total_ms = it->second.first;
    *launches = (da_int)it->second.second;
    return da_status_success;
}
da_status da_b200_get_stat(da_handle h, const char *name, double *value) {
    if (!h) return da_status_handle_not_initialized;
    if (!name || !value) return da_status_invalid_pointer;
    auto it = h->cuda.stats.find(name);
    *value = it == h->cuda.stats.end() ? 0.0 : it->second;
    return da_status_success;
}
da_status da_b200_reset_kernel_time(da_handle h) {
    if (!h) return da_status_handle_not_initialized;
    h->cuda.flush_timing();
    h->cuda.ktime.clear();
    return da_status_success;
}
da_status da_b200_device_memory(unsigned long long *free_bytes, unsigned long long *total_bytes) {
    if (!free_bytes || !total_bytes) return da_status_invalid_pointer;
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
        cudaGetLastError();
        return da_status_arch_not_supported;
    }
    *free_bytes = f;
    *total_bytes = t;
    return da_status_success;
}
da_status da_b200_nn_share_data(da_handle h, da_handle source) {
    if (!h || !source) return da_status_handle_not_initialized;
    h->err.clear();
    if (h == source)
        return h->err.error(da_status_invalid_input, "A handle cannot share its own data.");
    if (h->precision != source->precision)
        return h->err.error(da_status_wrong_type,
                            "The two handles were initialized with different precisions.");
    if (h->precision == da_single) {
        auto *a = as_nn<float>(h), *b = as_nn<float>(source);
        if (!a || !b)
            return h->err.error(da_status_invalid_handle_type,
                                "Both handles must be initialized with handle_type=da_handle_nn.");
        return a->share_data(*b);
    }
    auto *a = as_nn<double>(h), *b = as_nn<double>(source);
    if (!a || !b)
        return h->err.error(da_status_invalid_handle_type,
                            "Both handles must be initialized with handle_type=da_handle_nn.");
    return a->share_data(*b);
}
da_status da_b200_kmeans_shard_colmax_s(da_handle h, float *colmax) {
    KM_CALL(float, h, shard_colmax(colmax));
}
da_status da_b200_kmeans_shard_begin_s(da_handle h, const float *colmax_global,
                                       da_int n_global, const float *centres) {
    KM_CALL(float, h, shard_begin(colmax_global, n_global, centres));
}
da_status da_b200_kmeans_shard_partial_s(da_handle h, long long *acc) {
    KM_CALL(float, h, shard_partial(acc));
}
da_status da_b200_kmeans_shard_finalize_s(da_handle h, const long long *acc, double *scalars,
                                          da_int *flags) {
    KM_CALL(float, h, shard_finalize(acc, scalars, flags));
}
da_status da_b200_kmeans_shard_inertia_s(da_handle h, da_int relabel, double *inertia) {
    KM_CALL(float, h, shard_relabel(inertia, relabel != 0));
}
da_status da_b200_kmeans_shard_result_s(da_handle h, float *centres, da_int *labels) {
    KM_CALL(float, h, shard_result(centres, labels));
}
da_status da_b200_kmeans_init_centres_d(da_handle h, double *C, da_int ldc) {
    KM_CALL(double, h, initial_centres(C, ldc));
}
da_status da_b200_kmeans_init_centres_s(da_handle h, float *C, da_int ldc) {
    KM_CALL(float, h, initial_centres(C, ldc));
}

} // extern "C"
