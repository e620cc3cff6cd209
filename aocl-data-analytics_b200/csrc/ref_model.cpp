// Reading model files written by AOCL-DA's da_handle_save_model
// (utilities/model_persistence.{hpp,cpp}, utilities/basic_handle.cpp:
// 277-323, utilities/da_handle.cpp:63-160), for the handle types of this
// library: k-means (clustering/kmeans/kmeans.cpp:1882-1909), kNN
// (nearest_neighbors/nearest_neighbors.cpp:2329-2404) and IVF-flat
// (approximate_neighbors/approximate_neighbors.cpp:1346-1395).
//
// The stream is a sequence of fields in native byte order: integers, enums
// and da_int as int64, bool as one byte, reals in the working precision;
// strings and vectors as an int64 element count followed by the elements
// (nested vectors recursively).  It opens with the metadata: the keyword
// "AOCLDA_STORED_MODEL", the writer's da_int size (4 or 8), the
// serialization version (50301), the handle type, the precision in bytes
// (4 or 8) and the writer's version string; then the option registry (count,
// then per option its name and value: int64, real or label string); then
// the algorithm's fields.  A kNN model with a k-d or ball tree carries the
// tree after the fields; the B200 search is brute force, so it is not read.
#include "alg.hpp"
#include <cstring>

namespace b200 {

namespace {

constexpr int64_t kRefVersion = 50301; // model_persistence_min_version
constexpr char kRefKeyword[] = "AOCLDA_STORED_MODEL";

struct RefStream {
    const char *p;
    size_t n, pos = 0;
    bool ok = true;
    int64_t i64() {
        int64_t v = 0;
        if (!ok || n - pos < 8) {
            ok = false;
            return 0;
        }
        std::memcpy(&v, p + pos, 8);
        pos += 8;
        return v;
    }
    bool b() {
        if (!ok || n - pos < 1) {
            ok = false;
            return false;
        }
        return p[pos++] != 0;
    }
    template <typename T> T real() {
        T v{};
        if (!ok || n - pos < sizeof(T)) {
            ok = false;
            return v;
        }
        std::memcpy(&v, p + pos, sizeof(T));
        pos += sizeof(T);
        return v;
    }
    // element count of a container: non-negative and within the bytes left
    int64_t count(size_t elem) {
        const int64_t c = i64();
        if (!ok || c < 0 || (uint64_t)c > (n - pos) / (elem ? elem : 1)) {
            ok = false;
            return 0;
        }
        return c;
    }
    std::string str() {
        const int64_t c = count(1);
        if (!ok) return std::string();
        std::string s(p + pos, p + pos + c);
        pos += (size_t)c;
        return s;
    }
    template <typename T> std::vector<T> vec() {
        const int64_t c = count(sizeof(T));
        std::vector<T> v;
        if (!ok) return v;
        v.resize((size_t)c);
        if (c) std::memcpy(v.data(), p + pos, (size_t)c * sizeof(T));
        pos += (size_t)c * sizeof(T);
        return v;
    }
    std::vector<int64_t> ivec() { return vec<int64_t>(); }
    template <typename T> std::vector<std::vector<T>> vvec() {
        const int64_t c = count(8); // every inner vector has its own count
        std::vector<std::vector<T>> v;
        for (int64_t i = 0; ok && i < c; ++i) v.push_back(vec<T>());
        return v;
    }
};

// The option types of the reference's registries (basic_handle_options.hpp,
// kmeans_options.hpp, nearest_neighbors_options.hpp,
// approximate_neighbors_options.hpp): 'I' da_int, 'R' the working
// precision, 'S' a label.
char option_kind(da_handle_type type, const std::string &name) {
    static const std::pair<const char *, char> common[] = {{"storage order", 'S'},
                                                           {"check data", 'S'}};
    static const std::pair<const char *, char> km[] = {
        {"n_clusters", 'I'}, {"n_init", 'I'}, {"max_iter", 'I'}, {"low precision max_iter", 'I'},
        {"seed", 'I'}, {"afk-mc2 samples", 'I'}, {"initialization method", 'S'},
        {"algorithm", 'S'}, {"mixed precision", 'S'}, {"empty clusters", 'S'},
        {"distance", 'S'}, {"normalize data", 'S'}, {"convergence tolerance", 'R'},
        {"low precision convergence tolerance", 'R'}};
    static const std::pair<const char *, char> nn[] = {
        {"number of neighbors", 'I'}, {"leaf size", 'I'}, {"outlier label", 'I'},
        {"minkowski parameter", 'R'}, {"radius", 'R'}, {"outlier target", 'R'},
        {"algorithm", 'S'}, {"metric", 'S'}, {"weights", 'S'}, {"outlier handling", 'S'}};
    static const std::pair<const char *, char> ann[] = {
        {"number of neighbors", 'I'}, {"n_list", 'I'}, {"n_probe", 'I'},
        {"k-means_iter", 'I'}, {"seed", 'I'}, {"train fraction", 'R'}, {"algorithm", 'S'},
        {"metric", 'S'}};
    for (auto &e : common)
        if (name == e.first) return e.second;
    auto look = [&](const std::pair<const char *, char> *t, size_t m) {
        for (size_t i = 0; i < m; ++i)
            if (name == t[i].first) return t[i].second;
        return '\0';
    };
    if (type == da_handle_kmeans) return look(km, sizeof(km) / sizeof(km[0]));
    if (type == da_handle_nn) return look(nn, sizeof(nn) / sizeof(nn[0]));
    if (type == da_handle_approx_nn) return look(ann, sizeof(ann) / sizeof(ann[0]));
    return '\0';
}

// The registry (OptionRegistry::load_registry, utilities/options.hpp:
// 977-1009) into this library's registry: every saved option is known to the
// reference's registry of that handle; one this library does not register
// is read and dropped.
template <typename T>
da_status load_registry(RefStream &r, da_handle_type type, Registry &opts) {
    const int64_t count = r.i64();
    if (!r.ok || count < 0 || count > 64) return da_status_invalid_file_data;
    for (int64_t i = 0; i < count; ++i) {
        const std::string name = r.str();
        if (!r.ok) return da_status_invalid_file_data;
        da_status s = da_status_success;
        switch (option_kind(type, name)) {
        case 'I': {
            const int64_t v = r.i64();
            if (!r.ok) return da_status_invalid_file_data;
            s = opts.set_int(name, (da_int)v);
            break;
        }
        case 'R': {
            const T v = r.real<T>();
            if (!r.ok) return da_status_invalid_file_data;
            s = opts.set_real(name, (double)v);
            break;
        }
        case 'S': {
            const std::string v = r.str();
            if (!r.ok) return da_status_invalid_file_data;
            s = opts.set_string(name, v);
            break;
        }
        default: return da_status_invalid_file_data;
        }
        if (s != da_status_success && s != da_status_option_not_found)
            return da_status_invalid_file_data;
    }
    return da_status_success;
}

constexpr int64_t kRowMajor = 0, kColumnMajor = 1; // da_order of aoclda_types.h

// kmeans<T>::serialize (kmeans.cpp:1882-1909)
template <typename T> da_status load_kmeans(RefStream &r, KMeans<T> &km) {
    const bool trained = r.b();
    const int64_t ord = r.i64();
    (void)r.i64(); // algorithm
    const int64_t n = r.i64(), d = r.i64(), nit = r.i64();
    const T inertia = r.real<T>();
    (void)r.i64(); // seed
    const int64_t k = r.i64();
    (void)r.real<T>(); // tol
    (void)r.i64();     // max_iter
    (void)r.i64();     // n_init
    const std::vector<int64_t> lab = r.ivec();
    std::vector<T> cen = r.vec<T>();
    (void)r.vec<T>(); // workc1: the centres' squared norms
    const bool sph = r.b(), sph_norm = r.b();
    const int64_t imax = std::numeric_limits<da_int>::max();
    if (!r.ok || !trained || (ord != kRowMajor && ord != kColumnMajor) || n < 1 || d < 1 ||
        k < 1 || k > n || n > imax || d > imax || lab.size() != (size_t)n ||
        cen.size() / (size_t)k != (size_t)d || cen.size() != (size_t)k * (size_t)d)
        return da_status_invalid_file_data;
    for (int64_t v : lab)
        if (v < 0 || v >= k) return da_status_invalid_file_data;
    km.n_samples = (da_int)n;
    km.n_features = (da_int)d;
    km.n_clusters = (da_int)k;
    km.data_order = ord == kRowMajor ? row_major : column_major;
    km.best_n_iter = (da_int)nit;
    km.best_lp_n_iter = 0;
    km.best_inertia = (double)inertia;
    km.warn_maxit = false;
    km.best_centres = std::move(cen); // column-major k x d in both libraries
    km.best_labels.assign(lab.begin(), lab.end());
    km.best_labels_on_host = true;
    km.model_sph = sph;
    km.model_sph_norm = sph_norm;
    km.ld = pad4(km.n_features);
    km.initdone = false;
    km.model_trained = true;
    return da_status_success;
}

// neighbors<T>::serialize (nearest_neighbors.cpp:2329-2404): the training
// rows column-major n x d, then the labels and targets (empty when not set).
template <typename T> da_status load_nn(RefStream &r, NN<T> &nn) {
    const int64_t ord = r.i64(), n = r.i64(), d = r.i64();
    const bool has_labels = r.b(), has_targets = r.b();
    (void)r.b();       // is_up_to_date
    (void)r.b();       // classes_computed
    (void)r.ivec();    // classes
    (void)r.b();       // sort_results
    (void)r.b();       // model_trained
    (void)r.b();       // rnn_return_distances
    for (int i = 0; i < 6; ++i) (void)r.i64(); // n_neighbors .. leaf_size
    (void)r.b();       // get_squares
    (void)r.real<T>(); // p
    for (int i = 0; i < 3; ++i) (void)r.i64(); // weights, outlier_handling, n_classes
    (void)r.real<T>(); // radius
    (void)r.ivec();    // radius_neighbors_count
    (void)r.vvec<int64_t>();
    (void)r.vvec<T>();
    const bool has_x = r.b(); // istrained_Xtrain
    (void)r.b();
    (void)r.i64();
    (void)r.b();
    (void)r.i64();
    (void)r.i64();
    (void)r.b();
    (void)r.real<T>();
    (void)r.real<T>();
    std::vector<T> X = r.vec<T>();
    const std::vector<int64_t> y = r.ivec();
    std::vector<T> t = r.vec<T>();
    const int64_t imax = std::numeric_limits<da_int>::max();
    if (!r.ok || !has_x || (ord != kRowMajor && ord != kColumnMajor) || n < 1 || d < 1 ||
        n > imax || d > imax || X.size() / (size_t)n != (size_t)d ||
        X.size() != (size_t)n * (size_t)d || (has_labels && y.size() != (size_t)n) ||
        (has_targets && t.size() != (size_t)n))
        return da_status_invalid_file_data;
    // the rows in the handle's storage order, owned by the handle
    if (nn.order() == row_major) {
        nn.X_own.resize(X.size());
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < d; ++j) nn.X_own[(size_t)i * d + j] = X[(size_t)j * n + i];
    } else {
        nn.X_own = std::move(X);
    }
    da_status s = nn.set_data((da_int)n, (da_int)d, nn.X_own.data(),
                              nn.order() == row_major ? (da_int)d : (da_int)n);
    if (s != da_status_success) return s;
    if (has_labels) {
        nn.y_own.assign(y.begin(), y.end());
        s = nn.set_labels((da_int)n, nn.y_own.data());
        if (s != da_status_success) return s;
    }
    if (has_targets) {
        nn.t_own = std::move(t);
        s = nn.set_targets((da_int)n, nn.t_own.data());
        if (s != da_status_success) return s;
    }
    return da_status_success;
}

// approximate_neighbors<T>::serialize (approximate_neighbors.cpp:1346-1395)
template <typename T> da_status load_ivf(RefStream &r, IVF<T> &ivf) {
    (void)r.b(); // train_data_is_set
    const bool trained = r.b(), added = r.b();
    (void)r.i64(); // n_neighbors
    const int64_t algo = r.i64();
    (void)r.i64(); // internal_algo
    (void)r.i64(); // internal_metric
    const int64_t metric = r.i64();
    const int64_t iseed = r.i64();
    (void)r.i64(); // seed
    (void)r.i64(); // n_samples_train
    const int64_t ord = r.i64();
    (void)r.i64(); // n_samples
    const int64_t d = r.i64();
    (void)r.real<T>(); // train_fraction
    const int64_t nl = r.i64();
    (void)r.i64(); // n_probe
    (void)r.i64(); // max_iter
    const int64_t kit = r.i64();
    (void)r.i64();     // n_init
    (void)r.real<T>(); // kmeans_tol
    const std::vector<T> cen = r.vec<T>();
    const int64_t ldc = r.i64();
    const int64_t ni = r.i64();
    std::vector<std::vector<T>> rows = r.vvec<T>();
    const std::vector<std::vector<int64_t>> ids = r.vvec<int64_t>();
    const std::vector<int64_t> sizes = r.ivec();
    (void)r.ivec(); // old_list_sizes
    std::vector<std::vector<T>> norms = r.vvec<T>();
    const int64_t imax = std::numeric_limits<da_int>::max();
    if (!r.ok || !trained || (ord != kRowMajor && ord != kColumnMajor) || nl < 1 || d < 1 ||
        nl > imax || d > imax || ni < 0 || ni > imax || metric < 0 || metric > 3 ||
        cen.size() / (size_t)nl != (size_t)d || cen.size() != (size_t)nl * (size_t)d ||
        rows.size() != (size_t)nl || ids.size() != (size_t)nl || sizes.size() != (size_t)nl ||
        (ord == kColumnMajor ? ldc < nl : ldc < d))
        return da_status_invalid_file_data;
    int64_t total = 0;
    for (int64_t c = 0; c < nl; ++c) {
        const int64_t m = sizes[c];
        if (m < 0 || ids[c].size() != (size_t)m || rows[c].size() / (size_t)d != (size_t)m ||
            rows[c].size() != (size_t)m * (size_t)d ||
            (c < (int64_t)norms.size() && !norms[c].empty() && norms[c].size() != (size_t)m))
            return da_status_invalid_file_data;
        for (int64_t v : ids[c])
            if (v < 0 || v >= ni) return da_status_invalid_file_data;
        total += m;
    }
    if (total > ni) return da_status_invalid_file_data;
    ivf.n_list = (da_int)nl;
    ivf.n_features = (da_int)d;
    ivf.n_index = (da_int)ni;
    ivf.kmeans_iter = (da_int)kit;
    ivf.internal_seed = (da_int)iseed;
    ivf.algo = (da_int)algo;
    ivf.metric = (da_int)metric;
    ivf.data_order = ord == kRowMajor ? row_major : column_major;
    ivf.data_added = added;
    // centroids in the storage order with leading dimension ldc -> row-major
    ivf.centroids.assign((size_t)nl * d, T(0));
    for (int64_t c = 0; c < nl; ++c)
        for (int64_t j = 0; j < d; ++j)
            ivf.centroids[(size_t)c * d + j] =
                ord == kColumnMajor ? cen[(size_t)c + (size_t)j * ldc] : cen[(size_t)c * ldc + j];
    ivf.list_sizes.assign((size_t)nl, 0);
    ivf.list_rows.assign((size_t)nl, {});
    ivf.list_norms.assign((size_t)nl, {});
    ivf.list_ids.assign((size_t)nl, {});
    for (int64_t c = 0; c < nl; ++c) {
        const size_t m = (size_t)sizes[c];
        ivf.list_sizes[c] = (da_int)m;
        ivf.list_rows[c] = std::move(rows[c]);
        ivf.list_ids[c].assign(ids[c].begin(), ids[c].end());
        if (c < (int64_t)norms.size() && norms[c].size() == m) {
            ivf.list_norms[c] = std::move(norms[c]);
        } else { // squared norms (the inner-product and cosine indexes keep none)
            ivf.list_norms[c].assign(m, T(0));
            for (size_t i = 0; i < m; ++i)
                for (int64_t j = 0; j < d; ++j) {
                    const T v = ivf.list_rows[c][i * d + j];
                    ivf.list_norms[c][i] += v * v;
                }
        }
    }
    ivf.train_data_set = false;
    ivf.lists_on_device = false;
    ivf.model_trained = true;
    return ivf.make_coarse();
}

template <typename T> da_status load_alg(RefStream &r, da_handle_type type, AlgBase *alg) {
    da_status s = load_registry<T>(r, type, alg->opts);
    if (s != da_status_success) return s;
    if (type == da_handle_kmeans) {
        auto *km = dynamic_cast<KMeans<T> *>(alg);
        return km ? load_kmeans<T>(r, *km) : da_status_internal_error;
    }
    if (type == da_handle_nn) {
        auto *nn = dynamic_cast<NN<T> *>(alg);
        return nn ? load_nn<T>(r, *nn) : da_status_internal_error;
    }
    auto *ivf = dynamic_cast<IVF<T> *>(alg);
    return ivf ? load_ivf<T>(r, *ivf) : da_status_internal_error;
}

} // namespace

bool is_reference_model(const char *p, size_t n) {
    const size_t kl = sizeof(kRefKeyword) - 1;
    if (n < 8 + kl) return false;
    int64_t len;
    std::memcpy(&len, p, 8);
    return len == (int64_t)kl && std::memcmp(p + 8, kRefKeyword, kl) == 0;
}

// _da_handle::load_handle with deserialize_metadata and basic_handle::
// load_model: da_status_version_mismatch for a version other than the
// reference's 50301 (an older one is also refused by the reference),
// da_status_invalid_file_data for a bad keyword, da_int size, precision or
// field, da_status_not_implemented for a handle type outside this library.
da_status load_reference_model(const char *p, size_t n, da_handle *out,
                               da_status (*handle_init)(da_handle *, da_handle_type,
                                                        da_precision)) {
    RefStream r{p, n};
    const std::string kw = r.str();
    const int64_t int_size = r.i64(), version = r.i64(), type = r.i64(), prec = r.i64();
    (void)r.str(); // the writer's AOCL-DA version
    if (!r.ok || kw != kRefKeyword) return da_status_invalid_file_data;
    if (version != kRefVersion) return da_status_version_mismatch;
    if ((int_size != 4 && int_size != 8) || (prec != 4 && prec != 8))
        return da_status_invalid_file_data;
    if (type != da_handle_kmeans && type != da_handle_nn && type != da_handle_approx_nn)
        return da_status_not_implemented;
    da_handle h = nullptr;
    da_status s = handle_init(&h, (da_handle_type)type, prec == 4 ? da_single : da_double);
    if (s != da_status_success) return s;
    s = prec == 4 ? load_alg<float>(r, (da_handle_type)type, h->alg.get())
                  : load_alg<double>(r, (da_handle_type)type, h->alg.get());
    if (s != da_status_success) {
        delete h;
        return s;
    }
    *out = h;
    return da_status_success;
}

} // namespace b200
