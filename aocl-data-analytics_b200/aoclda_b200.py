"""ctypes binding of libaoclda_b200.so (the C ABI declared in include/aoclda_b200.h).

This is the Python-side view of the drop-in boundary: every call goes through
the exported ``da_*`` C symbols with host numpy buffers, exactly as a C caller
of AOCL-DA would make them.  There is no fallback: if the shared library is not
built, importing this module raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaoclda_b200.so")

# status codes (aoclda_error.h)
SUCCESS = 0
STATUS = {
    0: "success", 1: "internal_error", 2: "memory_error", 3: "invalid_pointer",
    4: "invalid_input", 5: "not_implemented", 7: "wrong_type", 9: "invalid_handle_type",
    10: "handle_not_initialized", 13: "incompatible_options", 14: "operation_failed",
    15: "invalid_leading_dimension",
    17: "invalid_array_dimension", 18: "unknown_query", 20: "no_data", 21: "maxit",
    25: "arch_not_supported", 400: "option_not_found", 401: "option_locked",
    402: "option_wrong_type", 403: "option_invalid_bounds", 404: "option_invalid_value",
    700: "outlier_warning", 900: "empty_clusters",
}
# handle types (aoclda_handle.h)
HANDLE_KMEANS = 3
HANDLE_NN = 8
HANDLE_APPROX_NN = 11
# results (aoclda_result.h)
RINFO = 1
TRAINED = 2
KMEANS_CENTRES = 501
KMEANS_LABELS = 502
RNN_COUNT, RNN_OFFSETS, RNN_INDICES, RNN_DISTANCES = 601, 602, 603, 604
RNN_INDICES_INDEX, RNN_DISTANCES_INDEX = 605, 606
KNN_SEARCH, RADIUS_SEARCH = 0, 1  # da_nn_search_mode
OUTLIER_WARNING = 700
APPROX_NN_CENTROIDS, APPROX_NN_LIST_SIZES = 801, 802
# metrics (aoclda_metrics.h)
METRICS = {"euclidean": 0, "sqeuclidean": 1, "minkowski": 2, "manhattan": 3, "cosine": 4,
           "euclidean_gemm": 5, "sqeuclidean_gemm": 6, "inner product": 7}
ROW_MAJOR, COLUMN_MAJOR = 0, 1

da_int = C.c_int32
_P = C.c_void_p


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is not built; run `make -C aocl-data-analytics_b200` (there is no CPU path)")
    lib = C.CDLL(path)
    h = C.POINTER(_P)
    sig = {
        "da_handle_init_d": (h, C.c_int), "da_handle_init_s": (h, C.c_int),
        "da_options_set_int": (_P, C.c_char_p, da_int),
        "da_options_set_string": (_P, C.c_char_p, C.c_char_p),
        "da_options_set_real_s": (_P, C.c_char_p, C.c_float),
        "da_options_set_real_d": (_P, C.c_char_p, C.c_double),
        "da_options_get_int": (_P, C.c_char_p, C.POINTER(da_int)),
        "da_options_get_real_s": (_P, C.c_char_p, C.POINTER(C.c_float)),
        "da_options_get_real_d": (_P, C.c_char_p, C.POINTER(C.c_double)),
        "da_options_get_string": (_P, C.c_char_p, C.c_char_p, C.POINTER(da_int)),
        "da_options_get_string_key": (_P, C.c_char_p, C.c_char_p, C.POINTER(da_int),
                                      C.POINTER(da_int)),
        "da_handle_get_error_severity": (_P, C.POINTER(C.c_int)),
        "da_handle_get_error_message": (_P, C.POINTER(C.c_void_p)),
        "da_handle_get_result_d": (_P, C.c_int, C.POINTER(da_int), _P),
        "da_handle_get_result_s": (_P, C.c_int, C.POINTER(da_int), _P),
        "da_handle_get_result_int": (_P, C.c_int, C.POINTER(da_int), _P),
        "da_nn_set_data_d": (_P, da_int, da_int, _P, da_int),
        "da_nn_set_data_s": (_P, da_int, da_int, _P, da_int),
        "da_nn_set_labels_d": (_P, da_int, _P), "da_nn_set_labels_s": (_P, da_int, _P),
        "da_nn_set_targets_d": (_P, da_int, _P), "da_nn_set_targets_s": (_P, da_int, _P),
        "da_nn_kneighbors_d": (_P, da_int, da_int, _P, da_int, _P, _P, da_int, da_int),
        "da_nn_kneighbors_s": (_P, da_int, da_int, _P, da_int, _P, _P, da_int, da_int),
        "da_nn_radius_neighbors_d": (_P, da_int, da_int, _P, da_int, C.c_double, da_int, da_int),
        "da_nn_radius_neighbors_s": (_P, da_int, da_int, _P, da_int, C.c_float, da_int, da_int),
        "da_approx_nn_set_training_data_d": (_P, da_int, da_int, _P, da_int),
        "da_approx_nn_set_training_data_s": (_P, da_int, da_int, _P, da_int),
        "da_approx_nn_train_d": (_P,), "da_approx_nn_train_s": (_P,),
        "da_approx_nn_add_d": (_P, da_int, da_int, _P, da_int),
        "da_approx_nn_add_s": (_P, da_int, da_int, _P, da_int),
        "da_approx_nn_train_and_add_d": (_P,), "da_approx_nn_train_and_add_s": (_P,),
        "da_approx_nn_kneighbors_d": (_P, da_int, da_int, _P, da_int, _P, _P, da_int, da_int),
        "da_approx_nn_kneighbors_s": (_P, da_int, da_int, _P, da_int, _P, _P, da_int, da_int),
        "da_nn_classes_d": (_P, C.POINTER(da_int), _P), "da_nn_classes_s": (_P, C.POINTER(da_int), _P),
        "da_nn_classifier_predict_proba_d": (_P, da_int, da_int, _P, da_int, _P, C.c_int),
        "da_nn_classifier_predict_proba_s": (_P, da_int, da_int, _P, da_int, _P, C.c_int),
        "da_nn_classifier_predict_d": (_P, da_int, da_int, _P, da_int, _P, C.c_int),
        "da_nn_classifier_predict_s": (_P, da_int, da_int, _P, da_int, _P, C.c_int),
        "da_nn_regressor_predict_d": (_P, da_int, da_int, _P, da_int, _P, C.c_int),
        "da_nn_regressor_predict_s": (_P, da_int, da_int, _P, da_int, _P, C.c_int),
        "da_kmeans_set_data_d": (_P, da_int, da_int, _P, da_int),
        "da_kmeans_set_data_s": (_P, da_int, da_int, _P, da_int),
        "da_kmeans_set_init_centres_d": (_P, _P, da_int),
        "da_kmeans_set_init_centres_s": (_P, _P, da_int),
        "da_kmeans_compute_d": (_P,), "da_kmeans_compute_s": (_P,),
        "da_kmeans_predict_d": (_P, da_int, da_int, _P, da_int, _P),
        "da_kmeans_predict_s": (_P, da_int, da_int, _P, da_int, _P),
        "da_kmeans_transform_d": (_P, da_int, da_int, _P, da_int, _P, da_int),
        "da_kmeans_transform_s": (_P, da_int, da_int, _P, da_int, _P, da_int),
        "da_pairwise_distances_d": (C.c_int, da_int, da_int, da_int, _P, da_int, _P, da_int, _P,
                                    da_int, C.c_double, C.c_int),
        "da_pairwise_distances_s": (C.c_int, da_int, da_int, da_int, _P, da_int, _P, da_int, _P,
                                    da_int, C.c_float, C.c_int),
    }
    sig.update({
        "da_b200_set_stream": (_P, _P),
        "da_b200_set_stream_priority": (_P, da_int),
        "da_b200_set_kernel_timing": (_P, da_int),
        "da_b200_get_kernel_time": (_P, C.c_char_p, C.POINTER(C.c_double), C.POINTER(da_int)),
        "da_b200_reset_kernel_time": (_P,),
        "da_b200_get_stat": (_P, C.c_char_p, C.POINTER(C.c_double)),
        "da_b200_kmeans_init_centres_d": (_P, _P, da_int),
        "da_b200_kmeans_init_centres_s": (_P, _P, da_int),
        "da_handle_save_model": (_P, C.c_char_p),
        "da_handle_load_model": (h, C.c_char_p),
        "da_b200_kmeans_shard_colmax_s": (_P, _P),
        "da_b200_kmeans_shard_begin_s": (_P, _P, da_int, _P),
        "da_b200_kmeans_shard_partial_s": (_P, _P),
        "da_b200_kmeans_shard_finalize_s": (_P, _P, _P, _P),
        "da_b200_kmeans_shard_inertia_s": (_P, da_int, C.POINTER(C.c_double)),
        "da_b200_kmeans_shard_result_s": (_P, _P, _P),
        "da_b200_nn_share_data": (_P, _P),
    })
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = list(args)
        f.restype = C.c_int
    lib.da_handle_destroy.argtypes = [h]
    lib.da_handle_destroy.restype = None
    lib.da_handle_refresh.argtypes = [_P]
    lib.da_handle_refresh.restype = None
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class DAError(RuntimeError):
    def __init__(self, status, where, message=""):
        super().__init__(f"{where}: status {status} ({STATUS.get(status, '?')}) {message}")
        self.status = status


class Handle:
    """A da_handle of one precision ('d' or 's') and one type (HANDLE_NN / HANDLE_KMEANS /
    HANDLE_APPROX_NN)."""

    def __init__(self, htype, prec="d"):
        self.L = lib()
        self.prec = prec
        self.dtype = np.float64 if prec == "d" else np.float32
        self.h = C.c_void_p()
        st = getattr(self.L, f"da_handle_init_{prec}")(C.byref(self.h), htype)
        if st != SUCCESS:
            raise DAError(st, "da_handle_init")

    def close(self):
        if self.h:
            self.L.da_handle_destroy(C.byref(self.h))

    def save_model(self, path):
        """da_handle_save_model: options and trained state to a file."""
        return self.call("da_handle_save_model", str(path).encode())

    @classmethod
    def load_model(cls, path, prec):
        """da_handle_load_model into a new object of this class; `prec` ("s"
        or "d") must be the precision the model was saved with."""
        L = lib()
        h = C.c_void_p()
        st = L.da_handle_load_model(C.byref(h), str(path).encode())
        if st != SUCCESS:
            raise DAError(st, "da_handle_load_model")
        obj = cls.__new__(cls)
        obj.L, obj.h, obj.prec = L, h, prec
        obj.dtype = np.float64 if prec == "d" else np.float32
        obj.order = ROW_MAJOR if obj.get_string("storage order") == "row-major" else COLUMN_MAJOR
        return obj

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream_priority(self, priority):
        """da_b200_set_stream_priority: the handle's own stream recreated with
        this CUDA priority (negative: higher)."""
        self.call("da_b200_set_stream_priority", int(priority))
        return self

    def kernel_time(self, name):
        ms = C.c_double()
        n = da_int()
        self.L.da_b200_get_kernel_time(self.h, name.encode(), C.byref(ms), C.byref(n))
        return ms.value, n.value

    def stat(self, name):
        v = C.c_double()
        self.L.da_b200_get_stat(self.h, name.encode(), C.byref(v))
        return v.value

    def message(self):
        p = C.c_void_p()
        self.L.da_handle_get_error_message(self.h, C.byref(p))
        if not p.value:
            return ""
        s = C.string_at(p.value).decode()
        C.CDLL(None).free(p)
        return s

    def call(self, name, *args, ok=(SUCCESS,)):
        st = getattr(self.L, name)(self.h, *args)
        if st not in ok:
            raise DAError(st, name, self.message())
        return st

    # options
    def set(self, name, value):
        if isinstance(value, str):
            return self.L.da_options_set_string(self.h, name.encode(), value.encode())
        if isinstance(value, (int, np.integer)):
            return self.L.da_options_set_int(self.h, name.encode(), int(value))
        return getattr(self.L, f"da_options_set_real_{self.prec}")(self.h, name.encode(), value)

    def get_string(self, name):
        buf = C.create_string_buffer(64)
        n = da_int(64)
        st = self.L.da_options_get_string(self.h, name.encode(), buf, C.byref(n))
        if st != SUCCESS:
            raise DAError(st, "da_options_get_string")
        return buf.value.decode()

    def get_int(self, name):
        v = da_int()
        st = self.L.da_options_get_int(self.h, name.encode(), C.byref(v))
        if st != SUCCESS:
            raise DAError(st, "da_options_get_int")
        return v.value


def _as(a, dtype, order):
    a = np.asarray(a, dtype=dtype)
    return np.asfortranarray(a) if order == COLUMN_MAJOR else np.ascontiguousarray(a)


def _ld(a, order):
    return a.shape[0] if order == COLUMN_MAJOR else a.shape[1]


class KNN(Handle):
    """Brute-force kNN through da_nn_* (host arrays, C-ABI calls)."""

    def __init__(self, prec="d", order=COLUMN_MAJOR, **options):
        super().__init__(HANDLE_NN, prec)
        self.order = order
        if order == ROW_MAJOR:
            self.set("storage order", "row-major")
        for k, v in options.items():
            st = self.set(k.replace("_", " "), v)
            if st != SUCCESS:
                raise DAError(st, f"option {k}")

    def fit(self, X, y=None, targets=None):
        self.X = _as(X, self.dtype, self.order)
        n, d = self.X.shape
        self.call(f"da_nn_set_data_{self.prec}", n, d, ptr(self.X), _ld(self.X, self.order))
        if y is not None:
            self.y = np.ascontiguousarray(y, dtype=np.int32)
            self.call(f"da_nn_set_labels_{self.prec}", n, ptr(self.y))
        if targets is not None:
            self.t = np.ascontiguousarray(targets, dtype=self.dtype)
            self.call(f"da_nn_set_targets_{self.prec}", n, ptr(self.t))
        return self

    def share(self, source):
        """da_b200_nn_share_data: the training data of the fitted handle
        `source`, held on the device once for both handles."""
        self.call("da_b200_nn_share_data", source.h)
        # the host arrays the handles point at live as long as either
        for a in ("X", "y", "t"):
            if hasattr(source, a):
                setattr(self, a, getattr(source, a))
        return self

    def kneighbors(self, Q, k, return_distance=True):
        Q = _as(Q, self.dtype, self.order)
        nq, d = Q.shape
        shape = (nq, k)
        ind = np.zeros(shape, dtype=np.int32, order="F" if self.order == COLUMN_MAJOR else "C")
        dist = np.zeros(shape, dtype=self.dtype, order="F" if self.order == COLUMN_MAJOR else "C")
        self.call(f"da_nn_kneighbors_{self.prec}", nq, d, ptr(Q), _ld(Q, self.order), ptr(ind),
                  ptr(dist) if return_distance else None, k, int(return_distance))
        return ind, dist

    def radius_neighbors(self, Q, radius, return_distance=True, sort_results=False):
        """da_nn_radius_neighbors: returns (count[n_q + 1], offsets[n_q + 1],
        indices, distances or None) from the result queries."""
        Q = _as(Q, self.dtype, self.order)
        nq, d = Q.shape
        self.call(f"da_nn_radius_neighbors_{self.prec}", nq, d, ptr(Q), _ld(Q, self.order), radius,
                  int(return_distance), int(sort_results))
        cnt = self.result_int(RNN_COUNT, nq + 1)
        off = self.result_int(RNN_OFFSETS, nq + 1)
        total = int(cnt[nq])
        ind = self.result_int(RNN_INDICES, max(total, 1))[:total]
        dist = None
        if return_distance:
            out = np.zeros(max(total, 1), dtype=self.dtype)
            dim = da_int(out.size)
            self.call(f"da_handle_get_result_{self.prec}", RNN_DISTANCES, C.byref(dim), ptr(out))
            dist = out[:total]
        return cnt, off, ind, dist

    def result_int(self, query, size):
        out = np.zeros(size, dtype=np.int32)
        dim = da_int(size)
        self.call("da_handle_get_result_int", query, C.byref(dim), ptr(out))
        return out

    def classes(self):
        n = da_int(0)
        self.call(f"da_nn_classes_{self.prec}", C.byref(n), None)
        out = np.zeros(n.value, dtype=np.int32)
        self.call(f"da_nn_classes_{self.prec}", C.byref(n), ptr(out))
        return out

    # predict_proba / predict / predict_reg: `mode` is KNN_SEARCH (the
    # "number of neighbors" nearest rows) or RADIUS_SEARCH (the rows within
    # the "radius" option); status 700 (outlier warning) is kept in
    # self.last_status with the results

    def predict_proba(self, Q, mode=KNN_SEARCH):
        Q = _as(Q, self.dtype, self.order)
        nq, d = Q.shape
        nc = len(self.classes())
        pr = np.zeros((nq, nc), dtype=self.dtype, order="F" if self.order == COLUMN_MAJOR else "C")
        self.last_status = self.call(f"da_nn_classifier_predict_proba_{self.prec}", nq, d, ptr(Q),
                                     _ld(Q, self.order), ptr(pr), mode,
                                     ok=(SUCCESS, OUTLIER_WARNING))
        return pr

    def predict(self, Q, mode=KNN_SEARCH):
        Q = _as(Q, self.dtype, self.order)
        nq, d = Q.shape
        y = np.zeros(nq, dtype=np.int32)
        self.last_status = self.call(f"da_nn_classifier_predict_{self.prec}", nq, d, ptr(Q),
                                     _ld(Q, self.order), ptr(y), mode,
                                     ok=(SUCCESS, OUTLIER_WARNING))
        return y

    def predict_reg(self, Q, mode=KNN_SEARCH):
        Q = _as(Q, self.dtype, self.order)
        nq, d = Q.shape
        y = np.zeros(nq, dtype=self.dtype)
        self.last_status = self.call(f"da_nn_regressor_predict_{self.prec}", nq, d, ptr(Q),
                                     _ld(Q, self.order), ptr(y), mode,
                                     ok=(SUCCESS, OUTLIER_WARNING))
        return y


class ApproxNN(Handle):
    """IVF-flat approximate neighbours through da_approx_nn_* (host arrays,
    C-ABI calls)."""

    def __init__(self, prec="d", order=COLUMN_MAJOR, **options):
        super().__init__(HANDLE_APPROX_NN, prec)
        self.order = order
        if order == ROW_MAJOR:
            self.set("storage order", "row-major")
        # option names: "n_list", "n_probe", "k-means_iter", "seed", "metric",
        # "algorithm" as they are; number_of_neighbors / train_fraction spelled
        # with underscores for keyword use
        names = {"number_of_neighbors": "number of neighbors", "train_fraction": "train fraction",
                 "kmeans_iter": "k-means_iter"}
        for k, v in options.items():
            st = self.set(names.get(k, k), v)
            if st != SUCCESS:
                raise DAError(st, f"option {k}")

    def set_training_data(self, X):
        self.X = _as(X, self.dtype, self.order)
        n, d = self.X.shape
        self.call(f"da_approx_nn_set_training_data_{self.prec}", n, d, ptr(self.X),
                  _ld(self.X, self.order))
        return self

    def train(self):
        self.call(f"da_approx_nn_train_{self.prec}")
        return self

    def add(self, X):
        A = _as(X, self.dtype, self.order)  # the index keeps its own copy of the rows
        n, d = A.shape
        self.call(f"da_approx_nn_add_{self.prec}", n, d, ptr(A), _ld(A, self.order))
        return self

    def train_and_add(self):
        self.call(f"da_approx_nn_train_and_add_{self.prec}")
        return self

    def kneighbors(self, Q, k, return_distance=True):
        Q = _as(Q, self.dtype, self.order)
        nq, d = Q.shape
        o = "F" if self.order == COLUMN_MAJOR else "C"
        ind = np.zeros((nq, k), dtype=np.int32, order=o)
        dist = np.zeros((nq, k), dtype=self.dtype, order=o)
        self.call(f"da_approx_nn_kneighbors_{self.prec}", nq, d, ptr(Q), _ld(Q, self.order),
                  ptr(ind), ptr(dist) if return_distance else None, k, int(return_distance))
        return ind, (dist if return_distance else None)

    def result(self, query, size):
        out = np.zeros(size, dtype=self.dtype)
        dim = da_int(size)
        self.call(f"da_handle_get_result_{self.prec}", query, C.byref(dim), ptr(out))
        return out

    def list_sizes(self, n_list):
        out = np.zeros(n_list, dtype=np.int32)
        dim = da_int(n_list)
        self.call("da_handle_get_result_int", APPROX_NN_LIST_SIZES, C.byref(dim), ptr(out))
        return out


class KMeans(Handle):
    """k-means through da_kmeans_* (host arrays, C-ABI calls)."""

    def __init__(self, n_clusters, prec="d", order=COLUMN_MAJOR, **options):
        super().__init__(HANDLE_KMEANS, prec)
        self.order = order
        if order == ROW_MAJOR:
            self.set("storage order", "row-major")
        st = self.set("n_clusters", int(n_clusters))
        if st != SUCCESS:
            raise DAError(st, "n_clusters")
        for k, v in options.items():
            st = self.set(k.replace("_", " ") if k not in ("n_init", "max_iter") else k, v)
            if st != SUCCESS:
                raise DAError(st, f"option {k}")

    def fit(self, A, C0=None, ok=(SUCCESS, 21)):
        self.A = _as(A, self.dtype, self.order)
        n, d = self.A.shape
        self.call(f"da_kmeans_set_data_{self.prec}", n, d, ptr(self.A), _ld(self.A, self.order),
                  ok=(SUCCESS, 13))
        if C0 is not None:
            self.C0 = _as(C0, self.dtype, self.order)
            self.set("initialization method", "supplied")
            self.call(f"da_kmeans_set_init_centres_{self.prec}", ptr(self.C0),
                      _ld(self.C0, self.order))
        self.status = self.call(f"da_kmeans_compute_{self.prec}", ok=ok)
        return self

    def result(self, query, size, dtype=None):
        dtype = dtype or self.dtype
        out = np.zeros(size, dtype=dtype)
        dim = da_int(size)
        fn = "da_handle_get_result_int" if dtype == np.int32 else f"da_handle_get_result_{self.prec}"
        self.call(fn, query, C.byref(dim), ptr(out))
        return out

    def set_data(self, A):
        """da_kmeans_set_data only (the caller keeps A alive)."""
        self.A = _as(A, self.dtype, self.order)
        n, d = self.A.shape
        return self.call(f"da_kmeans_set_data_{self.prec}", n, d, ptr(self.A),
                         _ld(self.A, self.order), ok=(SUCCESS, 13))

    def init_centres(self, k):
        n, d = self.A.shape
        out = np.zeros((k, d), dtype=self.dtype, order="F" if self.order == COLUMN_MAJOR else "C")
        self.call(f"da_b200_kmeans_init_centres_{self.prec}", ptr(out),
                  k if self.order == COLUMN_MAJOR else d)
        return out

    def rinfo(self):
        return self.result(RINFO, 6)

    def centres(self, k, d):
        flat = self.result(KMEANS_CENTRES, k * d)
        return flat.reshape((k, d), order="F" if self.order == COLUMN_MAJOR else "C")

    def labels(self, n):
        return self.result(KMEANS_LABELS, n, np.int32)

    def predict(self, Y):
        Y = _as(Y, self.dtype, self.order)
        m, d = Y.shape
        lab = np.zeros(m, dtype=np.int32)
        self.call(f"da_kmeans_predict_{self.prec}", m, d, ptr(Y), _ld(Y, self.order), ptr(lab))
        return lab

    def transform(self, X, k):
        X = _as(X, self.dtype, self.order)
        m, d = X.shape
        out = np.zeros((m, k), dtype=self.dtype, order="F" if self.order == COLUMN_MAJOR else "C")
        self.call(f"da_kmeans_transform_{self.prec}", m, d, ptr(X), _ld(X, self.order), ptr(out),
                  m if self.order == COLUMN_MAJOR else k)
        return out


def pairwise_distances(X, Y=None, metric="euclidean", p=2.0, prec="d", order=COLUMN_MAJOR):
    """da_pairwise_distances_{d,s}: returns (status, D)."""
    L = lib()
    dt = np.float64 if prec == "d" else np.float32
    X = _as(X, dt, order)
    m, k = X.shape
    if Y is not None:
        Y = _as(Y, dt, order)
        n = Y.shape[0]
    else:
        n = m
    D = np.zeros((m, n), dtype=dt, order="F" if order == COLUMN_MAJOR else "C")
    ldd = m if order == COLUMN_MAJOR else n
    st = getattr(L, f"da_pairwise_distances_{prec}")(
        order, m, n, k, ptr(X), _ld(X, order), ptr(Y), _ld(Y, order) if Y is not None else 0,
        ptr(D), ldd, p, METRICS[metric])
    return st, D


def kmeans_batched(Xs, C0s, max_iter=300, tol=1e-4):
    """da_b200_kmeans_batched_s over lists of fp32 data sets and initial
    centres (row-major); returns a list of dicts with centres, labels,
    n_iter, inertia and converged for every data set."""
    L = lib()
    m = len(Xs)
    Xs = [np.ascontiguousarray(x, dtype=np.float32) for x in Xs]
    C0s = [np.ascontiguousarray(c, dtype=np.float32) for c in C0s]
    ns = (da_int * m)(*[x.shape[0] for x in Xs])
    ds = (da_int * m)(*[x.shape[1] for x in Xs])
    ks = (da_int * m)(*[c.shape[0] for c in C0s])
    lds = (da_int * m)(*[x.shape[1] for x in Xs])
    fp = C.POINTER(C.c_float)
    A = (fp * m)(*[x.ctypes.data_as(fp) for x in Xs])
    C0 = (fp * m)(*[c.ctypes.data_as(fp) for c in C0s])
    outs = [np.zeros_like(c) for c in C0s]
    labs = [np.zeros(x.shape[0], dtype=np.int32) for x in Xs]
    CO = (fp * m)(*[o.ctypes.data_as(fp) for o in outs])
    ip = C.POINTER(da_int)
    LO = (ip * m)(*[l.ctypes.data_as(ip) for l in labs])
    nit = (da_int * m)()
    inert = (C.c_double * m)()
    conv = (da_int * m)()
    st = L.da_b200_kmeans_batched_s(m, ns, ds, ks, A, lds, C0, max_iter, C.c_double(tol), CO, LO,
                                    nit, inert, conv, None)
    if st != SUCCESS:
        raise DAError(st, "da_b200_kmeans_batched_s")
    return [{"centres": outs[i], "labels": labs[i], "n_iter": int(nit[i]),
             "inertia": float(inert[i]), "converged": int(conv[i])} for i in range(m)]


def device_memory():
    """da_b200_device_memory: (free, total) bytes of the current device."""
    L = lib()
    f, t = C.c_ulonglong(), C.c_ulonglong()
    st = L.da_b200_device_memory(C.byref(f), C.byref(t))
    if st != SUCCESS:
        raise DAError(st, "da_b200_device_memory")
    return f.value, t.value


def kmeans_batched_timing():
    """da_b200_kmeans_batched_timing: (upload, fit, download) device
    milliseconds of this thread's last kmeans_batched call."""
    L = lib()
    v = [C.c_double() for _ in range(3)]
    st = L.da_b200_kmeans_batched_timing(*[C.byref(x) for x in v])
    if st != SUCCESS:
        raise DAError(st, "da_b200_kmeans_batched_timing")
    return tuple(x.value for x in v)

