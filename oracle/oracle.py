"""ctypes wrapper of liboracle.so, the CPU restatement of the reference path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, to check results and to time the
CPU algorithm.  The product never
imports it.  Each wrapped function cites the AOCL-DA source it restates in
oracle.c.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

METRICS = {"euclidean": 0, "sqeuclidean": 1, "minkowski": 2, "manhattan": 3, "cosine": 4,
           "euclidean_gemm": 5, "sqeuclidean_gemm": 6, "inner product": 7}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        P = C.c_void_p
        i = C.c_int
        for sfx, T in (("s", C.c_float), ("d", C.c_double)):
            f = getattr(_lib, f"orc_pairwise_{sfx}")
            f.argtypes = [i, i, i, P, P, P, T, i, i]
            f.restype = None
            f = getattr(_lib, f"orc_knn_{sfx}")
            f.argtypes = [i, i, P, i, P, i, i, T, i, P, P]
            f.restype = None
            f = getattr(_lib, f"orc_kmeans_assign_{sfx}")
            f.argtypes = [i, i, P, i, P, P, P]
            f.restype = None
            f = getattr(_lib, f"orc_kmeans_lloyd_{sfx}")
            f.argtypes = [i, i, P, i, P, i, C.c_double, P, P, P, P]
            f.restype = None
        _lib.orc_kmeans_update_d.argtypes = [i, i, P, P, i, P, P]
        _lib.orc_kmeans_update_d.restype = None
        _lib.orc_kmeans_inertia_d.argtypes = [i, i, P, P, P]
        _lib.orc_kmeans_inertia_d.restype = C.c_double
        _lib.orc_kmeans_iteration_s.argtypes = [i, i, P, i, P, P]
        _lib.orc_kmeans_iteration_s.restype = i
        _lib.orc_knn_reference_ties_d.argtypes = [i, P, i, P]
        _lib.orc_knn_reference_ties_d.restype = None
        _lib.orc_num_threads.restype = i
        _lib.orc_random_rows.argtypes = [i, i, C.c_longlong, P]
        _lib.orc_random_rows.restype = i
        for sfx in ("s", "d"):
            f = getattr(_lib, f"orc_kmeanspp_{sfx}")
            f.argtypes = [i, i, P, i, C.c_longlong, i, P, P]
            f.restype = i
            f = getattr(_lib, f"orc_kmeanspp_cos_{sfx}")
            f.argtypes = [i, i, P, i, C.c_longlong, i, P]
            f.restype = i
            f = getattr(_lib, f"orc_kmeans_assign_sph_{sfx}")
            f.argtypes = [i, i, P, i, P, P, P]
            f.restype = None
            f = getattr(_lib, f"orc_kmeans_inertia_sph_{sfx}")
            f.argtypes = [i, i, P, P, P, i]
            f.restype = C.c_double
            f = getattr(_lib, f"orc_kmeans_sph_lloyd_{sfx}")
            f.argtypes = [i, i, P, i, P, i, C.c_double, i, P, P, P, P]
            f.restype = None
        _lib.orc_lloyd_blas_s.argtypes = [i, i, P, i, P, P, i, P, i]
        _lib.orc_lloyd_blas_s.restype = i
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _sfx(dt):
    return "d" if np.dtype(dt) == np.float64 else "s"


def default_kc(dtype, isa="avx512"):
    """KC slice length of the reference's packed blocking
    (partitioning_infrastructure.hpp:45-59)."""
    f64 = np.dtype(dtype) == np.float64
    if isa == "avx2":
        return 32 if f64 else 64
    return 512 if f64 else 256


def pairwise(X, Y=None, metric="euclidean", p=2.0, kc=None):
    X = np.ascontiguousarray(X)
    dt = X.dtype
    Yc = None if Y is None else np.ascontiguousarray(Y, dtype=dt)
    m, d = X.shape
    n = m if Y is None else Yc.shape[0]
    D = np.zeros((m, n), dtype=dt)
    getattr(lib(), f"orc_pairwise_{_sfx(dt)}")(m, n, d, _p(X), _p(Yc), _p(D), p,
                                               METRICS[metric], kc or default_kc(dt))
    return D


def knn(X, Q, k, metric="euclidean", p=2.0, kc=None):
    """Exact top-k with ties to the lower index; returns (ind, dist) q-major."""
    X = np.ascontiguousarray(X)
    dt = X.dtype
    Q = np.ascontiguousarray(Q, dtype=dt)
    nx, d = X.shape
    nq = Q.shape[0]
    ind = np.zeros((nq, k), dtype=np.int32)
    dist = np.zeros((nq, k), dtype=dt)
    getattr(lib(), f"orc_knn_{_sfx(dt)}")(nx, d, _p(X), nq, _p(Q), k, METRICS[metric], p,
                                          kc or default_kc(dt), _p(ind), _p(dist))
    return ind, dist


def radius(X, Q, r, metric="euclidean", p=2.0, sort=False, kc=None):
    """Radius neighbours (nearest_neighbors.cpp:1915-2068, brute force
    :2070-2247): per query the training rows with distance <= r -- squared
    distances against r^2 for euclidean and minkowski p = 2 -- in index order,
    or (sort) stably sorted by that distance (nearest_neighbors_utils.hpp:
    73-101); distances returned with the square root taken for those metrics.
    Returns a list of (indices, distances) per query."""
    sq = metric == "euclidean" or (metric == "minkowski" and p == 2.0)
    inner = "sqeuclidean" if sq else metric
    D = pairwise(Q, X, inner, p, kc)
    thr = np.asarray(r * r if sq else r, dtype=D.dtype)
    out = []
    for row in D:
        idx = np.nonzero(row <= thr)[0]
        val = row[idx]
        if sort:
            o = np.argsort(val, kind="stable")
            idx, val = idx[o], val[o]
        out.append((idx.astype(np.int32), np.sqrt(val) if sq else val))
    return out


def _radius_weights(dist, weights, dt):
    """get_weights (nearest_neighbors.cpp:1021-1033): 1, or 1 / distance with
    1 at distance <= eps."""
    if weights == "uniform":
        return [dt.type(1)] * len(dist)
    eps = np.finfo(dt).eps
    return [dt.type(1) if v <= eps else dt.type(1) / v for v in dist]


def _most_frequent(y):
    """most_frequent_element (nearest_neighbors.cpp:1037-1058): ties to the
    smallest label."""
    vals, cnt = np.unique(np.asarray(y), return_counts=True)
    return int(vals[np.argmax(cnt)])


def radius_predict_proba(X, y, Q, r, metric="euclidean", p=2.0, weights="uniform",
                         outlier="none", outlier_label=0):
    """Radius-mode class probabilities (predict_proba_compute_rnn,
    nearest_neighbors.cpp:1280-1479): per query, per class (sorted labels),
    the weights of its radius neighbours in index order, divided by their sum
    over the classes.  Returns (proba[nq, nc], warning); raises
    LookupError(query) where the reference fails (outlier "none", a query
    without neighbours).  Under "manual" the outlier label's column gets 1
    (the reference indexes that row by the label's value, which coincides for
    labels 0..nc-1)."""
    dt = np.asarray(X).dtype
    classes = np.unique(np.asarray(y))
    nc = len(classes)
    pos = {int(c): i for i, c in enumerate(classes)}
    mf = _most_frequent(y) if outlier == "most frequent" else None
    mi = pos.get(int(outlier_label), -1)
    proba = np.zeros((len(Q), nc), dtype=dt)
    warn = False
    for q, (idx, dist) in enumerate(radius(X, Q, r, metric, p)):
        if len(idx) == 0:
            if outlier == "none":
                raise LookupError(q)
            if outlier == "manual":
                warn = True
                if mi != -1:
                    proba[q, mi] = 1
            else:
                proba[q, pos[mf]] = 1
            continue
        w = _radius_weights(dist, weights, dt)
        acc = [dt.type(0)] * nc
        for j, i in enumerate(idx):
            c = pos[int(y[i])]
            acc[c] = dt.type(acc[c] + w[j])
        den = dt.type(0)
        for c in range(nc):
            den = dt.type(den + acc[c])
        for c in range(nc):
            proba[q, c] = dt.type(acc[c] / den)
    return proba, warn and outlier == "manual" and mi == -1


def radius_predict(X, y, Q, r, metric="euclidean", p=2.0, weights="uniform", outlier="none",
                   outlier_label=0):
    """Radius-mode labels (nearest_neighbors.cpp:1540-1603): the first largest
    probability's class; with outlier handling an all-zero row takes the
    outlier label or the most frequent label."""
    proba, _ = radius_predict_proba(X, y, Q, r, metric, p, weights, outlier, outlier_label)
    classes = np.unique(np.asarray(y))
    best = np.argmax(np.abs(proba), axis=1)
    lab = classes[best].astype(np.int32)
    if outlier != "none":
        fill = outlier_label if outlier == "manual" else _most_frequent(y)
        lab[proba[np.arange(len(Q)), best] == 0] = fill
    return lab


def radius_predict_reg(X, t, Q, r, metric="euclidean", p=2.0, weights="uniform", outlier="none",
                       outlier_target=0.0):
    """Radius-mode regression (predict_targets_rnn, nearest_neighbors.cpp:
    1763-1909): the mean target of the radius neighbours, or their weighted
    mean; a query without neighbours takes the mean training target ("most
    frequent") or the outlier target ("manual"), or fails ("none": raises
    LookupError(query)).  Returns (y, warning)."""
    dt = np.asarray(X).dtype
    t = np.asarray(t, dtype=dt)
    out = np.zeros(len(Q), dtype=dt)
    warn = False
    for q, (idx, dist) in enumerate(radius(X, Q, r, metric, p)):
        if len(idx) == 0:
            if outlier == "none":
                raise LookupError(q)
            if outlier == "most frequent":
                out[q] = t.astype(np.float64).mean()
            else:
                warn = True
                out[q] = outlier_target
            continue
        w = _radius_weights(dist, weights, dt)
        num = den = dt.type(0)
        for j, i in enumerate(idx):
            num = dt.type(num + t[i] * w[j])
            den = dt.type(den + w[j])
        out[q] = num / den
    return out, warn


def _gemm_sq(A, B):
    """|a|^2 + |b|^2 - 2 a.b in fp64 (the GEMM form of the squared euclidean
    distance used throughout the IVF-flat index)."""
    A = np.asarray(A, dtype=np.float64)
    B = np.asarray(B, dtype=np.float64)
    return (A * A).sum(1)[:, None] + (B * B).sum(1)[None, :] - 2.0 * A @ B.T


SPHERICAL_METRICS = ("inner product", "cosine")


def _ivf_key(A, B, metric):
    """The IVF-flat ranking key: the GEMM-form squared distance, or -a.b for
    the inner-product and cosine metrics (the GEMMs with alpha = -1 of
    approximate_neighbors.cpp:712-727, 1094-1100, 1148-1154).  fp64."""
    if metric in SPHERICAL_METRICS:
        return -(np.asarray(A, dtype=np.float64) @ np.asarray(B, dtype=np.float64).T)
    return _gemm_sq(A, B)


def normalise_rows(X):
    """normalize_rows of utilities/da_utils.cpp:858-905 in the working
    precision: the row's sum of squares accumulated feature by feature
    (v * v rounded, then added), norm = sqrt, factor 1 / norm (1 for a zero
    row), every element times the factor."""
    X = np.asarray(X)
    dt = X.dtype.type
    s = np.zeros(X.shape[0], dtype=X.dtype)
    for f in range(X.shape[1]):
        s = s + X[:, f] * X[:, f]
    nrm = np.sqrt(s)
    inv = np.where(nrm == 0, dt(1), dt(1) / np.where(nrm == 0, dt(1), nrm)).astype(X.dtype)
    return (X * inv[:, None]).astype(X.dtype)


def random_rows(n, k, seed):
    """The random-samples initial rows of k-means (oracle_kpp.cpp)."""
    out = np.zeros(min(k, n), dtype=np.int32)
    lib().orc_random_rows(n, k, int(seed), _p(out))
    return out


def ivf_train_spherical(X, n_list, seed, max_iter, metric):
    """The coarse quantiser of the inner-product / cosine index
    (approximate_neighbors.cpp:368-478): the training rows (normalised for
    cosine), random-samples initial centres, spherical Lloyd on the rows as
    given ("normalize data" off), tolerance sqrt(eps).  Returns the
    centroids (n_list x d)."""
    X = np.ascontiguousarray(X)
    Xt = normalise_rows(X) if metric == "cosine" else X
    C0 = Xt[random_rows(len(X), n_list, seed)]
    tol = float(np.sqrt(np.finfo(X.dtype).eps))
    C, _, _, _ = kmeans_sph_lloyd(Xt, C0, max_iter, tol, normalise=False)
    return C


def ivf_lists(C, X, metric="sqeuclidean"):
    """add_ivfflat (approximate_neighbors.cpp:565-842): every row joins the
    list of its nearest centroid (first minimum), after the rows already
    there.  Returns the list of every row (X normalised by the caller for
    cosine)."""
    return np.argmin(_ivf_key(X, C, metric), axis=1).astype(np.int32)


def ivf_kneighbors(C, X, Q, k, n_probe, metric="sqeuclidean", lists=None):
    """IVF-flat search (approximate_neighbors.cpp:971-1344): per query the
    n_probe nearest centroids (lower index on ties), then the k nearest index
    rows of those lists in (key, index) order; index -1 / distance +inf
    (-inf for the inner product) where the lists hold fewer than k rows;
    euclidean returns the square root of non-negative values, inner product
    the dot (-key), cosine 1 + key (X and Q normalised by the caller for
    cosine).  Distances in fp64.
    Returns (ind, dist, probes), q-major."""
    lists = ivf_lists(C, X, metric) if lists is None else lists
    dc = _ivf_key(Q, C, metric)
    nq = len(Q)
    ind = np.full((nq, k), -1, dtype=np.int32)
    dist = np.full((nq, k), np.inf)
    probes = np.zeros((nq, n_probe), dtype=np.int32)
    for q in range(nq):
        pr = np.lexsort((np.arange(len(C)), dc[q]))[:n_probe]
        probes[q] = pr
        rows = np.nonzero(np.isin(lists, pr))[0]
        if len(rows) == 0:
            continue
        dq = _ivf_key(Q[q:q + 1], X[rows], metric)[0]
        o = np.lexsort((rows, dq))[:k]
        ind[q, :len(o)] = rows[o]
        dist[q, :len(o)] = dq[o]
    if metric == "euclidean":
        pos = dist >= 0
        dist[pos] = np.sqrt(dist[pos])
    if metric == "inner product":   # empty slots: -inf, as the reference's scaling by -1
        dist = -dist
    elif metric == "cosine":
        dist = 1.0 + dist
    return ind, dist, probes


def kmeans_assign(X, Cn):
    X = np.ascontiguousarray(X)
    dt = X.dtype
    Cn = np.ascontiguousarray(Cn, dtype=dt)
    n, d = X.shape
    lab = np.zeros(n, dtype=np.int32)
    gap = np.zeros(n, dtype=np.float64)
    getattr(lib(), f"orc_kmeans_assign_{_sfx(dt)}")(n, d, _p(X), Cn.shape[0], _p(Cn), _p(lab),
                                                    _p(gap))
    return lab, gap


def kmeans_update(X, labels, k):
    Xd = np.ascontiguousarray(X, dtype=np.float64)
    n, d = Xd.shape
    Cn = np.zeros((k, d), dtype=np.float64)
    cnt = np.zeros(k, dtype=np.int32)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    lib().orc_kmeans_update_d(n, d, _p(Xd), _p(lab), k, _p(Cn), _p(cnt))
    return Cn, cnt


def kmeans_inertia(X, labels, Cn):
    Xd = np.ascontiguousarray(X, dtype=np.float64)
    n, d = Xd.shape
    return lib().orc_kmeans_inertia_d(n, d, _p(Xd), _p(np.ascontiguousarray(labels, np.int32)),
                                      _p(np.ascontiguousarray(Cn, np.float64)))


def kmeans_lloyd(X, C0, max_iter=300, tol=1e-4):
    X = np.ascontiguousarray(X)
    dt = X.dtype
    C0 = np.ascontiguousarray(C0, dtype=dt)
    n, d = X.shape
    k = C0.shape[0]
    Cout = np.zeros_like(C0)
    lab = np.zeros(n, dtype=np.int32)
    nit = np.zeros(1, dtype=np.int32)
    inertia = np.zeros(1, dtype=np.float64)
    getattr(lib(), f"orc_kmeans_lloyd_{_sfx(dt)}")(n, d, _p(X), k, _p(C0), max_iter, tol,
                                                   _p(Cout), _p(lab), _p(nit), _p(inertia))
    return Cout, lab, int(nit[0]), float(inertia[0])


def kmeans_iteration(X, C, labels):
    """One Lloyd iteration in place (CPU baseline timing)."""
    n, d = X.shape
    return lib().orc_kmeans_iteration_s(n, d, _p(X), C.shape[0], _p(C), _p(labels))


def knn_reference_ties(keys, k):
    keys = np.ascontiguousarray(keys, dtype=np.float64)
    ind = np.zeros(k, dtype=np.int32)
    lib().orc_knn_reference_ties_d(len(keys), _p(keys), k, _p(ind))
    return ind


def num_threads():
    return lib().orc_num_threads()


def kmeanspp(X, k, seed, cost_fp64=False, gemm=None):
    """Row indices of the k-means++ initial centres (oracle_kpp.cpp, after
    kmeans.cpp:1491-1664 and :1814-1822): the reference's std::mt19937_64
    draws, distances in GEMM form, candidate costs summed in the working
    precision (fp64 with cost_fp64).  gemm: an OpenBLAS handle (openblas())
    for BLAS dot products instead of the sequential fma chain."""
    X = np.ascontiguousarray(X)
    n, d = X.shape
    chosen = np.zeros(k, dtype=np.int32)
    fn = None
    if gemm is not None:
        fn = gemm.sgemm if X.dtype == np.float32 else gemm.dgemm
    r = getattr(lib(), f"orc_kmeanspp_{_sfx(X.dtype)}")(n, d, _p(X), k, int(seed),
                                                         1 if cost_fp64 else 0, fn, _p(chosen))
    if r < 0:
        raise ValueError("kmeanspp: bad arguments")
    return chosen


def kmeanspp_cosine(X, k, seed, normalise=True):
    """k-means++ rows of spherical k-means (oracle_kpp.cpp; the cosine
    distance of kmeans.cpp:1495-1510)."""
    X = np.ascontiguousarray(X)
    n, d = X.shape
    chosen = np.zeros(k, dtype=np.int32)
    r = getattr(lib(), f"orc_kmeanspp_cos_{_sfx(X.dtype)}")(n, d, _p(X), k, int(seed),
                                                             1 if normalise else 0, _p(chosen))
    if r < 0:
        raise ValueError("kmeanspp_cosine: bad arguments")
    return chosen


def kmeans_assign_sph(X, C):
    """Spherical assignment argmin_j -x.c_j (oracle.c) and the fp64 gap
    between the best two values (near-tie classification)."""
    X = np.ascontiguousarray(X)
    C = np.ascontiguousarray(C, dtype=X.dtype)
    n, d = X.shape
    lab = np.zeros(n, dtype=np.int32)
    gap = np.zeros(n, dtype=np.float64)
    getattr(lib(), f"orc_kmeans_assign_sph_{_sfx(X.dtype)}")(n, d, _p(X), C.shape[0], _p(C),
                                                             _p(lab), _p(gap))
    return lab, gap


def kmeans_inertia_sph(X, labels, C, normalise=True):
    X = np.ascontiguousarray(X)
    C = np.ascontiguousarray(C, dtype=X.dtype)
    n, d = X.shape
    return getattr(lib(), f"orc_kmeans_inertia_sph_{_sfx(X.dtype)}")(
        n, d, _p(X), _p(np.ascontiguousarray(labels, np.int32)), _p(C), 1 if normalise else 0)


def kmeans_sph_lloyd(X, C0, max_iter=300, tol=1e-4, normalise=True):
    """Spherical (cosine) Lloyd from the given centres (oracle.c)."""
    X = np.ascontiguousarray(X)
    dt = X.dtype
    C0 = np.ascontiguousarray(C0, dtype=dt)
    n, d = X.shape
    k = C0.shape[0]
    Cout = np.zeros_like(C0)
    lab = np.zeros(n, dtype=np.int32)
    nit = np.zeros(1, dtype=np.int32)
    inertia = np.zeros(1, dtype=np.float64)
    getattr(lib(), f"orc_kmeans_sph_lloyd_{_sfx(dt)}")(n, d, _p(X), k, _p(C0), max_iter, tol,
                                                       1 if normalise else 0, _p(Cout), _p(lab),
                                                       _p(nit), _p(inertia))
    return Cout, lab, int(nit[0]), float(inertia[0])


class openblas:
    """The OpenBLAS that ships with scipy (cblas_sgemm / cblas_dgemm and its
    thread-count setter), loaded for the CPU baseline."""

    def __init__(self):
        import glob
        import scipy
        libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
        cand = sorted(glob.glob(os.path.join(libs, "libscipy_openblas-*.so")))
        if not cand:
            raise OSError("scipy's OpenBLAS not found")
        self.path = cand[0]
        self.lib = C.CDLL(self.path)
        self.sgemm = C.cast(self.lib.scipy_cblas_sgemm, C.c_void_p).value
        self.dgemm = C.cast(self.lib.scipy_cblas_dgemm, C.c_void_p).value
        self.lib.scipy_openblas_set_num_threads.argtypes = [C.c_int]
        self.lib.scipy_openblas_get_num_threads.restype = C.c_int
        self.lib.scipy_openblas_get_config.restype = C.c_char_p

    def set_threads(self, t):
        self.lib.scipy_openblas_set_num_threads(int(t))

    def threads(self):
        return int(self.lib.scipy_openblas_get_num_threads())

    def config(self):
        return self.lib.scipy_openblas_get_config().decode()


def lloyd_blas(X, C, labels, n_iter, blas, threads=0):
    """n_iter Lloyd iterations of the reference's blocked BLAS form
    (oracle_blas.c, after kmeans_lloyd.hpp:106-405) in place on C (k x d,
    fp32) and labels; BLAS one thread per call inside the OpenMP region.
    Returns the number of labels changed by the last iteration."""
    n, d = X.shape
    old = blas.threads()
    blas.set_threads(1)
    try:
        r = lib().orc_lloyd_blas_s(n, d, _p(X), C.shape[0], _p(C), _p(labels), n_iter,
                                   blas.sgemm, threads)
    finally:
        blas.set_threads(old)
    if r < 0:
        raise MemoryError("lloyd_blas")
    return r
