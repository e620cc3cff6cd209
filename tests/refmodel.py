"""Writes model files in AOCL-DA's own da_handle_save_model format.

TEST INFRASTRUCTURE ONLY: restates the reference's serializer
(utilities/model_persistence.cpp: scalars as int64 / one-byte bool / the
working precision, strings and vectors as an int64 count then the elements;
serialize_metadata at :107-130; OptionRegistry::save_registry,
utilities/options.hpp:956-975) and the field lists of kmeans<T>::serialize
(clustering/kmeans/kmeans.cpp:1882-1909), neighbors<T>::serialize
(nearest_neighbors/nearest_neighbors.cpp:2329-2404) and
approximate_neighbors<T>::serialize
(approximate_neighbors/approximate_neighbors.cpp:1346-1395), so that the
tests can give this library the files an AOCL-DA user already has."""
import struct

import numpy as np

HANDLE_KMEANS, HANDLE_NN, HANDLE_APPROX_NN = 3, 8, 11
ROW_MAJOR, COLUMN_MAJOR = 0, 1


class Writer:
    def __init__(self, prec):
        self.b = bytearray()
        self.dt = np.float32 if prec == "s" else np.float64

    def i64(self, v):
        self.b += struct.pack("<q", int(v))

    def flag(self, v):
        self.b += struct.pack("<B", 1 if v else 0)

    def real(self, v):
        self.b += np.asarray(v, dtype=self.dt).tobytes()

    def text(self, s):
        s = s.encode()
        self.i64(len(s))
        self.b += s

    def vec(self, a, dt=None):
        a = np.ascontiguousarray(np.asarray(a, dtype=dt or self.dt)).ravel()
        self.i64(a.size)
        self.b += a.tobytes()

    def ivec(self, a):
        self.vec(a, np.int64)

    def vvec(self, lists, dt=None):
        self.i64(len(lists))
        for a in lists:
            self.vec(a, dt)

    def metadata(self, handle, keyword="AOCLDA_STORED_MODEL", int_size=4, version=50301,
                 precision=None, aoclda="5.3.1"):
        self.text(keyword)
        self.i64(int_size)
        self.i64(version)
        self.i64(handle)
        self.i64(precision if precision is not None else np.dtype(self.dt).itemsize)
        self.text(aoclda)

    def registry(self, opts):
        """opts: (name, kind, value) with kind "I", "R" or "S"."""
        self.i64(len(opts))
        for name, kind, v in opts:
            self.text(name)
            {"I": self.i64, "R": self.real, "S": self.text}[kind](v)

    def save(self, path):
        with open(path, "wb") as f:
            f.write(bytes(self.b))


def common_opts(order):
    return [("storage order", "S", "row-major" if order == ROW_MAJOR else "column-major"),
            ("check data", "S", "no")]


def kmeans_file(path, prec, order, C, labels, n_iter, inertia, distance="euclidean",
                normalise=True, seed=0, tol=1e-4, max_iter=300, n_init=1):
    """A computed k-means handle: C (k x d) the centres, labels per row."""
    k, d = C.shape
    w = Writer(prec)
    w.metadata(HANDLE_KMEANS)
    w.registry(common_opts(order) + [
        ("n_clusters", "I", k), ("n_init", "I", n_init), ("max_iter", "I", max_iter),
        ("low precision max_iter", "I", 200), ("seed", "I", seed), ("afk-mc2 samples", "I", 50),
        ("initialization method", "S", "k-means++"), ("algorithm", "S", "lloyd"),
        ("mixed precision", "S", "no"), ("empty clusters", "S", "ignore"),
        ("distance", "S", distance), ("normalize data", "S", "yes" if normalise else "no"),
        ("convergence tolerance", "R", tol), ("low precision convergence tolerance", "R", 1e-2)])
    w.flag(True)                       # model_trained
    w.i64(order)
    w.i64(0)                           # algorithm (lloyd)
    w.i64(len(labels))
    w.i64(d)
    w.i64(n_iter)
    w.real(inertia)
    w.i64(seed)
    w.i64(k)
    w.real(tol)
    w.i64(max_iter)
    w.i64(n_init)
    w.ivec(labels)
    w.vec(np.asarray(C).T)             # column-major k x d
    c64 = np.asarray(C, dtype=np.float64)
    w.vec(np.zeros(k) if distance == "cosine" else (c64 * c64).sum(1))
    w.flag(distance == "cosine")
    w.flag(normalise)
    w.save(path)


def nn_file(path, prec, order, X, y=None, t=None, n_neighbors=5, metric="euclidean",
            algorithm="brute", weights="uniform", tree_bytes=b""):
    """A kNN handle with its training rows (and labels / targets)."""
    n, d = X.shape
    w = Writer(prec)
    w.metadata(HANDLE_NN)
    w.registry(common_opts(order) + [
        ("number of neighbors", "I", n_neighbors), ("leaf size", "I", 30),
        ("outlier label", "I", -1), ("minkowski parameter", "R", 2.0), ("radius", "R", 1.0),
        ("outlier target", "R", 0.0), ("algorithm", "S", algorithm), ("metric", "S", metric),
        ("weights", "S", weights), ("outlier handling", "S", "none")])
    w.i64(order)
    w.i64(n)
    w.i64(d)
    w.flag(y is not None)
    w.flag(t is not None)
    w.flag(True)                       # is_up_to_date
    w.flag(False)                      # classes_computed
    w.ivec([])                         # classes
    w.flag(False)                      # sort_results
    w.flag(True)                       # model_trained
    w.flag(False)                      # rnn_return_distances
    for v in (n_neighbors, 3, 3, 0, 1, 30):  # n_neighbors, algo, working_algo, metric,
        w.i64(v)                             # internal_metric, leaf_size
    w.flag(False)                      # get_squares
    w.real(2.0)                        # p
    for v in (0, 0, -1):               # weights, outlier_handling, n_classes
        w.i64(v)
    w.real(1.0)                        # radius
    w.ivec([])
    w.vvec([], np.int64)
    w.vvec([])
    w.flag(True)                       # istrained_Xtrain
    w.flag(False)
    w.i64(-1)
    w.flag(False)
    w.i64(-1)
    w.i64(-1)
    w.flag(False)
    w.real(0.0)
    w.real(-1.0)
    w.vec(np.asarray(X).T)             # column-major n x d
    w.ivec([] if y is None else y)
    w.vec([] if t is None else t)
    w.b += tree_bytes                  # a k-d / ball tree follows (not read)
    w.save(path)


def ivf_file(path, prec, order, centroids, lists_rows, lists_ids, n_index, metric="sqeuclidean",
             n_probe=1, kmeans_iter=10, seed=0, list_norms=None):
    """A trained IVF-flat index: centroids (n_list x d), per list its rows
    (m x d) and global indices, in insertion order."""
    nl, d = centroids.shape
    mets = {"euclidean": 0, "sqeuclidean": 1, "inner product": 2, "cosine": 3}
    w = Writer(prec)
    w.metadata(HANDLE_APPROX_NN)
    w.registry(common_opts(order) + [
        ("number of neighbors", "I", 5), ("n_list", "I", nl), ("n_probe", "I", n_probe),
        ("k-means_iter", "I", kmeans_iter), ("seed", "I", seed), ("train fraction", "R", 1.0),
        ("algorithm", "S", "ivfflat"), ("metric", "S", metric)])
    w.flag(True)                       # train_data_is_set
    w.flag(True)                       # model_trained
    w.flag(n_index > 0)                # data_is_added
    w.i64(5)                           # n_neighbors
    w.i64(0)                           # algo
    w.i64(0)                           # internal_algo
    w.i64(1 if mets[metric] == 0 else mets[metric])  # internal_metric
    w.i64(mets[metric])
    w.i64(seed)                        # internal_seed
    w.i64(seed)
    w.i64(n_index)                     # n_samples_train
    w.i64(order)
    w.i64(n_index)                     # n_samples
    w.i64(d)
    w.real(1.0)                        # train_fraction
    w.i64(nl)
    w.i64(n_probe)
    w.i64(kmeans_iter)                 # max_iter
    w.i64(kmeans_iter)
    w.i64(1)                           # n_init
    w.real(np.sqrt(np.finfo(w.dt).eps))
    if order == COLUMN_MAJOR:
        w.vec(np.asarray(centroids).T)  # n_list x d column-major, ld = n_list
        w.i64(nl)
    else:
        w.vec(centroids)
        w.i64(d)
    w.i64(n_index)
    w.vvec([np.asarray(r).ravel() for r in lists_rows])
    w.vvec(lists_ids, np.int64)
    w.ivec([len(i) for i in lists_ids])
    w.ivec([0] * nl)                   # old_list_sizes
    w.vvec(list_norms if list_norms is not None else [[] for _ in range(nl)])
    w.vec(np.zeros(0) if order == COLUMN_MAJOR else np.zeros(0))  # the training rows
    w.save(path)
