"""IndexFlatL2 (python_package/aoclda/faiss/_index_flat_l2.py:37-160): exact
squared-L2 search through the kNN handle ("sqeuclidean"); IndexIVFFlat
(_index_ivfflat.py:41-160): the IVF-flat handle, the quantizer only fixing d.
search() returns (distances, int64 indices) as faiss does."""
import warnings

import numpy as np

from ..neighbors import approximate_neighbors, nearest_neighbors

METRIC_INNER_PRODUCT, METRIC_L2 = 0, 1
_METRIC_MAP = {METRIC_INNER_PRODUCT: "inner product", METRIC_L2: "sqeuclidean"}


class _ClusteringParameters:
    """The faiss ClusteringParameters fields the index training uses."""

    def __init__(self, niter=25, nredo=1, seed=-1, spherical=False,
                 max_points_per_centroid=None):
        self.niter, self.nredo, self.seed = niter, nredo, seed
        self.spherical, self.max_points_per_centroid = spherical, max_points_per_centroid


def _rows(X, d, where):
    X = np.asarray(X)
    if X.ndim != 2 or X.shape[1] != d:
        raise ValueError(f"{where}: expected array with {d} columns, got shape {X.shape}")
    return X


class IndexFlatL2:
    def __init__(self, d):
        self._d, self._nn, self._ntotal, self._all_data = d, None, 0, None
        self.aocl = True

    d = property(lambda self: self._d)
    ntotal = property(lambda self: self._ntotal)
    is_trained = property(lambda self: True)
    metric_type = property(lambda self: METRIC_L2)

    def add(self, X):
        X = _rows(X, self._d, "IndexFlatL2.add")
        self._all_data = X if self._all_data is None else np.concatenate([self._all_data, X])
        self._ntotal += X.shape[0]
        self._nn = nearest_neighbors(metric="sqeuclidean").fit(self._all_data)

    def train(self, X):
        pass

    def search(self, X, k):
        if self._nn is None:
            raise RuntimeError("IndexFlatL2.search: index is empty, call add() first")
        dist, ind = self._nn.kneighbors(X, n_neighbors=int(k))
        return dist, ind.astype(np.int64)

    def assign(self, X, k):
        return self.search(X, k)[1]

    def reset(self):
        self._all_data, self._ntotal, self._nn = None, 0, None

    def reconstruct(self, i):
        if self._all_data is None or not 0 <= i < self._ntotal:
            raise RuntimeError("IndexFlatL2.reconstruct: index out of range")
        return self._all_data[i].copy()

    def reconstruct_n(self, i0, ni):
        return self._all_data[i0:i0 + ni].copy()


class IndexIVFFlat:
    def __init__(self, quantizer, d, nlist, metric=METRIC_L2):
        if quantizer.d != d:
            raise ValueError(f"quantizer dimension {quantizer.d} does not match d={d}")
        if type(quantizer).__name__ not in ("IndexFlatL2", "IndexFlatIP"):
            warnings.warn("Non-Flat quantizer passed to IndexIVFFlat; the quantizer will be "
                          "ignored.", UserWarning)
        if metric not in _METRIC_MAP:
            raise ValueError(f"Unknown metric integer {metric}; expected 0 "
                             "(METRIC_INNER_PRODUCT) or 1 (METRIC_L2)")
        self._d, self._nlist, self._metric = d, nlist, metric
        self._ann, self._is_trained, self._nprobe = None, False, 1
        self.cp = _ClusteringParameters(niter=25, seed=0)
        self.aocl = True

    d = property(lambda self: self._d)
    nlist = property(lambda self: self._nlist)
    is_trained = property(lambda self: self._is_trained)
    metric_type = property(lambda self: self._metric)
    ntotal = property(lambda self: self._ann.n_index if self._ann is not None else 0)

    @property
    def nprobe(self):
        return self._nprobe

    @nprobe.setter
    def nprobe(self, value):
        self._nprobe = int(value)
        if self._ann is not None:
            self._ann.n_probe = self._nprobe

    def train(self, X):
        X = _rows(X, self._d, "IndexIVFFlat.train")
        frac = 1.0
        if self.cp.max_points_per_centroid is not None:
            frac = min(1.0, self.cp.max_points_per_centroid * self._nlist / X.shape[0])
        self._ann = approximate_neighbors(n_list=self._nlist, metric=_METRIC_MAP[self._metric],
                                          n_neighbors=1, n_probe=self._nprobe,
                                          kmeans_iter=self.cp.niter, train_fraction=frac,
                                          seed=self.cp.seed)
        self._ann.train(X)
        self._is_trained = True

    def add(self, X):
        if not self._is_trained:
            raise RuntimeError("IndexIVFFlat.add: the index is not trained")
        self._ann.add(_rows(X, self._d, "IndexIVFFlat.add"))

    def search(self, X, k):
        if self._ann is None:
            raise RuntimeError("IndexIVFFlat.search: the index is not trained")
        dist, ind = self._ann.kneighbors(_rows(X, self._d, "IndexIVFFlat.search"), int(k))
        return dist, ind.astype(np.int64)

    def reset(self):
        self._ann, self._is_trained = None, False
