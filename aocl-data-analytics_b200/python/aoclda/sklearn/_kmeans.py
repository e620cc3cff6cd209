"""scikit-learn KMeans over the B200 k-means handle
(python_package/aoclda/sklearn/_kmeans.py): init may be 'k-means++',
'random', 'random partitions' or an array of initial centres; n_init 'auto'
is 1 for k-means++ and 10 otherwise; random_state an integer or None (-1:
a random seed)."""
import warnings

import numpy as np
from sklearn.cluster import KMeans as _KMeans

from ..clustering import kmeans as _kmeans_da


class KMeans(_KMeans):
    _params = ('n_clusters', 'init', 'n_init', 'max_iter', 'tol', 'verbose', 'random_state',
               'copy_x', 'algorithm')

    def __init__(self, n_clusters=8, *, init='k-means++', n_init='auto', max_iter=300,
                 tol=0.0001, verbose=None, random_state=None, copy_x=None, algorithm='lloyd',
                 distance='euclidean', normalize_data=False, empty_clusters='ignore',
                 afk_mcmc_samples=50, mixed_precision=False, low_precision_max_iter=200,
                 low_precision_tol=0.01):
        self.n_clusters, self.init, self.n_init = n_clusters, init, n_init
        self.max_iter, self.tol, self.verbose = max_iter, tol, verbose
        self.random_state, self.copy_x, self.algorithm = random_state, copy_x, algorithm
        if copy_x is not None or verbose is not None:
            warnings.warn("The parameters copy_x and verbose are not supported and have been "
                          "ignored.", category=RuntimeWarning)
        if callable(init):
            raise ValueError("init must be set to 'random', 'random partitions', 'k-means++' "
                             "or an array.")
        if isinstance(random_state, np.random.RandomState):
            raise ValueError("random_state must be an integer or None.")
        self.aocl = True
        seed = -1 if random_state is None else int(random_state)
        alg = "lloyd" if algorithm in ("full", "auto") else algorithm
        common = dict(max_iter=max_iter, seed=seed, algorithm=alg, distance=distance,
                      normalize_data=normalize_data, tol=tol, empty_clusters=empty_clusters,
                      afk_mcmc_samples=afk_mcmc_samples, mixed_precision=mixed_precision,
                      low_precision_max_iter=low_precision_max_iter,
                      low_precision_tol=low_precision_tol)
        if isinstance(init, np.ndarray):
            self.kmeans = _kmeans_da(n_clusters, initialization_method="supplied", n_init=1,
                                     C=init, **common)
        else:
            n = (1 if init == "k-means++" else 10) if n_init == "auto" else n_init
            self.kmeans = _kmeans_da(n_clusters, initialization_method=init, n_init=n,
                                     **common)

    def fit(self, X, y=None, sample_weight=None):
        self.kmeans.fit(X)
        return self

    def transform(self, X):
        return self.kmeans.transform(X)

    def predict(self, X):
        return self.kmeans.predict(X)

    def fit_transform(self, X, y=None, sample_weight=None):
        return self.fit(X).transform(X)

    def fit_predict(self, X, y=None, sample_weight=None):
        return self.fit(X).predict(X)

    def get_params(self, deep=True):
        return {k: getattr(self, k) for k in self._params}

    def score(self, X, y=None, sample_weight=None):
        raise RuntimeError("This feature is not implemented")

    @property
    def cluster_centers_(self):
        return self.kmeans.cluster_centres

    @property
    def labels_(self):
        return self.kmeans.labels

    @property
    def inertia_(self):
        return self.kmeans.inertia

    @property
    def n_iter_(self):
        return self.kmeans.n_iter
