"""faiss-compatible Kmeans (python_package/aoclda/faiss/_kmeans.py:37-140)
over the B200 k-means handle: train(x), centroids, obj, assign(x) ->
(squared distances, labels)."""
import warnings

import numpy as np

from ..clustering import kmeans


class Kmeans:
    def __init__(self, d, k, niter=25, nredo=1, verbose=False, seed=-1, spherical=False, *,
                 algorithm='lloyd', initialization_method='k-means++', normalize_data=False,
                 tol=1.0e-4, empty_clusters='ignore', afk_mcmc_samples=50,
                 mixed_precision=False, low_precision_max_iter=10, low_precision_tol=1.0e-2,
                 **kwargs):
        for kw in kwargs:
            warnings.warn(f"Kmeans: '{kw}' is not supported by the B200 backend.", UserWarning)
        if verbose:
            warnings.warn("Kmeans: 'verbose' is not supported by the B200 backend.", UserWarning)
        self.d, self.k = d, k
        self._args = dict(n_init=nredo, max_iter=niter, seed=seed,
                          distance="cosine" if spherical else "euclidean", algorithm=algorithm,
                          initialization_method=initialization_method,
                          normalize_data=normalize_data, tol=tol, empty_clusters=empty_clusters,
                          afk_mcmc_samples=afk_mcmc_samples, mixed_precision=mixed_precision,
                          low_precision_max_iter=low_precision_max_iter,
                          low_precision_tol=low_precision_tol)
        self._kmeans, self.obj, self.aocl = None, [], True

    def train(self, x):
        x = np.asarray(x)
        if x.ndim != 2 or x.shape[1] != self.d:
            raise ValueError(f"Kmeans.train: expected array with {self.d} columns, got shape "
                             f"{x.shape}")
        self._kmeans = kmeans(self.k, **self._args).fit(x)
        self.obj = [self._kmeans.inertia]
        return self.obj[-1]

    @property
    def centroids(self):
        return None if self._kmeans is None else self._kmeans.cluster_centres

    def assign(self, x):
        """(squared distance to the nearest centre, its index) per row."""
        lab = self._kmeans.predict(x)
        dist = self._kmeans.transform(x)
        return (dist[np.arange(len(lab)), lab] ** 2).astype(dist.dtype), lab.astype(np.int64)
