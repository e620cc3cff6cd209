"""kmeans with the reference's Python interface
(python_interface/python_package/aoclda/clustering.py:36-326) over the B200
k-means handle."""
import numpy as np

from ._binding import ab, convert, dump_model, load_model


class kmeans():
    """k-means clustering (clustering.py:36-326).  The handle is created at
    fit() in the precision of the data (float32: single, otherwise double);
    C gives the initial centres ("supplied" initialisation)."""

    def __init__(self, n_clusters=1, initialization_method='k-means++', C=None, n_init=10,
                 max_iter=300, seed=-1, algorithm='lloyd', distance='euclidean',
                 normalize_data=False, tol=1.0e-4, empty_clusters='ignore',
                 afk_mcmc_samples=50, mixed_precision=False, low_precision_max_iter=200,
                 low_precision_tol=1.0e-2, check_data=False):
        self._opts = {
            "n_clusters": int(n_clusters), "n_init": int(n_init), "max_iter": int(max_iter),
            "seed": int(seed), "initialization method": initialization_method,
            "algorithm": algorithm, "distance": distance,
            "normalize data": "yes" if normalize_data else "no",
            "empty clusters": empty_clusters, "afk-mc2 samples": int(afk_mcmc_samples),
            "mixed precision": "yes" if mixed_precision else "no",
            "low precision max_iter": int(low_precision_max_iter),
            "check data": "yes" if check_data else "no"}
        self._reals = {"convergence tolerance": float(tol),
                       "low precision convergence tolerance": float(low_precision_tol)}
        self.C = C
        self._h = None
        self._k, self._d = int(n_clusters), None

    def fit(self, A):
        A, prec, order = convert(A)
        h = ab.KMeans(self._k, prec, order=order)
        for name, v in list(self._opts.items()) + list(self._reals.items()):
            st = h.set(name, v)
            if st != ab.SUCCESS:
                raise ab.DAError(st, f"option {name}")
        C0 = None if self.C is None else convert(self.C, prec, order)[0]
        h.fit(A, C0)
        self._h, self._d = h, A.shape[1]
        return self

    def _rinfo(self):
        return self._h.rinfo()

    @property
    def cluster_centres(self):
        return np.ascontiguousarray(self._h.centres(self._k, self._d))

    @property
    def labels(self):
        return self._h.labels(int(self._rinfo()[0]))

    @property
    def inertia(self):
        return float(self._rinfo()[4])

    @property
    def n_iter(self):
        return int(self._rinfo()[3])

    @property
    def lp_n_iter(self):
        return int(self._rinfo()[5])

    @property
    def n_samples(self):
        return int(self._rinfo()[0])

    @property
    def n_features(self):
        return int(self._rinfo()[1])

    @property
    def n_clusters(self):
        return int(self._rinfo()[2])

    def transform(self, X):
        """Distances of every row to every centre, m x n_clusters."""
        X = convert(X, self._h.prec, self._h.order)[0]
        return np.ascontiguousarray(self._h.transform(X, self._k))

    def predict(self, Y):
        Y = convert(Y, self._h.prec, self._h.order)[0]
        return self._h.predict(Y)

    # pickling (clustering.py:282-323): the parameters and the fitted model
    def __getstate__(self):
        st = {k: v for k, v in self.__dict__.items() if k != "_h"}
        st["_model"] = None if self._h is None else (dump_model(self._h), self._h.prec)
        return st

    def __setstate__(self, st):
        model = st.pop("_model")
        self.__dict__.update(st)
        self._h = None if model is None else load_model(ab.KMeans, model[0], model[1])
