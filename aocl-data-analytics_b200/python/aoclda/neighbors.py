"""nearest_neighbors and approximate_neighbors with the reference's Python
interface (python_interface/python_package/aoclda/neighbors.py:39-800) over
the B200 kNN, radius and IVF-flat handles."""
import numpy as np

from ._binding import ab, convert, dump_model, load_model

_MODES = {"knn": ab.KNN_SEARCH, "radius_neighbors": ab.RADIUS_SEARCH,
          "radius": ab.RADIUS_SEARCH}


def _mode(search_mode):
    if search_mode not in _MODES:
        raise ValueError("search_mode must be 'knn' or 'radius_neighbors'. Got search_mode=" +
                         str(search_mode))
    return _MODES[search_mode]


class nearest_neighbors():
    """Brute-force nearest neighbours (neighbors.py:39-575): kneighbors,
    radius_neighbors, classifier / regressor predict in kNN or radius mode.
    The handle is created at fit() in the precision of the data (float32:
    single, otherwise double)."""

    def __init__(self, n_neighbors=5, weights='uniform', algorithm='auto', leaf_size=30,
                 metric='euclidean', p=2.0, radius=1.0, outlier_handling=None,
                 check_data=False):
        if not isinstance(n_neighbors, int) and n_neighbors is not None:
            raise ValueError("Number of neighbors must be an integer or None. Got n_neighbors=" +
                             str(n_neighbors))
        if not isinstance(radius, (int, float)) and radius is not None:
            raise ValueError("Radius must be a number or None. Got radius=" + str(radius))
        if radius is not None and radius < 0.0:
            raise ValueError("Radius must be positive. Got radius=" + str(radius))
        self.n_neighbors = n_neighbors
        self.weights, self.algorithm, self.leaf_size = weights, algorithm, leaf_size
        self.metric, self.p, self.radius = metric, p, radius
        self.outlier_handling = outlier_handling
        self.check_data = check_data
        self.y = None
        self._h = None

    def fit(self, X, y=None):
        if X is None:
            raise ValueError("fit() is not implemented for X=None")
        X, prec, order = convert(X)
        self._h = ab.KNN(prec, order=order, number_of_neighbors=self.n_neighbors or 1,
                         weights=self.weights, algorithm=self.algorithm.replace("_", " "),
                         leaf_size=int(self.leaf_size), metric=self.metric,
                         minkowski_parameter=float(self.p),
                         radius=float(self.radius if self.radius is not None else 0.0),
                         check_data="yes" if self.check_data else "no")
        self._h.fit(X)
        self.y = None if y is None else np.asarray(y)
        return self

    def _queries(self, X, what):
        if X is None:
            raise ValueError(f"{what}() is not implemented for X=None")
        if self._h is None:
            raise RuntimeError("fit() must be called first")
        return convert(X, self._h.prec, self._h.order)[0]

    def kneighbors(self, X, n_neighbors=None, return_distance=True):
        """(distances, indices), or indices only, n_queries x n_neighbors."""
        Q = self._queries(X, "kneighbors")
        if not isinstance(n_neighbors, int) and n_neighbors is not None:
            raise ValueError("Number of neighbors must be an integer or None. Got n_neighbors=" +
                             str(n_neighbors))
        if n_neighbors is not None and n_neighbors <= 0:
            raise ValueError("Number of neighbors must be positive or None. Got n_neighbors=" +
                             str(n_neighbors))
        if n_neighbors is None and self.n_neighbors is None:
            raise ValueError("n_neighbors cannot be None in kneighbors() if it was None in the "
                             "constructor.")
        k = n_neighbors if n_neighbors is not None else self.n_neighbors
        ind, dist = self._h.kneighbors(Q, k, return_distance)
        ind = np.ascontiguousarray(ind)
        return (np.ascontiguousarray(dist), ind) if return_distance else ind

    def radius_neighbors(self, X, radius=None, return_distance=True, sort_results=False):
        """Per query the rows within the radius: (distances, indices) as
        object arrays of 1-D arrays, or indices only."""
        Q = self._queries(X, "radius_neighbors")
        if radius is None:
            if self.radius is None:
                raise ValueError("radius cannot be None in radius_neighbors() if it was None "
                                 "in the constructor.")
            radius = self.radius
        if radius < 0:
            raise ValueError("Radius must be positive. Got radius=" + str(radius))
        cnt, off, ind, dist = self._h.radius_neighbors(Q, float(radius), return_distance,
                                                       sort_results)
        nq = Q.shape[0]
        starts = np.concatenate([[0], np.cumsum(cnt[:nq])])
        ind_l = np.empty(nq, dtype=object)
        dist_l = np.empty(nq, dtype=object)
        for q in range(nq):
            ind_l[q] = ind[starts[q]:starts[q + 1]].astype(np.int32)
            if return_distance:
                dist_l[q] = dist[starts[q]:starts[q + 1]].copy()
        return (dist_l, ind_l) if return_distance else ind_l

    def _outliers(self, search_mode, regression):
        """The reference's outlier_handling argument (neighbors.py:360-400):
        None, 'most_frequent', or the outlier label (classification) /
        target (regression) for "manual"."""
        h = self._h
        if _mode(search_mode) != ab.RADIUS_SEARCH:
            return
        oh = self.outlier_handling
        if oh is None:
            h.set("outlier handling", "none")
        elif isinstance(oh, str):
            if oh not in ("most_frequent", "most frequent"):
                raise ValueError("outlier_handling must be None, 'most_frequent', or a number. "
                                 "Got outlier_handling=" + oh)
            h.set("outlier handling", "most frequent")
        else:
            h.set("outlier handling", "manual")
            if regression:
                h.set("outlier target", float(oh))
            else:
                if float(oh) != int(oh):
                    raise ValueError("outlier_handling must be None, 'most_frequent', or an "
                                     "integer for classification. Got outlier_handling=" +
                                     str(oh))
                h.set("outlier label", int(oh))

    def _labels(self):
        if self.y is None:
            raise ValueError("Labels y were not provided during fit(). Classification is not "
                             "available.")
        self._h.y = np.ascontiguousarray(self.y, dtype=np.int32)
        self._h.call(f"da_nn_set_labels_{self._h.prec}", len(self._h.y), ab.ptr(self._h.y))

    def _targets(self):
        if self.y is None:
            raise ValueError("Targets y were not provided during fit(). Regression is not "
                             "available.")
        self._h.t = np.ascontiguousarray(self.y, dtype=self._h.dtype)
        self._h.call(f"da_nn_set_targets_{self._h.prec}", len(self._h.t), ab.ptr(self._h.t))

    def classifier_predict_proba(self, X, search_mode="knn"):
        Q = self._queries(X, "classifier_predict_proba")
        self._labels()
        self._outliers(search_mode, False)
        return np.ascontiguousarray(self._h.predict_proba(Q, _mode(search_mode)))

    def classifier_predict(self, X, search_mode="knn"):
        Q = self._queries(X, "classifier_predict")
        self._labels()
        self._outliers(search_mode, False)
        return self._h.predict(Q, _mode(search_mode))

    def regressor_predict(self, X, search_mode="knn"):
        Q = self._queries(X, "regressor_predict")
        self._targets()
        self._outliers(search_mode, True)
        return self._h.predict_reg(Q, _mode(search_mode))

    # pickling (neighbors.py:537-572): the parameters, the labels / targets
    # and the handle's model file (the training rows are in it)
    def __getstate__(self):
        st = {k: v for k, v in self.__dict__.items() if k != "_h"}
        st["_model"] = None if self._h is None else (dump_model(self._h), self._h.prec)
        return st

    def __setstate__(self, st):
        model = st.pop("_model")
        self.__dict__.update(st)
        self._h = None if model is None else load_model(ab.KNN, model[0], model[1])


class approximate_neighbors():
    """IVF-flat approximate neighbours (neighbors.py:578-800)."""

    def __init__(self, n_neighbors=5, algorithm='ivfflat', metric='sqeuclidean', n_list=1,
                 n_probe=1, kmeans_iter=10, train_fraction=1.0, seed=0, check_data=False):
        self._opts = dict(number_of_neighbors=n_neighbors, algorithm=algorithm, metric=metric,
                          n_list=n_list, n_probe=n_probe, kmeans_iter=kmeans_iter, seed=seed,
                          train_fraction=float(train_fraction))
        self._check = check_data
        self._n_probe = n_probe
        self._h = None
        self._X = None

    @property
    def n_probe(self):
        return self._n_probe

    @n_probe.setter
    def n_probe(self, value):
        self._n_probe = value
        self._opts["n_probe"] = value
        if self._h is not None:
            self._h.set("n_probe", int(value))

    def _handle(self, X):
        X, prec, order = convert(X)
        self._h = ab.ApproxNN(prec, order=order, **self._opts)
        self._h.set("check data", "yes" if self._check else "no")
        return X

    def train(self, X_train):
        self._X = self._handle(X_train)
        self._h.set_training_data(self._X).train()
        return self

    def train_and_add(self, X_train):
        self._X = self._handle(X_train)
        self._h.set_training_data(self._X).train_and_add()
        return self

    def add(self, X_add):
        if self._h is None:
            raise RuntimeError("train() must be called first")
        self._h.add(convert(X_add, self._h.prec, self._h.order)[0])
        return self

    def kneighbors(self, X_test, n_neighbors=0, return_distance=True):
        if self._h is None:
            raise RuntimeError("train() must be called first")
        Q = convert(X_test, self._h.prec, self._h.order)[0]
        k = n_neighbors if n_neighbors and n_neighbors > 0 else \
            self._h.get_int("number of neighbors")
        ind, dist = self._h.kneighbors(Q, k, return_distance)
        ind = np.ascontiguousarray(ind)
        return (np.ascontiguousarray(dist), ind) if return_distance else ind

    def _rinfo(self):
        return self._h.result(ab.RINFO, 4)

    @property
    def cluster_centroids(self):
        nl, _, d, _ = (int(v) for v in self._rinfo())
        c = self._h.result(ab.APPROX_NN_CENTROIDS, nl * d)
        return c.reshape(nl, d) if self._h.order == ab.ROW_MAJOR else c.reshape(d, nl).T.copy()

    @property
    def list_sizes(self):
        return self._h.list_sizes(int(self._rinfo()[0]))

    @property
    def n_list(self):
        return int(self._rinfo()[0])

    @property
    def n_index(self):
        return int(self._rinfo()[1]) if self._h is not None else 0

    @property
    def n_features(self):
        return int(self._rinfo()[2])

    @property
    def kmeans_iter(self):
        return int(self._rinfo()[3])

    # pickling (neighbors.py:735-765): the parameters and the trained index
    def __getstate__(self):
        st = {k: v for k, v in self.__dict__.items() if k not in ("_h", "_X")}
        st["_model"] = None if self._h is None else (dump_model(self._h), self._h.prec)
        return st

    def __setstate__(self, st):
        model = st.pop("_model")
        self.__dict__.update(st)
        self._X = None
        self._h = None if model is None else load_model(ab.ApproxNN, model[0], model[1])
