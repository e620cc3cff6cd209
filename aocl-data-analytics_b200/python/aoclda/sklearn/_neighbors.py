"""scikit-learn neighbour estimators over the B200 kNN / radius handle
(python_package/aoclda/sklearn/_neighbors.py): the sklearn constructor
arguments, validated as there; metric_params / n_jobs are ignored with a
warning; methods outside the path raise."""
import warnings

from sklearn.neighbors import KNeighborsClassifier as _KNC
from sklearn.neighbors import KNeighborsRegressor as _KNR
from sklearn.neighbors import NearestNeighbors as _NN
from sklearn.neighbors import RadiusNeighborsClassifier as _RNC
from sklearn.neighbors import RadiusNeighborsRegressor as _RNR

from ..neighbors import nearest_neighbors as _nn_da

_ALGORITHMS = ('auto', 'ball_tree', 'brute', 'kd_tree')
_METRICS = ('euclidean', 'l2', 'sqeuclidean', 'manhattan', 'l1', 'cityblock', 'cosine',
            'minkowski', 'euclidean_gemm', 'sqeuclidean_gemm')
# sklearn's tree names -> the library's "algorithm" option
_ALGO = {'auto': 'auto', 'brute': 'brute', 'kd_tree': 'kd tree', 'ball_tree': 'ball tree'}


def _check(algorithm, weights, metric, metric_params, n_jobs):
    if metric_params is not None or n_jobs is not None:
        warnings.warn("The parameters metric_params and n_jobs are not supported and have been "
                      "ignored.", category=RuntimeWarning)
    if algorithm not in _ALGORITHMS:
        raise ValueError("Invalid algorithm chosen, available options are ", _ALGORITHMS)
    if weights not in ('uniform', 'distance', None):
        raise ValueError("Invalid weights chosen, available options are 'uniform', 'distance' "
                         "and None.")
    if metric not in _METRICS:
        raise ValueError("Invalid metric provided, available options are ", _METRICS)
    return weights or 'uniform'


class _Base:
    def _model(self, **extra):
        return _nn_da(weights=self.weights, algorithm=_ALGO[self.algorithm],
                      leaf_size=self.leaf_size, metric=self.metric, p=float(self.p), **extra)

    def get_params(self, deep=True):
        return {k: getattr(self, k) for k in self._params}

    def score(self, X, y, sample_weight=None):
        raise RuntimeError("This feature is not implemented")

    def get_metadata_routing(self):
        raise RuntimeError("This feature is not implemented")


class NearestNeighbors(_Base, _NN):
    _params = ('n_neighbors', 'radius', 'algorithm', 'leaf_size', 'metric', 'p', 'metric_params',
               'n_jobs')

    def __init__(self, *, n_neighbors=5, radius=1.0, algorithm='auto', leaf_size=30,
                 metric='minkowski', p=2, metric_params=None, n_jobs=None):
        self.n_neighbors, self.radius, self.algorithm = n_neighbors, radius, algorithm
        self.leaf_size, self.metric, self.p = leaf_size, metric, p
        self.metric_params, self.n_jobs = metric_params, n_jobs
        self.weights = _check(algorithm, 'uniform', metric, metric_params, n_jobs)
        self.aocl = True
        self.nn_model = self._model(n_neighbors=n_neighbors, radius=radius)

    def fit(self, X, y=None):
        self.nn_model.fit(X, y)
        return self

    def kneighbors(self, X=None, n_neighbors=None, return_distance=True):
        return self.nn_model.kneighbors(X, n_neighbors, return_distance)

    def radius_neighbors(self, X=None, radius=None, return_distance=True, sort_results=False):
        return self.nn_model.radius_neighbors(X, radius, return_distance, sort_results)

    def kneighbors_graph(self, X=None, n_neighbors=None, mode='connectivity'):
        raise RuntimeError("This feature is not implemented")


class KNeighborsClassifier(_Base, _KNC):
    _params = ('n_neighbors', 'weights', 'algorithm', 'leaf_size', 'p', 'metric', 'metric_params',
               'n_jobs')

    def __init__(self, n_neighbors=5, *, weights='uniform', algorithm='auto', leaf_size=30, p=2,
                 metric='minkowski', metric_params=None, n_jobs=None):
        if n_neighbors is not None and n_neighbors <= 0:
            raise ValueError("Number of neighbors must be positive or None. Got n_neighbors=" +
                             str(n_neighbors))
        self.n_neighbors, self.algorithm, self.leaf_size = n_neighbors, algorithm, leaf_size
        self.p, self.metric = p, metric
        self.metric_params, self.n_jobs = metric_params, n_jobs
        self.weights = _check(algorithm, weights, metric, metric_params, n_jobs)
        self.aocl = True
        self.nn_model = self._model(n_neighbors=n_neighbors)

    def fit(self, X, y):
        self.nn_model.fit(X, y)
        return self

    def kneighbors(self, X=None, n_neighbors=None, return_distance=True):
        return self.nn_model.kneighbors(X, n_neighbors, return_distance)

    def predict_proba(self, X):
        return self.nn_model.classifier_predict_proba(X, "knn")

    def predict(self, X):
        return self.nn_model.classifier_predict(X, "knn")

    def kneighbors_graph(self, X=None, n_neighbors=None, mode='connectivity'):
        raise RuntimeError("This feature is not implemented")


class KNeighborsRegressor(_Base, _KNR):
    _params = KNeighborsClassifier._params

    def __init__(self, n_neighbors=5, *, weights='uniform', algorithm='auto', leaf_size=30, p=2,
                 metric='minkowski', metric_params=None, n_jobs=None):
        if n_neighbors is not None and n_neighbors <= 0:
            raise ValueError("Number of neighbors must be positive or None. Got n_neighbors=" +
                             str(n_neighbors))
        self.n_neighbors, self.algorithm, self.leaf_size = n_neighbors, algorithm, leaf_size
        self.p, self.metric = p, metric
        self.metric_params, self.n_jobs = metric_params, n_jobs
        self.weights = _check(algorithm, weights, metric, metric_params, n_jobs)
        self.aocl = True
        self.nn_model = self._model(n_neighbors=n_neighbors)

    def fit(self, X, y):
        self.nn_model.fit(X, y)
        return self

    def kneighbors(self, X=None, n_neighbors=None, return_distance=True):
        return self.nn_model.kneighbors(X, n_neighbors, return_distance)

    def predict(self, X):
        return self.nn_model.regressor_predict(X, "knn")

    def kneighbors_graph(self, X=None, n_neighbors=None, mode='connectivity'):
        raise RuntimeError("This feature is not implemented")


class RadiusNeighborsClassifier(_Base, _RNC):
    _params = ('radius', 'weights', 'algorithm', 'leaf_size', 'p', 'metric', 'outlier_label',
               'metric_params', 'n_jobs')

    def __init__(self, radius=1.0, *, weights='uniform', algorithm='auto', leaf_size=30, p=2,
                 metric='minkowski', outlier_label=None, metric_params=None, n_jobs=None):
        self.radius, self.algorithm, self.leaf_size = radius, algorithm, leaf_size
        self.p, self.metric, self.outlier_label = p, metric, outlier_label
        self.metric_params, self.n_jobs = metric_params, n_jobs
        self.weights = _check(algorithm, weights, metric, metric_params, n_jobs)
        self.aocl = True
        self.nn_model = self._model(radius=radius, outlier_handling=outlier_label)

    def fit(self, X, y):
        self.nn_model.fit(X, y)
        return self

    def radius_neighbors(self, X=None, radius=None, return_distance=True, sort_results=False):
        return self.nn_model.radius_neighbors(X, radius, return_distance, sort_results)

    def predict_proba(self, X):
        return self.nn_model.classifier_predict_proba(X, "radius_neighbors")

    def predict(self, X):
        return self.nn_model.classifier_predict(X, "radius_neighbors")


class RadiusNeighborsRegressor(_Base, _RNR):
    _params = ('radius', 'weights', 'algorithm', 'leaf_size', 'p', 'metric', 'metric_params',
               'n_jobs')

    def __init__(self, radius=1.0, *, weights='uniform', algorithm='auto', leaf_size=30, p=2,
                 metric='minkowski', metric_params=None, n_jobs=None):
        self.radius, self.algorithm, self.leaf_size = radius, algorithm, leaf_size
        self.p, self.metric = p, metric
        self.metric_params, self.n_jobs = metric_params, n_jobs
        self.weights = _check(algorithm, weights, metric, metric_params, n_jobs)
        self.aocl = True
        self.nn_model = self._model(radius=radius)

    def fit(self, X, y):
        self.nn_model.fit(X, y)
        return self

    def radius_neighbors(self, X=None, radius=None, return_distance=True, sort_results=False):
        return self.nn_model.radius_neighbors(X, radius, return_distance, sort_results)

    def predict(self, X):
        return self.nn_model.regressor_predict(X, "radius_neighbors")
