"""scikit-learn pairwise_distances over da_pairwise_distances_?
(python_package/aoclda/sklearn/_metrics.py:35-53)."""
import warnings

from ..metrics import pairwise_distances as _pd_da


def pairwise_distances(X, Y=None, metric='euclidean', p=2.0, n_jobs=None,
                       force_all_finite=True, **kwds):
    if force_all_finite is not False:
        warnings.warn("The parameter force_all_finite is not supported and has been ignored. "
                      "No checks are performed on input data.", category=RuntimeWarning)
    if n_jobs is not None:
        warnings.warn("The parameter n_jobs is not supported and has been ignored.",
                      category=RuntimeWarning)
    return _pd_da(X, Y, metric=metric, p=p)
