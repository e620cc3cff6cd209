"""pairwise_distances with the reference's Python interface
(python_interface/python_package/aoclda/metrics.py) over
da_pairwise_distances_?."""
import numpy as np

from ._binding import ab, convert


def pairwise_distances(X, Y=None, metric="euclidean", p=2.0, check_data=False):
    """Distances between the rows of X and of Y (X with itself when Y is
    None): a numpy array of shape (m, n) in the precision of X."""
    X, prec, order = convert(X)
    Yc = None if Y is None else convert(Y, prec, order)[0]
    st, D = ab.pairwise_distances(X, Yc, metric=metric, p=float(p), prec=prec, order=order)
    if st != ab.SUCCESS:
        raise ab.DAError(st, "da_pairwise_distances")
    return np.ascontiguousarray(D)
