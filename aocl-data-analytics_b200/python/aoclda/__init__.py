"""B200 drop-in for the parts of the ``aoclda`` Python package that sit on
the distance / nearest-neighbour / k-means path
(python_interface/python_package/aoclda/neighbors.py, clustering.py,
sklearn/_neighbors.py, sklearn/_kmeans.py, faiss/*.py): the same class
names, arguments and return values, each call going through
libaoclda_b200.so's C ABI with host numpy arrays.  There is no CPU path: if
the library is not built, importing this package raises.

Put ``aocl-data-analytics_b200/python`` on ``sys.path`` (or PYTHONPATH) in
place of the reference package.
"""
from ._binding import ab  # noqa: F401
from . import clustering, neighbors  # noqa: F401

__all__ = ["neighbors", "clustering"]
