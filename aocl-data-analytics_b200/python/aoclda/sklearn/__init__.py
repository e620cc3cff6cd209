"""scikit-learn patch: skpatch() replaces sklearn's NearestNeighbors,
KNeighborsClassifier / Regressor, RadiusNeighborsClassifier / Regressor,
KMeans and pairwise_distances by the B200 classes
(python_package/aoclda/sklearn/patch_sklearn.py), undo_skpatch() restores
them."""
from .patch_sklearn import skpatch, undo_skpatch  # noqa: F401
