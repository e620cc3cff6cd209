"""Argument checks of da_nn_radius_neighbors_? that come before any device
work (the reference's order and statuses)."""
import numpy as np

INVALID_INPUT, NO_DATA, INCOMPATIBLE = 4, 20, 13


def test_radius_argument_checks(ab):
    L = ab.lib()
    Q = np.zeros((4, 3))
    nn = ab.KNN("d")
    # sort without distances
    assert L.da_nn_radius_neighbors_d(nn.h, 4, 3, ab.ptr(Q), 4, 1.0, 0, 1) == INVALID_INPUT
    # no training data
    assert L.da_nn_radius_neighbors_d(nn.h, 4, 3, ab.ptr(Q), 4, 1.0, 1, 0) == NO_DATA
    nn.close()
    ip = ab.KNN("d", metric="inner product").fit(np.ones((10, 3)))
    assert L.da_nn_radius_neighbors_d(ip.h, 4, 3, ab.ptr(Q), 4, 1.0, 1, 0) == INCOMPATIBLE
    ip.close()


def test_radius_predict_argument_checks(ab):
    """Radius-mode predict: an unknown search mode (4), inner product with
    distance weights (13), no labels / targets (20) -- all before device
    work."""
    L = ab.lib()
    Q = np.zeros((4, 3))
    y = np.zeros(4, dtype=np.int32)
    yr = np.zeros(4)
    X = np.ones((10, 3))
    nn = ab.KNN("d").fit(X)
    assert L.da_nn_classifier_predict_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(y), 1) == NO_DATA
    assert L.da_nn_regressor_predict_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(yr), 1) == NO_DATA
    nn.close()
    nn = ab.KNN("d").fit(X, y=np.arange(10, dtype=np.int32) % 3, targets=np.arange(10.0))
    pr = np.zeros((4, 3))
    assert L.da_nn_classifier_predict_proba_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(pr), 2) == \
        INVALID_INPUT
    assert L.da_nn_classifier_predict_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(y), 2) == INVALID_INPUT
    assert L.da_nn_regressor_predict_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(yr), 2) == INVALID_INPUT
    nn.close()
    nn = ab.KNN("d", metric="inner product", weights="distance")
    nn.fit(X, y=np.arange(10, dtype=np.int32) % 3, targets=np.arange(10.0))
    assert L.da_nn_classifier_predict_proba_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(pr), 1) == \
        INCOMPATIBLE
    assert L.da_nn_classifier_predict_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(y), 1) == INCOMPATIBLE
    assert L.da_nn_regressor_predict_d(nn.h, 4, 3, ab.ptr(Q), 4, ab.ptr(yr), 1) == INCOMPATIBLE
    # the outlier options take the reference's values, NaN target included
    assert nn.set("outlier handling", "most frequent") == 0
    assert nn.set("outlier label", -999) == 0
    assert nn.set("outlier target", float("nan")) == 0
    nn.close()
