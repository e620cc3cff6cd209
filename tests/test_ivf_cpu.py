"""Argument checks of the IVF-flat handle (da_approx_nn_*) that come before
any device work, with the reference's statuses (approximate_neighbors.cpp:
152-274, 525-560, 858-920)."""
import numpy as np
import pytest

INVALID_HANDLE_TYPE, WRONG_TYPE, INVALID_DIM, NO_DATA = 9, 7, 17, 20


def test_ivf_argument_checks(ab):
    L = ab.lib()
    X = np.random.default_rng(0).standard_normal((50, 3))
    a = ab.ApproxNN("d", n_list=2, n_probe=1)
    assert L.da_approx_nn_train_d(a.h) == NO_DATA                  # no training data
    a.set_training_data(X)
    for call in (lambda: a.kneighbors(X[:2], 2), lambda: a.add(X)):
        with pytest.raises(ab.DAError) as e:                       # nothing trained
            call()
        assert e.value.status == NO_DATA
    # single-precision entry point on a double handle
    assert L.da_approx_nn_train_s(a.h) == WRONG_TYPE
    a.close()
    # n_list above the number of rows
    b = ab.ApproxNN("d", n_list=60)
    b.set_training_data(X)
    with pytest.raises(ab.DAError) as e:
        b.train()
    assert e.value.status == INVALID_DIM
    b.close()
    # a kNN handle is not an IVF handle
    nn = ab.KNN("d")
    assert L.da_approx_nn_train_d(nn.h) == INVALID_HANDLE_TYPE
    nn.close()


def test_ivf_options(ab):
    a = ab.ApproxNN("s", n_list=7, n_probe=3, kmeans_iter=25, seed=-1, train_fraction=0.5,
                    number_of_neighbors=4)
    assert (a.get_int("n_list"), a.get_int("n_probe"), a.get_int("k-means_iter"),
            a.get_int("seed"), a.get_int("number of neighbors")) == (7, 3, 25, -1, 4)
    assert a.get_string("metric") == "sqeuclidean" and a.get_string("algorithm") == "ivfflat"
    assert a.set("train fraction", 0.0) != 0      # (0, 1]
    assert a.set("n_list", 0) != 0
    a.close()
