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
