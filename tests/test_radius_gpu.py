"""Radius neighbours (da_nn_radius_neighbors_?) on the GPU against the oracle
restatement of the reference's brute-force radius search: per query the
training rows within the radius, in index order or sorted by distance, and
their distances -- bit for bit (to an ulp of pow() for minkowski p = 3) --
for several metrics, both precisions and both storage orders; plus the
count / offsets / per-query result queries."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def data(rng, n, nq, d, dt):
    means = rng.uniform(-3, 3, (6, d))
    X = (means[rng.integers(0, 6, n)] + rng.standard_normal((n, d))).astype(dt)
    Q = (means[rng.integers(0, 6, nq)] + rng.standard_normal((nq, d))).astype(dt)
    X[5] = X[3]       # ties
    Q[0] = X[7]       # a query on a training row
    return X, Q


@pytest.mark.parametrize("metric,p,radius", [("euclidean", 2.0, 2.2), ("sqeuclidean", 2.0, 4.0),
                                              ("manhattan", 2.0, 4.5), ("cosine", 2.0, 0.08),
                                              ("minkowski", 3.0, 1.9), ("minkowski", 2.0, 2.2)])
@pytest.mark.parametrize("prec,order,sort", [("s", 1, False), ("d", 0, True), ("s", 0, True)])
def test_radius_matches_oracle(gpu, ab, orc, metric, p, radius, prec, order, sort):
    dt = np.float32 if prec == "s" else np.float64
    rng = np.random.default_rng(len(metric) + int(10 * p))
    X, Q = data(rng, 3000, 64, 7, dt)
    nn = ab.KNN(prec, order=order, metric=metric, minkowski_parameter=p).fit(X)
    cnt, off, ind, dist = nn.radius_neighbors(Q, radius, True, sort)
    ref = orc.radius(X, Q, radius, metric, p, sort)
    assert cnt[-1] == sum(len(r[0]) for r in ref) > 64
    for qi, (ri, rd) in enumerate(ref):
        assert cnt[qi] == len(ri)
        if len(ri) == 0:
            assert off[qi] == -1
            continue
        o = off[qi]
        np.testing.assert_array_equal(ind[o:o + len(ri)], ri)
        if metric == "minkowski" and p == 3.0:
            # pow() of the device and the host libm may differ by an ulp
            np.testing.assert_allclose(dist[o:o + len(ri)], rd, rtol=8 * np.finfo(dt).eps)
        else:
            np.testing.assert_array_equal(dist[o:o + len(ri)], rd.astype(dt))
    assert off[-1] == cnt[-1]
    nn.close()


def test_radius_result_queries(gpu, ab):
    rng = np.random.default_rng(9)
    X, Q = data(rng, 2000, 20, 5, np.float64)
    nn = ab.KNN("d", order=ab.ROW_MAJOR, radius=1.5).fit(X)
    cnt, off, ind, dist = nn.radius_neighbors(Q, -1.0, True, True)   # radius from the option
    L = ab.lib()
    q = 3
    buf = np.array([q] + [0] * (int(cnt[q]) + 3), dtype=np.int32)
    dim = ab.da_int(buf.size)
    assert L.da_handle_get_result_int(nn.h, ab.RNN_INDICES_INDEX, C.byref(dim), ab.ptr(buf)) == 0
    np.testing.assert_array_equal(buf[:cnt[q]], ind[off[q]:off[q] + cnt[q]])
    dbuf = np.zeros(int(cnt[q]) + 3)
    dbuf[0] = q
    dim = ab.da_int(dbuf.size)
    assert L.da_handle_get_result_d(nn.h, ab.RNN_DISTANCES_INDEX, C.byref(dim), ab.ptr(dbuf)) == 0
    np.testing.assert_array_equal(dbuf[:cnt[q]], dist[off[q]:off[q] + cnt[q]])
    assert np.all(np.diff(dist[off[q]:off[q] + cnt[q]]) >= 0)
    # too small an array: the size needed comes back with a warning
    small = np.zeros(1, dtype=np.int32)
    dim = ab.da_int(1)
    assert L.da_handle_get_result_int(nn.h, ab.RNN_INDICES, C.byref(dim), ab.ptr(small)) == 17
    assert dim.value == cnt[-1]
    # without distances, the distance queries report no data
    nn.radius_neighbors(Q, 1.5, False, False)
    dim = ab.da_int(dbuf.size)
    assert L.da_handle_get_result_d(nn.h, ab.RNN_DISTANCES, C.byref(dim), ab.ptr(dbuf)) == 20
    nn.close()


def test_radius_hand_problem(gpu, ab):
    """The reference's own radius-5 expectations on its hand problem."""
    from conftest import golden
    z = golden("nn_small.npz")
    r = float(z["radius"][0])
    for metric, pre in (("euclidean", "rad_euc"), ("sqeuclidean", "rad_sq")):
        nn = ab.KNN("d", algorithm="brute", metric=metric).fit(z["X_train"])
        cnt, off, ind, dist = nn.radius_neighbors(z["X_test"], r, True, True)
        np.testing.assert_array_equal(cnt[:-1], z[pre + "_cnt"])
        np.testing.assert_array_equal(ind, z[pre + "_ind"])
        np.testing.assert_allclose(dist, z[pre + "_dist"], rtol=40 * np.finfo(float).eps)
        nn.close()
