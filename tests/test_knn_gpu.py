"""Parity of the GPU kNN path (C-ABI calls) with the oracle and the reference's
golden vectors.  Distances of the direct-difference metrics are bit-exact to
the reference's summation order; neighbour indices are exact under the
(distance, index) order, which differs from the reference only on exact ties
(counted with fp64 distances)."""
import numpy as np
import pytest

from conftest import golden
from test_oracle_golden import classify_mismatch

pytestmark = pytest.mark.gpu


def mixture(rng, n, d, comps=8, scale=5.0, dtype=np.float64):
    means = rng.uniform(-scale, scale, (comps, d))
    lab = rng.integers(0, comps, n)
    return (means[lab] + rng.standard_normal((n, d))).astype(dtype), lab.astype(np.int32)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("metric", ["euclidean", "sqeuclidean", "manhattan"])
@pytest.mark.parametrize("nx,nq,d,k", [(1000, 77, 32, 10), (333, 65, 5, 1), (2500, 130, 130, 100),
                                       (700, 9, 3, 7), (129, 64, 300, 33)])
def test_knn_bitexact_vs_oracle(gpu, ab, orc, dtype, order, metric, nx, nq, d, k):
    rng = np.random.default_rng(nx + nq + d + k)
    X, _ = mixture(rng, nx, d, dtype=dtype)
    Q, _ = mixture(rng, nq, d, dtype=dtype)
    nn = ab.KNN("d" if dtype == np.float64 else "s", order=order, metric=metric,
                algorithm="brute").fit(X)
    ind, dist = nn.kneighbors(Q, k)
    oi, od = orc.knn(X, Q, k, metric)
    np.testing.assert_array_equal(dist, od)  # bit-exact
    np.testing.assert_array_equal(ind, oi)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("metric,p", [("cosine", 2.0), ("minkowski", 3.0), ("minkowski", 1.0),
                                      ("minkowski", 2.0), ("euclidean_gemm", 2.0),
                                      ("sqeuclidean_gemm", 2.0), ("inner product", 2.0)])
def test_knn_other_metrics(gpu, ab, orc, dtype, metric, p):
    rng = np.random.default_rng(7)
    X, _ = mixture(rng, 900, 24, dtype=dtype)
    Q, _ = mixture(rng, 70, 24, dtype=dtype)
    nn = ab.KNN("d" if dtype == np.float64 else "s", metric=metric, algorithm="brute",
                minkowski_parameter=p).fit(X)
    ind, dist = nn.kneighbors(Q, 12)
    oi, od = orc.knn(X, Q, 12, metric, p=p)
    if metric == "minkowski" and p == 3.0:
        # pow() of the device and the host libm may differ by an ulp
        np.testing.assert_allclose(dist, od, rtol=8 * np.finfo(dtype).eps)
        assert (ind != oi).mean() < 0.01
    else:
        np.testing.assert_array_equal(dist, od)
        np.testing.assert_array_equal(ind, oi)


@pytest.mark.parametrize("tag", ["2092x2071x5", "2125x2068x20"])
@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("order", [0, 1])
def test_knn_golden_csv(gpu, ab, tag, prec, order):
    z = golden(f"nn_{tag}.npz")
    dt = np.float64 if prec == "d" else np.float32
    X = z["X_train"].astype(dt)
    Q = z["X_test"].astype(dt)
    eps = np.finfo(dt).eps
    nn = ab.KNN(prec, order=order, algorithm="brute", number_of_neighbors=5)
    nn.fit(X, y=z["y_train"].astype(np.int32), targets=z["y_train"].astype(dt))
    ind, dist = nn.kneighbors(Q, 5)
    np.testing.assert_allclose(dist, z["k_dist"], rtol=500 * eps, atol=500 * eps)
    d64 = np.sqrt(((Q.astype(np.float64)[:, None, :] - X.astype(np.float64)[None]) ** 2).sum(-1))
    assert classify_mismatch(X, Q, ind, z["k_ind"], d64) == 0
    np.testing.assert_allclose(nn.predict_proba(Q), z["proba_uniform"], rtol=500 * eps,
                               atol=500 * eps)
    np.testing.assert_array_equal(nn.predict(Q), z["class_uniform"])
    np.testing.assert_allclose(nn.predict_reg(Q), z["reg_uniform"], rtol=500 * eps, atol=500 * eps)


@pytest.mark.parametrize("tag", ["2092x2071x5", "2125x2068x20"])
def test_knn_golden_csv_distance_weights(gpu, ab, tag):
    z = golden(f"nn_{tag}.npz")
    nn = ab.KNN("d", algorithm="brute", number_of_neighbors=5, weights="distance")
    nn.fit(z["X_train"], y=z["y_train"].astype(np.int32), targets=z["y_train"])
    eps = np.finfo(float).eps
    np.testing.assert_allclose(nn.predict_proba(z["X_test"]), z["proba_distance"],
                               rtol=500 * eps, atol=500 * eps)
    np.testing.assert_array_equal(nn.predict(z["X_test"]), z["class_distance"])
    np.testing.assert_allclose(nn.predict_reg(z["X_test"]), z["reg_distance"], rtol=500 * eps,
                               atol=500 * eps)


def test_knn_small_hand_problem(gpu, ab):
    z = golden("nn_small.npz")
    for k, ki, kd in ((3, "kind3", "kdist3"), (4, "kind4", "kdist4")):
        nn = ab.KNN("d", algorithm="brute").fit(z["X_train"])
        ind, dist = nn.kneighbors(z["X_test"], k)
        want_d = z[kd].reshape(k, 3).T
        np.testing.assert_allclose(dist, want_d, rtol=40 * np.finfo(float).eps)
        d64 = np.sqrt(((z["X_test"][:, None] - z["X_train"][None]) ** 2).sum(-1))
        assert classify_mismatch(None, None, ind, z[ki].reshape(k, 3).T, d64) == 0


def test_knn_batch_invariance(gpu, ab):
    """A query's neighbours and distances do not depend on the batch it is in."""
    rng = np.random.default_rng(11)
    X, _ = mixture(rng, 5000, 48, dtype=np.float32)
    Q, _ = mixture(rng, 300, 48, dtype=np.float32)
    nn = ab.KNN("s", algorithm="brute").fit(X)
    ind_all, dist_all = nn.kneighbors(Q, 20)
    for lo, hi in ((0, 1), (17, 18), (5, 133), (250, 300)):
        i, d = nn.kneighbors(Q[lo:hi], 20)
        np.testing.assert_array_equal(i, ind_all[lo:hi])
        np.testing.assert_array_equal(d, dist_all[lo:hi])


def test_knn_duplicates_ties_lower_index(gpu, ab):
    """Exact duplicate training rows: ties resolve to the lower index."""
    rng = np.random.default_rng(5)
    base = rng.standard_normal((400, 16)).astype(np.float32)
    X = np.concatenate([base, base[::-1]])  # every row twice
    nn = ab.KNN("s", algorithm="brute").fit(X)
    ind, dist = nn.kneighbors(base[:50], 6)
    for q in range(50):
        for r in range(0, 6, 2):
            assert dist[q, r] == dist[q, r + 1]
            assert ind[q, r] < ind[q, r + 1]


def test_knn_k_equals_n_and_large_k(gpu, ab, orc):
    rng = np.random.default_rng(9)
    X = rng.standard_normal((256, 8))
    Q = rng.standard_normal((20, 8))
    nn = ab.KNN("d", algorithm="brute").fit(X)
    ind, dist = nn.kneighbors(Q, 128)
    oi, od = orc.knn(X, Q, 128)
    np.testing.assert_array_equal(ind, oi)
    np.testing.assert_array_equal(dist, od)
    X2 = rng.standard_normal((100, 8)).astype(np.float32)
    nn2 = ab.KNN("s", algorithm="brute").fit(X2)
    ind, dist = nn2.kneighbors(X2[:5], 100)
    oi, od = orc.knn(X2, X2[:5], 100)
    np.testing.assert_array_equal(ind, oi)
