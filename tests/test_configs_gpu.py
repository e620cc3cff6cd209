"""Parity at the benchmark configurations themselves, against the oracle.

* fp64 brute-force kNN, 10,000 x 32 training rows from a 16-component
  isotropic Gaussian mixture (means U[-5, 5]^32, sigma 1, labels = component
  id), 2,000 queries from the same mixture, seed 0, k = 10, euclidean,
  uniform weights: neighbour indices, distances and predicted labels equal
  the oracle's (nearest_neighbors.cpp:568-816, 1166-1272, 1489-1603).
* fp32 k-means, 1,000,000 x 64 from a 256-component mixture, k = 256,
  k-means++ from seed 1, max_iter 50, tol 1e-4, on the default tensor-core
  path: the initial centres are the oracle's k-means++ rows; the returned
  labels are the oracle's fp32 assignment to the returned centres; the
  inertia is their fp64 inertia to 1e-5; labels, centres and iteration count
  equal the plain fp32 path's.
* The kNN tensor-core pass against the oracle (not only against the plain
  path) above the size where the library switches to it: 200,000 x 128,
  256 queries, k = 100, euclidean and cosine.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def c1_data(seed=0, n=10_000, nq=2_000, d=32, comps=16):
    rng = np.random.default_rng(seed)
    means = rng.uniform(-5.0, 5.0, (comps, d))
    lab = rng.integers(0, comps, n)
    X = means[lab] + rng.standard_normal((n, d))
    ql = rng.integers(0, comps, nq)
    Q = means[ql] + rng.standard_normal((nq, d))
    return X, lab.astype(np.int64), Q


def c2_data(n=1_000_000, d=64, k=256, seed=1):
    rng = np.random.default_rng(seed)
    means = rng.uniform(-10.0, 10.0, (k, d))
    sig = rng.uniform(0.5, 2.0, k)
    w = rng.dirichlet(np.ones(k))
    lab = rng.choice(k, n, p=w)
    X = means[lab] + rng.standard_normal((n, d)) * sig[lab, None]
    return np.ascontiguousarray(X, dtype=np.float32)


def vote_uniform(ind, y):
    """Uniform-weight vote of the neighbours (predict_proba_compute_knn,
    nearest_neighbors.cpp:1166-1272) and the first class of maximal
    probability (cblas_iamax, :1489-1603); classes in sorted order."""
    classes = np.unique(y)
    pos = np.searchsorted(classes, y)
    counts = np.zeros((ind.shape[0], classes.size))
    for r in range(ind.shape[1]):
        np.add.at(counts, (np.arange(ind.shape[0]), pos[ind[:, r]]), 1.0)
    return classes[np.argmax(counts, axis=1)]


def tie_count(X, Q, ind, k):
    """Queries whose k-th and (k+1)-th fp64 distances differ by less than
    1e-12 relative: there the neighbour set depends on rounding or on the
    tie rule."""
    Xd, Qd = X.astype(np.float64), Q.astype(np.float64)
    n = 0
    for q in range(Q.shape[0]):
        d2 = ((Xd - Qd[q]) ** 2).sum(1)
        part = np.partition(d2, k)[: k + 1]
        part.sort()
        if part[k] - part[k - 1] <= 1e-12 * max(part[k], 1e-300):
            n += 1
    return n


@pytest.mark.parametrize("order", [0, 1])
def test_c1_knn_fp64_exact(gpu, ab, orc, order):
    X, y, Q = c1_data()
    k = 10
    nn = ab.KNN("d", order=order, metric="euclidean", weights="uniform",
                number_of_neighbors=k).fit(X, y=y)
    ind, dist = nn.kneighbors(Q, k)
    pred = nn.predict(Q)
    nn.close()
    oi, od = orc.knn(X, Q, k)
    np.testing.assert_array_equal(ind, oi)
    np.testing.assert_array_equal(dist, od)
    np.testing.assert_array_equal(pred, vote_uniform(oi, y))
    # the labels of this mixture are well separated: no near-ties at the k-th place
    assert tie_count(X, Q[:200], oi[:200], k) == 0


def test_c2_kmeans_1M_bf16x3_vs_oracle(gpu, ab, orc):
    n, d, k = 1_000_000, 64, 256
    X = c2_data(n, d, k)
    km = ab.KMeans(k, "s", order=ab.ROW_MAJOR, max_iter=50, n_init=1, seed=1)
    km.set("convergence tolerance", 1e-4)
    km.set_data(X)
    C0 = km.init_centres(k)
    chosen = orc.kmeanspp(X, k, 1)
    np.testing.assert_array_equal(C0, X[chosen])
    assert km.stat("tensor_core") in (0.0, 1.0)
    out = {}
    for mode in ("bf16x3", "plain"):
        h = ab.KMeans(k, "s", order=ab.ROW_MAJOR, max_iter=50, n_init=1)
        h.set("convergence tolerance", 1e-4)
        h.set("precision mode", mode)
        h.fit(X, C0=C0)
        out[mode] = (h.labels(n), h.centres(k, d), h.rinfo(), h.stat("tensor_core"))
        h.close()
    km.close()
    lab, C, r, tc = out["bf16x3"]
    assert tc == 1.0 and out["plain"][3] == 0.0
    np.testing.assert_array_equal(lab, out["plain"][0])
    np.testing.assert_array_equal(C, out["plain"][1])
    np.testing.assert_array_equal(r, out["plain"][2])
    lab_o, _ = orc.kmeans_assign(X, C)
    np.testing.assert_array_equal(lab, lab_o)
    inertia64 = orc.kmeans_inertia(X, lab, C.astype(np.float64))
    assert abs(r[4] - inertia64) <= 1e-5 * inertia64


@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
def test_knn_tensor_core_vs_oracle(gpu, ab, orc, metric):
    rng = np.random.default_rng(17)
    nx, nq, d, k, comps = 200_000, 256, 128, 100, 256
    means = rng.uniform(-10.0, 10.0, (comps, d))
    sig = rng.uniform(0.5, 2.0, comps)
    lab = rng.integers(0, comps, nx)
    X = (means[lab] + rng.standard_normal((nx, d)) * sig[lab, None]).astype(np.float32)
    dup = rng.integers(0, nx, nx // 100)          # 1% exact duplicates: ties
    X[rng.integers(0, nx, dup.size)] = X[dup]
    ql = rng.integers(0, comps, nq)
    Q = (means[ql] + rng.standard_normal((nq, d)) * sig[ql, None]).astype(np.float32)
    nn = ab.KNN("s", order=ab.ROW_MAJOR, metric=metric, precision_mode="bf16x3").fit(X)
    ind, dist = nn.kneighbors(Q, k)
    assert nn.stat("tensor_core") == 1.0
    nn.close()
    oi, od = orc.knn(X, Q, k, metric=metric)
    np.testing.assert_array_equal(ind, oi)
    np.testing.assert_array_equal(dist, od)
