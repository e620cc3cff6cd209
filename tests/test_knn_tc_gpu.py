"""The tensor-core kNN path (bf16x3 candidate pass with a certified per-query
threshold, exact re-score; euclidean, squared euclidean and cosine) against
the plain fp32 SIMT path on the same data:
neighbour indices and distances must be identical (bit for bit), including
rows duplicated to force exact ties.  Sizes are large enough that the
library chooses the tensor-core pass (it reports it through the
"tensor_core" statistic)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixture(rng, n, d, comps, scale=5.0):
    means = rng.uniform(-scale, scale, (comps, d))
    lab = rng.integers(0, comps, n)
    return (means[lab] + rng.standard_normal((n, d))).astype(np.float32)


def run(ab, X, Q, k, metric, mode, order):
    nn = ab.KNN("s", order=order, metric=metric, precision_mode=mode).fit(X)
    ind, dist = nn.kneighbors(Q, k)
    used_tc = nn.stat("tensor_core")
    fallback = nn.stat("knn_tc_fallback_queries")
    nn.close()
    return ind, dist, used_tc, fallback


@pytest.mark.parametrize("nx,nq,d,k,metric,order", [
    (200_000, 700, 128, 100, "euclidean", 0),
    (150_000, 300, 100, 10, "sqeuclidean", 0),
    (140_000, 1_025, 32, 1, "euclidean", 1),
    (130_000, 600, 64, 256, "euclidean", 0),
    (300_000, 40, 64, 10, "euclidean", 0),       # 64-query tiles
    (180_000, 100, 96, 100, "sqeuclidean", 0),   # 128-query tiles
    (300_000, 1, 64, 1, "euclidean", 1),
    (1_000_000, 1, 96, 100, "euclidean", 0),     # one query, all blocks on its list
    (600_000, 3, 64, 256, "sqeuclidean", 1),
    (220_000, 70, 80, 10, "euclidean", 0),       # last K block of 16 columns
    (200_000, 50, 96, 10, "cosine", 1),          # last K block of 32 columns
    (200_000, 700, 128, 100, "cosine", 0),
    (300_000, 40, 64, 10, "cosine", 1),
])
def test_knn_tc_equals_plain(gpu, ab, nx, nq, d, k, metric, order):
    rng = np.random.default_rng(nx + nq + d + k)
    X = mixture(rng, nx, d, comps=64)
    dup = rng.integers(0, nx, nx // 100)       # 1% exact duplicates -> ties
    X[rng.integers(0, nx, dup.size)] = X[dup]
    Q = mixture(rng, nq, d, comps=64)
    Q[:min(5, nq)] = X[:min(5, nq)]             # queries that hit training rows
    pi, pd, ptc, _ = run(ab, X, Q, k, metric, "plain", order)
    ti, td, ttc, fb = run(ab, X, Q, k, metric, "bf16x3", order)
    assert ptc == 0.0
    assert ttc == 1.0 and fb == 0.0
    np.testing.assert_array_equal(td, pd)
    np.testing.assert_array_equal(ti, pi)


def test_knn_tc_fallback_queries(gpu, ab):
    """Queries whose candidates the tensor-core pass cannot resolve (here: 10,000
    copies of one row at the query's own position, more exact ties than its
    re-score holds) are searched on the plain path alone; all results still
    equal the plain path's."""
    rng = np.random.default_rng(11)
    nx, nq, d, k = 200_000, 600, 64, 10
    X = mixture(rng, nx, d, comps=64)
    X[rng.choice(nx, 10000, replace=False)] = X[0]
    Q = mixture(rng, nq, d, comps=64)
    Q[[3, 77, 500]] = X[0]
    pi, pd, _, _ = run(ab, X, Q, k, "euclidean", "plain", 0)
    ti, td, ttc, fb = run(ab, X, Q, k, "euclidean", "bf16x3", 0)
    assert ttc == 1.0 and fb >= 3.0
    np.testing.assert_array_equal(td, pd)
    np.testing.assert_array_equal(ti, pi)
