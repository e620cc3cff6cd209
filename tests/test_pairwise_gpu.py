"""da_pairwise_distances through the C ABI vs the oracle restatement of the
reference's packed distance kernels (bit-exact for the direct-difference and
dot-product families; Minkowski within a few ulp because pow() differs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

METRICS = ["euclidean", "sqeuclidean", "manhattan", "cosine", "euclidean_gemm",
           "sqeuclidean_gemm", "inner product"]


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("metric", METRICS)
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (23, 19, 8), (25, 32, 26), (130, 70, 257),
                                   (64, 128, 4), (300, 2, 600)])
def test_pairwise_vs_oracle(gpu, ab, orc, prec, order, metric, m, n, k):
    dt = np.float64 if prec == "d" else np.float32
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    X = rng.standard_normal((m, k)).astype(dt)
    Y = rng.standard_normal((n, k)).astype(dt)
    st, D = ab.pairwise_distances(X, Y, metric, prec=prec, order=order)
    assert st == 0
    want = orc.pairwise(X, Y, metric)
    if metric == "euclidean_gemm":
        # sqrt of a negative rounding residue is NaN in both
        np.testing.assert_array_equal(np.isnan(D), np.isnan(want))
        D, want = np.nan_to_num(D), np.nan_to_num(want)
    np.testing.assert_array_equal(D, want)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("metric", ["euclidean", "cosine", "euclidean_gemm", "sqeuclidean"])
def test_pairwise_x_is_y(gpu, ab, orc, prec, metric):
    dt = np.float64 if prec == "d" else np.float32
    X = np.random.default_rng(1).standard_normal((57, 9)).astype(dt)
    st, D = ab.pairwise_distances(X, None, metric, prec=prec)
    assert st == 0
    want = orc.pairwise(X, None, metric)
    np.testing.assert_array_equal(np.nan_to_num(D), np.nan_to_num(want))
    assert np.all(np.diag(D) == 0)


@pytest.mark.parametrize("p", [1.0, 2.0, 3.0, 0.5])
def test_pairwise_minkowski(gpu, ab, orc, p):
    X = np.random.default_rng(2).standard_normal((40, 13))
    Y = np.random.default_rng(3).standard_normal((30, 13))
    st, D = ab.pairwise_distances(X, Y, "minkowski", p=p)
    assert st == 0
    np.testing.assert_allclose(D, orc.pairwise(X, Y, "minkowski", p=p), rtol=1e-14)


def test_pairwise_errors(gpu, ab):
    X = np.zeros((4, 3))
    st, _ = ab.pairwise_distances(X, None, "minkowski", p=-1.0)
    assert st == 4
    st, _ = ab.pairwise_distances(np.zeros((0, 3)), None, "euclidean")
    assert st == 17
