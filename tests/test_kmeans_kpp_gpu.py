"""k-means++ initial centres of the GPU handle against the oracle's
restatement of kmeans.cpp:1491-1664 (the reference's std::mt19937_64 engine,
std::discrete_distribution draws and candidate costs): the same rows, for
several seeds, fp32 and fp64, row- and column-major data.  The device maps
the engine's draws to rows through a certified parallel prefix and redoes
uncertain draws with the reference's sequential sums; with
AOCLDA_B200_KPP_EXACT_DRAWS=1 every draw takes the sequential path, which
must give the same rows."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gmm(rng, n, d, comps, dtype):
    means = rng.uniform(-10.0, 10.0, (comps, d))
    sig = rng.uniform(0.5, 2.0, comps)
    w = rng.dirichlet(np.ones(comps))
    lab = rng.choice(comps, n, p=w)
    return (means[lab] + rng.standard_normal((n, d)) * sig[lab, None]).astype(dtype)


def gpu_chosen(ab, X, k, seed, prec, order):
    km = ab.KMeans(k, prec, order=order, n_init=1, seed=seed)
    km.set("initialization method", "k-means++")
    km.set_data(X)
    C0 = km.init_centres(k)
    exact = km.stat("kmeans_pp_exact_draws")
    km.close()
    # every centre is a row of X: find which
    Xc = np.ascontiguousarray(X)
    rows = {Xc[i].tobytes(): i for i in range(Xc.shape[0] - 1, -1, -1)}
    return np.array([rows[np.ascontiguousarray(c).tobytes()] for c in C0]), exact


@pytest.mark.parametrize("seed", [0, 1, 7])
@pytest.mark.parametrize("prec,order", [("s", 1), ("d", 0)])
def test_kmeanspp_matches_oracle(gpu, ab, orc, seed, prec, order):
    rng = np.random.default_rng(100 + seed)
    dt = np.float32 if prec == "s" else np.float64
    X = gmm(rng, 50_000, 64, 64, dt)
    k = 64
    want = orc.kmeanspp(X, k, seed)
    got, _ = gpu_chosen(ab, X, k, seed, prec, order)
    np.testing.assert_array_equal(got, want)


def test_kmeanspp_exact_draw_path(gpu, ab, orc):
    rng = np.random.default_rng(5)
    X = gmm(rng, 20_000, 16, 20, np.float32)
    want = orc.kmeanspp(X, 40, 3)
    os.environ["AOCLDA_B200_KPP_EXACT_DRAWS"] = "1"
    try:
        got, exact = gpu_chosen(ab, X, 40, 3, "s", 1)
    finally:
        del os.environ["AOCLDA_B200_KPP_EXACT_DRAWS"]
    assert exact == 39 * (2 + int(np.log(40)))
    np.testing.assert_array_equal(got, want)


def test_kmeanspp_coincident_rows(gpu, ab, orc):
    X = np.ones((500, 3), dtype=np.float64)
    got = ab.KMeans(4, "d", order=1, n_init=1, seed=2)
    got.set("initialization method", "k-means++")
    got.set_data(X)
    C0 = got.init_centres(4)
    got.close()
    np.testing.assert_array_equal(C0, X[:4])
    np.testing.assert_array_equal(orc.kmeanspp(X, 4, 2), np.arange(4))
