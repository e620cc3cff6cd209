"""Batched k-means (da_b200_kmeans_batched_s): every data set of the batch
must give exactly what da_kmeans_compute_s gives on its own with "precision
mode" = "plain", supplied initial centres, n_init = 1 -- the same labels,
centres and iteration count (the inertia to within fp64 rounding of a
different summation order: relative 1e-12)."""
import numpy as np
import pytest


def mixture(rng, n, d, comps):
    means = rng.uniform(-10.0, 10.0, (comps, d))
    sig = rng.uniform(0.5, 2.0, comps)
    lab = rng.integers(0, comps, n)
    return (means[lab] + rng.standard_normal((n, d)) * sig[lab, None]).astype(np.float32)


def make_batch(seed, count):
    rng = np.random.default_rng(seed)
    Xs, C0s = [], []
    for _ in range(count):
        n = int(np.clip(rng.lognormal(np.log(4000), 0.8), 300, 30000))
        d = int(rng.choice([3, 16, 32, 64, 100, 128]))
        k = int(rng.integers(2, 65))
        X = mixture(rng, n, d, k)
        C0 = X[rng.choice(n, k, replace=False)].copy()
        Xs.append(X)
        C0s.append(C0)
    return Xs, C0s


@pytest.mark.gpu
@pytest.mark.parametrize("seed,count,max_iter,tol", [(1, 24, 30, 1e-4), (2, 9, 5, 0.0),
                                                     (3, 6, 300, 1e-6)])
def test_batched_equals_single(gpu, ab, seed, count, max_iter, tol):
    Xs, C0s = make_batch(seed, count)
    out = ab.kmeans_batched(Xs, C0s, max_iter=max_iter, tol=tol)
    for X, C0, r in zip(Xs, C0s, out):
        n, d = X.shape
        k = C0.shape[0]
        km = ab.KMeans(k, "s", order=ab.ROW_MAJOR, max_iter=max_iter, n_init=1)
        km.set("convergence tolerance", tol)
        km.set("precision mode", "plain")
        km.fit(X, C0)
        info = km.rinfo()
        assert int(info[3]) == r["n_iter"]
        np.testing.assert_array_equal(km.labels(n), r["labels"])
        np.testing.assert_array_equal(km.centres(k, d), r["centres"])
        assert abs(info[4] - r["inertia"]) <= 1e-12 * max(1.0, abs(info[4]))
        km.close()


def test_batched_argument_checks(ab):
    import ctypes as C
    L = ab.lib()
    nil = C.c_void_p()
    assert L.da_b200_kmeans_batched_s(0, nil, nil, nil, nil, nil, nil, 10, C.c_double(1e-4), nil,
                                      nil, nil, nil, nil, None) == 17  # invalid_array_dimension
    assert L.da_b200_kmeans_batched_s(1, None, None, None, None, None, None, 10,
                                      C.c_double(1e-4), None, None, None, None, None,
                                      None) == 3  # invalid_pointer


@pytest.mark.gpu
def test_batched_timing_and_one_at_a_time(gpu, ab):
    """The device timings of the last call are reported, and a data set
    fitted alone (other tile shapes' groups absent) gives the same result as
    in the batch."""
    Xs, C0s = make_batch(5, 8)
    out = ab.kmeans_batched(Xs, C0s, max_iter=20, tol=1e-4)
    up, fit, down = ab.kmeans_batched_timing()
    assert up > 0.0 and fit > 0.0 and down > 0.0
    for X, C0, r in zip(Xs, C0s, out):
        r1 = ab.kmeans_batched([X], [C0], max_iter=20, tol=1e-4)[0]
        assert r1["n_iter"] == r["n_iter"]
        np.testing.assert_array_equal(r1["labels"], r["labels"])
        np.testing.assert_array_equal(r1["centres"], r["centres"])
        assert r1["inertia"] == r["inertia"]
