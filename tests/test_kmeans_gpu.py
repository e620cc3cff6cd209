"""Parity of the GPU k-means path (C-ABI calls) with the reference's golden
case and the oracle.  Labels: exact except near-ties (classified with fp64
distances); centres and inertia: relative error 1e-5 (fp32) / 1e-12 (fp64)
against the fp64 oracle evaluated on the same labels."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def gmm(rng, n, d, k, lo=-10, hi=10, dtype=np.float32):
    means = rng.uniform(lo, hi, (k, d))
    sig = rng.uniform(0.5, 2.0, k)
    w = rng.dirichlet(np.ones(k))
    lab = rng.choice(k, n, p=w)
    return (means[lab] + rng.standard_normal((n, d)) * sig[lab, None]).astype(dtype)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("order", [1, 0])
def test_kmeans_lloyd80_golden(gpu, ab, prec, order):
    z = golden("kmeans_lloyd80.npz")
    km = ab.KMeans(16, prec, order=order, max_iter=30, n_init=1)
    km.set("convergence tolerance", 1e-4)
    km.fit(z["A"], C0=z["C"])
    r = km.rinfo()
    assert list(r[:4]) == [80, 2, 16, 4]
    assert abs(r[4] - 45.78715) < 1e-4 * 45.78715
    np.testing.assert_array_equal(km.labels(80), z["expected_labels"])
    np.testing.assert_allclose(km.centres(16, 2), z["expected_centres"], rtol=1e-4, atol=1e-4)
    assert list(km.predict(z["Y"])) == list(z["expected_Y_labels"])
    tr = km.transform(z["X"], 16)
    np.testing.assert_allclose(tr, z["expected_X_transform"], rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("n,d,k", [(20000, 64, 37), (5000, 3, 8), (12345, 130, 100), (3000, 16, 300)])
def test_kmeans_supplied_vs_oracle_fp32(gpu, ab, orc, n, d, k):
    rng = np.random.default_rng(n + d + k)
    A = gmm(rng, n, d, k)
    C0 = A[rng.choice(n, k, replace=False)].copy()
    km = ab.KMeans(k, "s", order=0, max_iter=40, n_init=1)
    km.fit(A, C0=C0)
    C, lab, nit, inertia = orc.kmeans_lloyd(A, C0, max_iter=40, tol=1e-4)
    r = km.rinfo()
    glab = km.labels(n)
    gC = km.centres(k, d)
    if np.array_equal(glab, lab):
        assert int(r[3]) == nit
        np.testing.assert_allclose(gC, C, rtol=1e-5, atol=1e-5 * np.abs(C).max())
    # Whatever the trajectory, the returned labels are the fp32 assignment to
    # the returned centres (same fma order as the oracle -> exact), and the
    # inertia is their fp64 inertia.
    lab2, gap = orc.kmeans_assign(A, gC)
    np.testing.assert_array_equal(glab, lab2)
    inertia64 = orc.kmeans_inertia(A, glab, gC.astype(np.float64))
    assert abs(r[4] - inertia64) <= 1e-5 * inertia64


@pytest.mark.parametrize("n,d,k", [(4000, 8, 12), (999, 33, 5)])
def test_kmeans_supplied_vs_oracle_fp64(gpu, ab, orc, n, d, k):
    rng = np.random.default_rng(n * d)
    A = gmm(rng, n, d, k, dtype=np.float64)
    C0 = A[rng.choice(n, k, replace=False)].copy()
    km = ab.KMeans(k, "d", order=1, max_iter=100, n_init=1)
    km.fit(A, C0=C0)
    C, lab, nit, inertia = orc.kmeans_lloyd(A, C0, max_iter=100, tol=1e-4)
    np.testing.assert_array_equal(km.labels(n), lab)
    assert int(km.rinfo()[3]) == nit
    np.testing.assert_allclose(km.centres(k, d), C, rtol=1e-12, atol=1e-12)
    assert abs(km.rinfo()[4] - inertia) <= 1e-12 * inertia


def test_kmeans_step_labels_and_update(gpu, ab, orc):
    """One iteration from supplied centres: labels == oracle (fp32 formula),
    centres == fp64 means of those labels."""
    rng = np.random.default_rng(21)
    n, d, k = 50000, 64, 256
    A = gmm(rng, n, d, 64)
    C0 = A[rng.choice(n, k, replace=False)].copy()
    km = ab.KMeans(k, "s", order=0, max_iter=1, n_init=1)
    km.fit(A, C0=C0, ok=(0, 21))
    lab0, gap0 = orc.kmeans_assign(A, C0)
    Cn, cnt = orc.kmeans_update(A, lab0, k)
    np.testing.assert_allclose(km.centres(k, d), Cn.astype(np.float32), rtol=1e-6, atol=1e-6)


def test_kmeans_kmeanspp_and_random_inits_run(gpu, ab):
    rng = np.random.default_rng(1)
    A = gmm(rng, 20000, 16, 20)
    for init in ("k-means++", "random", "random partitions", "afk-mc2"):
        km = ab.KMeans(20, "s", order=0, max_iter=50, n_init=2, seed=1)
        km.set("initialization method", init)
        km.fit(A)
        r = km.rinfo()
        lab = km.labels(20000)
        assert r[4] > 0 and lab.min() >= 0 and lab.max() < 20
    # same seed -> identical result (deterministic device reductions)
    outs = []
    for _ in range(2):
        km = ab.KMeans(20, "s", order=0, max_iter=50, n_init=1, seed=7)
        km.fit(A)
        outs.append((km.labels(20000), km.centres(20, 16), km.rinfo()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    np.testing.assert_array_equal(outs[0][2], outs[1][2])


def test_kmeans_empty_cluster_modes(gpu, ab):
    A = np.asfortranarray(np.array([[0.0, 0.0], [0.1, 0.0], [10.0, 10.0], [10.1, 10.0]]))
    C0 = np.asfortranarray(np.array([[0.0, 0.0], [10.0, 10.0], [100.0, 100.0]]))
    km = ab.KMeans(3, "d", max_iter=10)
    km.fit(A, C0=C0)
    c = km.centres(3, 2)
    np.testing.assert_allclose(c[2], [0.0, 0.0])  # empty cluster -> zero vector
    km = ab.KMeans(3, "d", max_iter=10)
    km.set("empty clusters", "error")
    km.fit(A, C0=C0, ok=(900,))
    km = ab.KMeans(3, "d", max_iter=10)
    km.set("empty clusters", "split")
    km.fit(A, C0=C0)
    assert len(set(km.labels(4))) == 3


@pytest.mark.parametrize("n,d,k", [(100000, 64, 256), (33333, 37, 100), (20000, 128, 64),
                                   (5000, 200, 16), (70000, 96, 250), (4000, 8, 3)])
def test_kmeans_bf16_tensor_core_equals_plain(gpu, ab, n, d, k):
    """Both BF16 tensor-core candidate passes (one term, three-term split) must
    return exactly the plain fp32 path's labels, centres, iteration count and
    inertia."""
    rng = np.random.default_rng(n + k)
    A = gmm(rng, n, d, max(k // 2, 2))
    C0 = A[rng.choice(n, k, replace=False)].copy()
    out = {}
    for mode in ("plain", "bf16", "bf16x3"):
        km = ab.KMeans(k, "s", order=0, max_iter=25, n_init=1)
        km.set("precision mode", mode)
        km.fit(A, C0=C0)
        out[mode] = (km.labels(n), km.centres(k, d), km.rinfo())
    for mode in ("bf16", "bf16x3"):
        np.testing.assert_array_equal(out["plain"][0], out[mode][0])
        np.testing.assert_array_equal(out["plain"][1], out[mode][1])
        np.testing.assert_array_equal(out["plain"][2], out[mode][2])
