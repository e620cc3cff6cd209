"""The ``aoclda`` drop-in Python package on the GPU: nearest_neighbors,
kmeans, approximate_neighbors, pairwise_distances and the scikit-learn /
faiss classes return the oracle's results (bit for bit where the library
path is bit-exact), and the scikit-learn estimators agree with stock
scikit-learn on the same data."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def data(rng, n, nq, d, dt=np.float64):
    means = rng.uniform(-4, 4, (5, d))
    X = (means[rng.integers(0, 5, n)] + rng.standard_normal((n, d))).astype(dt)
    Q = (means[rng.integers(0, 5, nq)] + rng.standard_normal((nq, d))).astype(dt)
    return X, Q


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("fortran", [False, True])
def test_nearest_neighbors_matches_oracle(gpu, da, orc, dt, fortran):
    from aoclda.neighbors import nearest_neighbors
    rng = np.random.default_rng(1)
    X, Q = data(rng, 3000, 200, 9, dt)
    if fortran:
        X, Q = np.asfortranarray(X), np.asfortranarray(Q)
    nn = nearest_neighbors(n_neighbors=7).fit(X)
    dist, ind = nn.kneighbors(Q)
    oi, od = orc.knn(np.ascontiguousarray(X), np.ascontiguousarray(Q), 7)
    np.testing.assert_array_equal(ind, oi)
    np.testing.assert_array_equal(dist, od)
    assert dist.dtype == dt
    ind_only = nn.kneighbors(Q, n_neighbors=3, return_distance=False)
    np.testing.assert_array_equal(ind_only, oi[:, :3])
    rd, ri = nn.radius_neighbors(Q[:20], radius=2.0, sort_results=True)
    ref = orc.radius(np.ascontiguousarray(X), np.ascontiguousarray(Q[:20]), 2.0, sort=True)
    for q in range(20):
        np.testing.assert_array_equal(ri[q], ref[q][0])
        np.testing.assert_array_equal(rd[q], ref[q][1].astype(dt))


def test_classifier_regressor_match_sklearn(gpu, da):
    import sklearn.neighbors as skn
    from aoclda.sklearn import _neighbors as dan
    rng = np.random.default_rng(2)
    X, Q = data(rng, 2000, 300, 6)
    y = rng.integers(0, 4, len(X)).astype(np.int64)
    t = rng.standard_normal(len(X))
    for w in ("uniform", "distance"):
        a = dan.KNeighborsClassifier(n_neighbors=9, weights=w).fit(X, y)
        b = skn.KNeighborsClassifier(n_neighbors=9, weights=w, algorithm="brute").fit(X, y)
        np.testing.assert_allclose(a.predict_proba(Q), b.predict_proba(Q), rtol=1e-12, atol=1e-12)
        np.testing.assert_array_equal(a.predict(Q), b.predict(Q))
        a = dan.KNeighborsRegressor(n_neighbors=9, weights=w).fit(X, t)
        b = skn.KNeighborsRegressor(n_neighbors=9, weights=w, algorithm="brute").fit(X, t)
        np.testing.assert_allclose(a.predict(Q), b.predict(Q), rtol=1e-12, atol=1e-12)
        a = dan.RadiusNeighborsClassifier(radius=3.0, weights=w, outlier_label=1).fit(X, y)
        b = skn.RadiusNeighborsClassifier(radius=3.0, weights=w, outlier_label=1,
                                          algorithm="brute").fit(X, y)
        np.testing.assert_array_equal(a.predict(Q), b.predict(Q))
        a = dan.RadiusNeighborsRegressor(radius=3.0, weights=w).fit(X, t)
        b = skn.RadiusNeighborsRegressor(radius=3.0, weights=w, algorithm="brute").fit(X, t)
        np.testing.assert_allclose(a.predict(Q), b.predict(Q), rtol=1e-12, atol=1e-12)
    a = dan.NearestNeighbors(n_neighbors=4).fit(X)
    b = skn.NearestNeighbors(n_neighbors=4, algorithm="brute").fit(X)
    (da_d, da_i), (sk_d, sk_i) = a.kneighbors(Q), b.kneighbors(Q)
    np.testing.assert_array_equal(da_i, sk_i)
    np.testing.assert_allclose(da_d, sk_d, rtol=1e-12)


def test_kmeans_shims_match_oracle(gpu, da, orc):
    from aoclda.clustering import kmeans
    from aoclda.faiss import Kmeans
    from aoclda.sklearn._kmeans import KMeans
    z = golden("kmeans_lloyd80.npz")
    km = kmeans(n_clusters=16, C=z["C"], initialization_method="supplied", n_init=1,
                max_iter=30).fit(z["A"])
    np.testing.assert_array_equal(km.labels, z["expected_labels"])
    assert km.n_iter == int(z["expected_rinfo"][3])
    np.testing.assert_allclose(km.cluster_centres, z["expected_centres"], rtol=1e-4, atol=1e-5)
    sk = KMeans(n_clusters=16, init=z["C"], max_iter=30).fit(z["A"])
    np.testing.assert_array_equal(sk.labels_, z["expected_labels"])
    np.testing.assert_array_equal(sk.predict(z["A"]), z["expected_labels"])
    assert abs(sk.inertia_ - z["expected_rinfo"][4]) < 1e-4
    tr = sk.transform(z["A"][:5])
    d2 = ((z["A"][:5, None, :] - sk.cluster_centers_[None]) ** 2).sum(-1)
    np.testing.assert_allclose(tr, np.sqrt(d2), rtol=1e-10)
    fk = Kmeans(2, 16, niter=30, seed=3)
    obj = fk.train(z["A"])
    D, I = fk.assign(z["A"])
    assert I.dtype == np.int64 and obj > 0 and fk.centroids.shape == (16, 2)
    tr = fk._kmeans.transform(z["A"])
    np.testing.assert_allclose(D, (tr ** 2).min(axis=1), rtol=1e-12)


def test_faiss_indexes_and_ann(gpu, da, orc):
    from aoclda.faiss import IndexFlatL2, IndexIVFFlat
    from aoclda.neighbors import approximate_neighbors
    rng = np.random.default_rng(3)
    X, Q = data(rng, 5000, 100, 16, np.float32)
    flat = IndexFlatL2(16)
    flat.add(X[:2500])
    flat.add(X[2500:])
    assert flat.ntotal == 5000
    D, I = flat.search(Q, 5)
    oi, od = orc.knn(X, Q, 5, "sqeuclidean")
    assert I.dtype == np.int64
    np.testing.assert_array_equal(I, oi)
    np.testing.assert_array_equal(D, od)
    # every list probed: the exact neighbours (fp64 oracle within GEMM-form rounding)
    ivf = IndexIVFFlat(flat, 16, 8)
    ivf.train(X)
    ivf.add(X)
    ivf.nprobe = 8
    D2, I2 = ivf.search(Q, 5)
    assert ivf.ntotal == 5000 and I2.dtype == np.int64
    np.testing.assert_allclose(D2, od, rtol=1e-4, atol=1e-2)
    assert (I2 == oi).mean() > 0.99
    ann = approximate_neighbors(n_neighbors=5, n_list=8, n_probe=8, seed=1).train_and_add(X)
    assert ann.n_index == 5000 and ann.n_list == 8 and ann.list_sizes.sum() == 5000
    assert ann.cluster_centroids.shape == (8, 16)
    d3, i3 = ann.kneighbors(Q)
    assert (i3 == oi).mean() > 0.99


def test_pairwise_distances_shim(gpu, da, orc):
    from aoclda.metrics import pairwise_distances
    rng = np.random.default_rng(4)
    X, Y = data(rng, 300, 200, 11)
    for m in ("euclidean", "sqeuclidean", "manhattan", "cosine"):
        np.testing.assert_allclose(pairwise_distances(X, Y, metric=m), orc.pairwise(X, Y, m),
                                   rtol=1e-13, atol=1e-13)


def test_pickle_kmeans_and_ann(gpu, da):
    """Pickled k-means and IVF-flat objects answer as the originals."""
    import pickle

    from aoclda.clustering import kmeans
    from aoclda.neighbors import approximate_neighbors
    rng = np.random.default_rng(6)
    X, Q = data(rng, 4000, 50, 8)
    km = kmeans(n_clusters=5, n_init=1, seed=2).fit(X)
    km2 = pickle.loads(pickle.dumps(km))
    np.testing.assert_array_equal(km2.cluster_centres, km.cluster_centres)
    np.testing.assert_array_equal(km2.labels, km.labels)
    np.testing.assert_array_equal(km2.predict(Q), km.predict(Q))
    ann = approximate_neighbors(n_neighbors=4, n_list=6, n_probe=2, seed=1).train_and_add(X)
    ann2 = pickle.loads(pickle.dumps(ann))
    assert ann2.n_index == 4000
    for a, b in zip(ann2.kneighbors(Q), ann.kneighbors(Q)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("algorithm", ["lloyd", "elkan"])
def test_kmeans_spherical_shim(gpu, da, orc, dt, algorithm):
    """kmeans_test.py:313-337 of the reference (distance="cosine",
    normalize_data=False on its 6 x 3 array): unit-length centres; and
    the oracle's spherical Lloyd from the same initial centres."""
    from aoclda.clustering import kmeans
    a = golden("kmeans_spherical.npz")["py_a"].astype(dt)
    km = kmeans(n_clusters=2, algorithm=algorithm, distance="cosine", normalize_data=False,
                seed=42, n_init=1)
    km.fit(a)
    tol = 1e-6 if dt == np.float32 else 1e-12
    np.testing.assert_allclose(np.linalg.norm(km.cluster_centres.astype(np.float64), axis=1),
                               1.0, atol=tol)
    # supplied initial centres: the oracle's trajectory
    C0 = a[[0, 3]].copy()
    km = kmeans(n_clusters=2, C=C0, initialization_method="supplied", n_init=1,
                algorithm=algorithm, distance="cosine", normalize_data=True)
    km.fit(a)
    C, lab, _, _ = orc.kmeans_sph_lloyd(a, C0, 300, 1e-4, normalise=True)
    np.testing.assert_array_equal(km.labels, lab)
    np.testing.assert_allclose(km.cluster_centres, C, rtol=1e-5 if dt == np.float32 else 1e-12,
                               atol=1e-6 if dt == np.float32 else 1e-12)
