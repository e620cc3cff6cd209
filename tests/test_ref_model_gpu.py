"""Models saved by AOCL-DA (its da_handle_save_model format, written by
tests/refmodel.py) serve on the GPU after da_handle_load_model: a k-means
model predicts and transforms as the handle whose centres it holds, a kNN
model searches and predicts as a handle given the same training data, an
IVF-flat index returns the oracle's neighbours for its centroids and lists."""
import numpy as np
import pytest

import refmodel as rm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["s", "d"])
@pytest.mark.parametrize("distance", ["euclidean", "cosine"])
def test_kmeans_reference_model_serves(gpu, ab, tmp_path, prec, distance):
    dt = np.float32 if prec == "s" else np.float64
    rng = np.random.default_rng(2)
    A = (rng.standard_normal((20000, 16)) + rng.integers(0, 5, (20000, 1)) * 3).astype(dt)
    Y = A[:700] + dt(0.01)
    km = ab.KMeans(12, prec, order=ab.ROW_MAJOR, n_init=1, seed=4, distance=distance)
    km.fit(A)
    C = km.centres(12, 16)
    lab = km.labels(20000)
    r = km.rinfo()
    f = tmp_path / "km.model"
    rm.kmeans_file(f, prec, rm.ROW_MAJOR, C, lab, int(r[3]), r[4], distance=distance)
    km2 = ab.KMeans.load_model(f, prec)
    np.testing.assert_array_equal(km2.centres(12, 16), C)
    np.testing.assert_array_equal(km2.labels(20000), lab)
    np.testing.assert_array_equal(km2.predict(Y), km.predict(Y))
    np.testing.assert_array_equal(km2.transform(Y, 12), km.transform(Y, 12))
    km.close()
    km2.close()


@pytest.mark.parametrize("prec", ["s", "d"])
@pytest.mark.parametrize("order", [rm.COLUMN_MAJOR, rm.ROW_MAJOR])
def test_knn_reference_model_serves(gpu, ab, tmp_path, prec, order):
    dt = np.float32 if prec == "s" else np.float64
    rng = np.random.default_rng(5)
    X = rng.standard_normal((5000, 12)).astype(dt)
    y = rng.integers(0, 4, 5000)
    Q = rng.standard_normal((300, 12)).astype(dt)
    f = tmp_path / "nn.model"
    rm.nn_file(f, prec, order, X, y=y, n_neighbors=6, metric="euclidean", algorithm="ball tree",
               weights="distance", tree_bytes=b"\x00" * 256)
    nn = ab.KNN.load_model(f, prec)
    ref = ab.KNN(prec, order=order, number_of_neighbors=6, weights="distance").fit(X, y)
    ind, dist = nn.kneighbors(Q, 6)
    rind, rdist = ref.kneighbors(Q, 6)
    np.testing.assert_array_equal(ind, rind)
    np.testing.assert_array_equal(dist, rdist)
    np.testing.assert_array_equal(nn.predict(Q), ref.predict(Q))
    nn.close()
    ref.close()


@pytest.mark.parametrize("prec", ["s", "d"])
@pytest.mark.parametrize("metric", ["sqeuclidean", "euclidean", "inner product", "cosine"])
def test_ivf_reference_model_serves(gpu, ab, orc, tmp_path, prec, metric):
    dt = np.float32 if prec == "s" else np.float64
    rng = np.random.default_rng(8)
    X = (rng.standard_normal((6000, 10)) + rng.integers(0, 8, (6000, 1)) * 2).astype(dt)
    Q = X[rng.choice(6000, 200, replace=False)] + dt(0.05)
    nl = 8
    C = X[rng.choice(6000, nl, replace=False)].astype(np.float64)
    if metric in ("inner product", "cosine"):
        C /= np.linalg.norm(C, axis=1, keepdims=True)
    C = C.astype(dt)
    Xs = orc.normalise_rows(X) if metric == "cosine" else X
    lists = orc.ivf_lists(C.astype(np.float64), Xs, metric)
    rows = [Xs[lists == c] for c in range(nl)]
    ids = [np.nonzero(lists == c)[0] for c in range(nl)]
    norms = None
    if metric in ("sqeuclidean", "euclidean"):
        norms = []
        for r in rows:           # the reference's list norms: v * v summed feature by feature
            s = np.zeros(len(r), dtype=dt)
            for j in range(r.shape[1]):
                s = s + r[:, j] * r[:, j]
            norms.append(s)
    f = tmp_path / "ivf.model"
    rm.ivf_file(f, prec, rm.ROW_MAJOR, C, rows, ids, 6000, metric=metric, n_probe=3,
                list_norms=norms)
    h = ab.ApproxNN.load_model(f, prec)
    np.testing.assert_array_equal(h.list_sizes(nl), np.bincount(lists, minlength=nl))
    ind, dist = h.kneighbors(Q, 10)
    Qs = orc.normalise_rows(Q) if metric == "cosine" else Q
    rind, rdist, _ = orc.ivf_kneighbors(C.astype(np.float64), Xs, Qs, 10, 3, metric, lists)
    tol = 64 * np.finfo(dt).eps * (np.abs(Xs).max() ** 2) * 10
    if metric == "euclidean":
        tol = np.sqrt(tol)
    np.testing.assert_allclose(dist, rdist, rtol=0, atol=tol)
    assert (ind == rind).mean() > 0.995
    h.close()
