"""Model persistence on the GPU: a fitted k-means handle and a kNN handle
saved with da_handle_save_model and loaded with da_handle_load_model answer
exactly as the originals -- k-means centres, labels, run information and
predict; kNN neighbours, distances and class predictions; IVF-flat
centroids, list sizes, run information, searches and further adds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,order", [("s", 1), ("d", 0)])
def test_kmeans_model_round_trip(gpu, ab, tmp_path, prec, order):
    rng = np.random.default_rng(5)
    n, d, k = 20_000, 24, 12
    means = rng.uniform(-8, 8, (k, d))
    X = means[rng.integers(0, k, n)] + rng.standard_normal((n, d))
    km = ab.KMeans(k, prec, order=order, max_iter=40, n_init=1, seed=3)
    km.fit(X)
    f = tmp_path / "km.bin"
    km.save_model(f)
    km2 = ab.KMeans.load_model(f, prec)
    np.testing.assert_array_equal(km2.centres(k, d), km.centres(k, d))
    np.testing.assert_array_equal(km2.labels(n), km.labels(n))
    np.testing.assert_array_equal(km2.rinfo(), km.rinfo())
    Y = X[:777] + 0.25
    np.testing.assert_array_equal(km2.predict(Y), km.predict(Y))
    km.close()
    km2.close()


@pytest.mark.parametrize("prec,order,metric", [("s", 1, "euclidean"), ("d", 0, "manhattan")])
def test_knn_model_round_trip(gpu, ab, tmp_path, prec, order, metric):
    rng = np.random.default_rng(6)
    X = rng.standard_normal((5_000, 16))
    y = rng.integers(0, 5, 5_000).astype(np.int32)
    Q = rng.standard_normal((300, 16))
    nn = ab.KNN(prec, order=order, metric=metric, number_of_neighbors=9).fit(X, y)
    f = tmp_path / "nn.bin"
    nn.save_model(f)
    ref_ind, ref_dist = nn.kneighbors(Q, 9)
    ref_pred = nn.predict(Q)
    nn.close()          # the original is gone: the loaded handle owns its rows
    nn2 = ab.KNN.load_model(f, prec)
    ind, dist = nn2.kneighbors(Q, 9)
    np.testing.assert_array_equal(ind, ref_ind)
    np.testing.assert_array_equal(dist, ref_dist)
    np.testing.assert_array_equal(nn2.predict(Q), ref_pred)
    nn2.close()


@pytest.mark.parametrize("prec,order", [("s", 0), ("d", 1)])
def test_ivf_model_round_trip(gpu, ab, tmp_path, prec, order):
    rng = np.random.default_rng(8)
    means = rng.uniform(-8, 8, (12, 20))
    X = means[rng.integers(0, 12, 8000)] + rng.standard_normal((8000, 20))
    Q = X[:300] + 0.1
    h = ab.ApproxNN(prec, order=order, metric="euclidean", n_list=12, n_probe=3, seed=2)
    h.set_training_data(X).train_and_add()
    f = tmp_path / "ivf.bin"
    h.save_model(f)
    h2 = ab.ApproxNN.load_model(f, prec)
    assert h2.get_int("n_list") == 12 and h2.get_int("n_probe") == 3
    np.testing.assert_array_equal(h2.result(ab.APPROX_NN_CENTROIDS, 240),
                                  h.result(ab.APPROX_NN_CENTROIDS, 240))
    np.testing.assert_array_equal(h2.list_sizes(12), h.list_sizes(12))
    np.testing.assert_array_equal(h2.result(ab.RINFO, 4), h.result(ab.RINFO, 4))
    for a, b in zip(h2.kneighbors(Q, 9), h.kneighbors(Q, 9)):
        np.testing.assert_array_equal(a, b)
    h.add(X[:100])
    h2.add(X[:100])
    for a, b in zip(h2.kneighbors(Q, 9), h.kneighbors(Q, 9)):
        np.testing.assert_array_equal(a, b)
    h.close()
    h2.close()
