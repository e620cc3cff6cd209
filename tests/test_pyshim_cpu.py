"""The ``aoclda`` drop-in Python package without a GPU: imports, the
scikit-learn patch and its undo, and the argument checks that come before
any library call (the reference's python_package/aoclda behaviour)."""
import numpy as np
import pytest


def test_imports_and_skpatch(da):
    import sklearn.cluster as skc
    import sklearn.metrics as skm
    import sklearn.neighbors as skn
    names = ["NearestNeighbors", "KNeighborsClassifier", "KNeighborsRegressor",
             "RadiusNeighborsClassifier", "RadiusNeighborsRegressor"]
    before = {n: getattr(skn, n) for n in names}
    km0, pd0 = skc.KMeans, skm.pairwise_distances
    done = da.sklearn.skpatch(print_patched=False)
    try:
        assert set(done) == set(names + ["KMeans", "pairwise_distances"])
        for n in names:
            assert getattr(skn, n).__module__ == "aoclda.sklearn._neighbors"
        assert skc.KMeans.__module__ == "aoclda.sklearn._kmeans"
        assert skm.pairwise_distances.__module__ == "aoclda.sklearn._metrics"
    finally:
        da.sklearn.undo_skpatch(print_patched=False)
    assert all(getattr(skn, n) is before[n] for n in names)
    assert skc.KMeans is km0 and skm.pairwise_distances is pd0
    # one symbol by name
    assert da.sklearn.skpatch("KMeans", print_patched=False) == ["KMeans"]
    da.sklearn.undo_skpatch("KMeans", print_patched=False)
    assert skc.KMeans is km0


def test_argument_checks(da):
    from aoclda.neighbors import nearest_neighbors
    from aoclda.sklearn._kmeans import KMeans
    from aoclda.sklearn._neighbors import KNeighborsClassifier, NearestNeighbors
    with pytest.raises(ValueError):
        nearest_neighbors(n_neighbors=2.5)
    with pytest.raises(ValueError):
        nearest_neighbors(radius=-1.0)
    with pytest.raises(RuntimeError):
        nearest_neighbors().kneighbors(np.zeros((2, 3)))      # before fit
    with pytest.raises(ValueError):
        KNeighborsClassifier(n_neighbors=0)
    with pytest.raises(ValueError):
        KNeighborsClassifier(metric="chebyshev")
    with pytest.raises(ValueError):
        NearestNeighbors(algorithm="lsh")
    with pytest.warns(RuntimeWarning):
        NearestNeighbors(n_jobs=4)
    with pytest.raises(ValueError):
        KMeans(init=lambda X, k, rs: X[:k])
    with pytest.raises(ValueError):
        KMeans(random_state=np.random.RandomState(0))
    p = KNeighborsClassifier(n_neighbors=3, weights="distance").get_params()
    assert p["n_neighbors"] == 3 and p["weights"] == "distance" and p["metric"] == "minkowski"


def test_faiss_shim_checks(da):
    from aoclda.faiss import IndexFlatL2, IndexIVFFlat
    q = IndexFlatL2(8)
    assert q.d == 8 and q.ntotal == 0 and q.is_trained
    with pytest.raises(RuntimeError):
        q.search(np.zeros((1, 8), dtype=np.float32), 1)
    with pytest.raises(ValueError):
        q.add(np.zeros((3, 7), dtype=np.float32))
    with pytest.raises(ValueError):
        IndexIVFFlat(q, 9, 4)
    with pytest.raises(ValueError):
        IndexIVFFlat(q, 8, 4, metric=7)
    ivf = IndexIVFFlat(q, 8, 4)
    assert not ivf.is_trained and ivf.ntotal == 0 and ivf.nprobe == 1
    ivf.nprobe = 3
    assert ivf.nprobe == 3
    with pytest.raises(RuntimeError):
        ivf.add(np.zeros((3, 8), dtype=np.float32))
    try:
        import faiss  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError):
            da.faiss.patch_faiss()


def test_nearest_neighbors_pickle(da):
    """Pickling keeps the parameters, the labels and the handle's model
    (training rows included): the unpickled object pickles to the same
    model bytes."""
    import pickle

    from aoclda.neighbors import nearest_neighbors
    rng = np.random.default_rng(5)
    X = rng.standard_normal((40, 4))
    y = rng.integers(0, 3, 40)
    nn = nearest_neighbors(n_neighbors=3, metric="manhattan", weights="distance").fit(X, y)
    nn2 = pickle.loads(pickle.dumps(nn))
    assert (nn2.n_neighbors, nn2.metric, nn2.weights) == (3, "manhattan", "distance")
    np.testing.assert_array_equal(nn2.y, y)
    assert nn2._h.get_int("number of neighbors") == 3
    assert nn2._h.get_string("metric") == "manhattan"
    assert nn.__getstate__()["_model"] == nn2.__getstate__()["_model"]
    # an unfitted object pickles too
    nn3 = pickle.loads(pickle.dumps(nearest_neighbors(n_neighbors=2)))
    assert nn3._h is None and nn3.n_neighbors == 2
