"""IVF-flat approximate neighbours (da_approx_nn_*) on the GPU.

The reference's functionality cases (ann_tests.hpp, squared euclidean and
their euclidean conversions) run through the C ABI with their own leading
dimensions, following the reference's test_functionality: empty lists after
train, no empty list after add, expected neighbours and distances (3000 eps),
train_and_add, return_distance = false, centroids and run information equal to
a k-means handle with the same options, list sizes, and a second add of the
same rows.  On seeded clustered data the search is checked against the oracle
restatement given the trained centroids: the lists, the probes and the k
nearest rows of the probed lists."""
import numpy as np
import pytest

from conftest import golden
from test_oracle_golden import ann_case

pytestmark = pytest.mark.gpu


def setup_handle(ab, prec, o, metric="sqeuclidean"):
    h = ab.ApproxNN(prec, order=ab.ROW_MAJOR if o["row"] else ab.COLUMN_MAJOR, metric=metric,
                    algorithm="ivfflat", number_of_neighbors=o["k"], n_list=o["n_list"],
                    n_probe=o["n_probe"], seed=o["seed"], kmeans_iter=o["kmeans_iter"],
                    train_fraction=o["train_fraction"])
    return h


def raw(z, i, key, dt):
    return np.ascontiguousarray(z[f"c{i}_{key}"], dtype=dt)


def search(ab, h, nq, d, Qraw, ldq, k, row, dt, with_dist=True):
    ind = np.zeros(nq * k, dtype=np.int32)
    dist = np.zeros(nq * k, dtype=dt)
    h.call(f"da_approx_nn_kneighbors_{h.prec}", nq, d, ab.ptr(Qraw), ldq, ab.ptr(ind),
           ab.ptr(dist) if with_dist else None, k, int(with_dist))
    shape = (nq, k) if row else (k, nq)
    ind, dist = ind.reshape(shape), dist.reshape(shape)
    return (ind, dist) if row else (ind.T, dist.T)


def sort_pairs(ind):
    a = ind.reshape(ind.shape[0], -1, 2)
    return np.sort(a, axis=2).reshape(ind.shape)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("metric", ["sqeuclidean", "euclidean"])
def test_ivf_functionality_cases(gpu, ab, prec, metric):
    z = golden("ann_functionality.npz")
    dt = np.float64 if prec == "d" else np.float32
    eps = 3000 * np.finfo(dt).eps
    for i, name in enumerate(z["names"]):
        o, X, Q, wi, wd = ann_case(z, i)
        if metric == "euclidean":
            wd = np.sqrt(wd)
        n, d = X.shape
        nq, k, nl = Q.shape[0], o["k"], o["n_list"]
        meta = z[f"c{i}_meta"]
        ldx, ldq = int(meta[6]), int(meta[7])
        Xr, Qr = raw(z, i, "X_train", dt), raw(z, i, "X_test", dt)
        h = setup_handle(ab, prec, o, metric)
        h.call(f"da_approx_nn_set_training_data_{prec}", n, d, ab.ptr(Xr), ldx)
        h.call(f"da_approx_nn_train_{prec}")
        assert not h.list_sizes(nl).any(), name
        h.call(f"da_approx_nn_add_{prec}", n, d, ab.ptr(Xr), ldx)
        if not name.startswith("Zero"):
            assert (h.list_sizes(nl) > 0).all(), name
        ind, dist = search(ab, h, nq, d, Qr, ldq, k, o["row"], dt)
        np.testing.assert_allclose(dist, wd, rtol=eps, atol=eps, err_msg=name)
        if wi is not None:
            np.testing.assert_array_equal(ind, wi, err_msg=name)
        else:
            assert ((ind >= 0) & (ind < n)).all()
            assert all(len(set(r)) == k for r in ind.tolist())
        # train_and_add, then without and with distances
        h.call(f"da_approx_nn_set_training_data_{prec}", n, d, ab.ptr(Xr), ldx)
        h.call(f"da_approx_nn_train_and_add_{prec}")
        ind2, _ = search(ab, h, nq, d, Qr, ldq, k, o["row"], dt, with_dist=False)
        np.testing.assert_array_equal(ind2, ind, err_msg=name)
        ind3, dist3 = search(ab, h, nq, d, Qr, ldq, k, o["row"], dt)
        np.testing.assert_array_equal(ind3, ind, err_msg=name)
        np.testing.assert_array_equal(dist3, dist, err_msg=name)
        # centroids and run information as a k-means handle with the same
        # options (not for a subsample, which the k-means API cannot take)
        if o["train_fraction"] == 1.0:
            km = ab.KMeans(nl, prec, order=ab.ROW_MAJOR if o["row"] else ab.COLUMN_MAJOR,
                           initialization_method="random", n_init=1, max_iter=o["kmeans_iter"],
                           seed=o["seed"])
            assert km.set("convergence tolerance", float(np.sqrt(np.finfo(dt).eps))) == 0
            Xd = np.ascontiguousarray(X, dtype=dt) if o["row"] else np.asfortranarray(X, dtype=dt)
            km.fit(Xd)
            want_c = km.centres(nl, d)
            got_c = h.result(ab.APPROX_NN_CENTROIDS, nl * d)
            got_c = got_c.reshape(nl, d) if o["row"] else got_c.reshape(d, nl).T
            np.testing.assert_allclose(got_c, want_c, rtol=2 * np.finfo(dt).eps,
                                       atol=2 * np.finfo(dt).eps, err_msg=name)
            rinfo = h.result(ab.RINFO, 4)
            assert rinfo.tolist() == [nl, n, d, km.rinfo()[3]], name
            km.close()
        assert h.list_sizes(nl).sum() == n
        # the same rows added again: every neighbour twice, indices + n
        h.call(f"da_approx_nn_add_{prec}", n, d, ab.ptr(Xr), ldx)
        ind4, dist4 = search(ab, h, nq, d, Qr, ldq, 2 * k, o["row"], dt)
        np.testing.assert_allclose(dist4, np.repeat(wd, 2, axis=1), rtol=eps, atol=eps,
                                   err_msg=name)
        if wi is not None:
            want = np.stack([wi, wi + n], axis=2).reshape(nq, 2 * k)
            np.testing.assert_array_equal(sort_pairs(ind4), sort_pairs(want), err_msg=name)
        assert h.list_sizes(nl).sum() == 2 * n
        assert h.result(ab.RINFO, 4)[1] == 2 * n
        h.close()


def blobs(rng, n, d, n_blobs, dt):
    centres = rng.uniform(-10, 10, (n_blobs, d))
    X = centres[rng.integers(0, n_blobs, n)] + rng.standard_normal((n, d))
    return X.astype(dt), centres


@pytest.mark.parametrize("prec,order", [("s", 0), ("d", 1), ("s", 1)])
@pytest.mark.parametrize("metric", ["sqeuclidean", "euclidean"])
@pytest.mark.parametrize("n_probe,k", [(3, 10), (1, 2000), (16, 50)])
def test_ivf_matches_oracle(gpu, ab, orc, prec, order, metric, n_probe, k):
    dt = np.float32 if prec == "s" else np.float64
    rng = np.random.default_rng(7 + n_probe + k)
    X, centres = blobs(rng, 20000, 24, 16, dt)
    Q = (centres[rng.integers(0, 16, 300)] + rng.standard_normal((300, 24))).astype(dt)
    h = ab.ApproxNN(prec, order=order, metric=metric, n_list=16, n_probe=n_probe, seed=3,
                    kmeans_iter=20)
    h.set_training_data(X).train_and_add()
    C = h.result(ab.APPROX_NN_CENTROIDS, 16 * 24)
    C = C.reshape(16, 24) if order == ab.ROW_MAJOR else C.reshape(24, 16).T
    lists = orc.ivf_lists(C.astype(np.float64), X)
    ind, dist = h.kneighbors(Q, k)
    rind, rdist, _ = orc.ivf_kneighbors(C.astype(np.float64), X, Q, k, n_probe, metric, lists)
    fin = np.isfinite(rdist)
    # GEMM-form distances: rounding relative to |q|^2 + |x|^2
    tol = 64 * np.finfo(dt).eps * 2.0 * (np.abs(X).max() ** 2) * 24
    if metric == "euclidean":
        tol = np.sqrt(tol)
    if dt == np.float64:
        # fp64: the same lists, probes and neighbours as the oracle
        np.testing.assert_array_equal(h.list_sizes(16), np.bincount(lists, minlength=16))
        assert (np.isfinite(dist) == fin).all() and ((ind == -1) == ~fin).all()
        np.testing.assert_allclose(dist[fin], rdist[fin], rtol=0, atol=tol)
        bad = ind != rind
        assert np.abs(dist[bad] - rdist[bad]).max(initial=0) <= tol
        assert bad.mean() < 0.001
    else:
        # fp32: a row within rounding of two centroids may join either list,
        # so: nearly the same lists, every returned distance the true one of
        # its row, ascending, and the oracle's neighbours found
        assert np.abs(h.list_sizes(16) - np.bincount(lists, minlength=16)).sum() <= 0.002 * len(X)
        ok = ind >= 0
        Xd, Qd = X.astype(np.float64), Q.astype(np.float64)
        true = ((Qd[:, None, :] - Xd[np.where(ok, ind, 0)]) ** 2).sum(-1)
        if metric == "euclidean":
            true = np.sqrt(true)
        np.testing.assert_allclose(dist[ok], true[ok], rtol=0, atol=tol)
        assert (np.diff(np.where(ok, dist.astype(np.float64), 1e300), axis=1) >= -tol).all()
        hits = sum(len(set(a[a >= 0]) & set(b[b >= 0])) for a, b in zip(ind, rind))
        assert hits >= 0.98 * (rind >= 0).sum()
    if k == 2000:
        assert (~fin).any()  # the probed list holds fewer than k rows
    h.close()


def test_ivf_option_locks_and_checks(gpu, ab):
    rng = np.random.default_rng(1)
    X, _ = blobs(rng, 500, 5, 4, np.float64)
    h = ab.ApproxNN("d", n_list=4, n_probe=2).set_training_data(X).train()
    # kneighbors before add
    with pytest.raises(ab.DAError) as e:
        h.kneighbors(X[:3], 2)
    assert e.value.status == 20
    h.add(X)
    assert h.set("n_list", 5) == 0
    with pytest.raises(ab.DAError) as e:
        h.kneighbors(X[:3], 2)
    assert e.value.status == 401
    assert h.set("n_list", 4) == 0
    assert h.set("n_probe", 5) == 0
    with pytest.raises(ab.DAError) as e:        # n_probe > n_list
        h.kneighbors(X[:3], 2)
    assert e.value.status == 4
    assert h.set("n_probe", 4) == 0
    with pytest.raises(ab.DAError) as e:        # k > rows in the index
        h.kneighbors(X[:3], 501)
    assert e.value.status == 4
    with pytest.raises(ab.DAError) as e:        # wrong n_features
        h.kneighbors(X[:3, :4], 2)
    assert e.value.status == 4
    # n_probe = n_list: the exact neighbours
    ind, dist = h.kneighbors(X[:50], 7)
    d2 = ((X[:50, None, :] - X[None]) ** 2).sum(-1)
    np.testing.assert_allclose(dist, np.sort(d2, axis=1)[:, :7], rtol=1e-9, atol=1e-9)
    # k = 0 takes the "number of neighbors" option (5)
    out = np.zeros(4 * 5, dtype=np.int32)
    dd = np.zeros(4 * 5)
    Xf = np.asfortranarray(X[:4])
    assert h.L.da_approx_nn_kneighbors_d(h.h, 4, 5, ab.ptr(Xf), 4, ab.ptr(out), ab.ptr(dd), 0,
                                         1) == 0
    np.testing.assert_array_equal(out.reshape(5, 4).T, ind[:4, :5])
    h.close()
