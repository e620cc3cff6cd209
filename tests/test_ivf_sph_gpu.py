"""IVF-flat with the inner-product and cosine metrics on the GPU.

The reference's functionality cases for these metrics (ann_tests.hpp,
converted into tests/golden/ann_functionality_spherical.npz) run through the
C ABI following its test_functionality: empty lists after train, expected
neighbours and distances (3000 eps), train_and_add, return_distance = false,
list sizes, a second add of the same rows; the coarse quantiser is spherical
k-means, so the centroids are unit length (UnitNormIPCentroids) and equal to
the oracle's (random rows, spherical Lloyd).  On seeded data the search is
checked against the oracle given the trained centroids."""
import numpy as np
import pytest

from conftest import golden
from test_ivf_gpu import raw, search, setup_handle, sort_pairs
from test_oracle_golden import ann_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["d", "s"])
def test_ivf_spherical_functionality_cases(gpu, ab, orc, prec):
    z = golden("ann_functionality_spherical.npz")
    dt = np.float64 if prec == "d" else np.float32
    eps = 3000 * np.finfo(dt).eps
    for i, name in enumerate(z["names"]):
        metric = str(z["metrics"][i])
        o, X, Q, wi, wd = ann_case(z, i)
        n, d = X.shape
        nq, k, nl = Q.shape[0], o["k"], o["n_list"]
        meta = z[f"c{i}_meta"]
        ldx, ldq = int(meta[6]), int(meta[7])
        Xr, Qr = raw(z, i, "X_train", dt), raw(z, i, "X_test", dt)
        h = setup_handle(ab, prec, o, metric)
        h.call(f"da_approx_nn_set_training_data_{prec}", n, d, ab.ptr(Xr), ldx)
        h.call(f"da_approx_nn_train_{prec}")
        assert not h.list_sizes(nl).any(), name
        # the centroids: unit length, the oracle's spherical k-means
        got_c = h.result(ab.APPROX_NN_CENTROIDS, nl * d)
        got_c = got_c.reshape(nl, d) if o["row"] else got_c.reshape(d, nl).T
        want_c = orc.ivf_train_spherical(X.astype(dt), nl, o["seed"], o["kmeans_iter"], metric)
        np.testing.assert_allclose(got_c, want_c, rtol=8 * np.finfo(dt).eps,
                                   atol=8 * np.finfo(dt).eps, err_msg=name)
        nz = np.abs(got_c).sum(1) > 0
        np.testing.assert_allclose((got_c[nz].astype(np.float64) ** 2).sum(1), 1.0,
                                   atol=1e-6 if prec == "s" else 1e-12, err_msg=name)
        h.call(f"da_approx_nn_add_{prec}", n, d, ab.ptr(Xr), ldx)
        ind, dist = search(ab, h, nq, d, Qr, ldq, k, o["row"], dt)
        np.testing.assert_allclose(dist, wd, rtol=eps, atol=eps, err_msg=name)
        if wi is not None:
            np.testing.assert_array_equal(ind, wi, err_msg=name)
        else:
            assert ((ind >= 0) & (ind < n)).all()
            assert all(len(set(r)) == k for r in ind.tolist())
        h.call(f"da_approx_nn_set_training_data_{prec}", n, d, ab.ptr(Xr), ldx)
        h.call(f"da_approx_nn_train_and_add_{prec}")
        ind2, _ = search(ab, h, nq, d, Qr, ldq, k, o["row"], dt, with_dist=False)
        np.testing.assert_array_equal(ind2, ind, err_msg=name)
        ind3, dist3 = search(ab, h, nq, d, Qr, ldq, k, o["row"], dt)
        np.testing.assert_array_equal(ind3, ind, err_msg=name)
        np.testing.assert_array_equal(dist3, dist, err_msg=name)
        assert h.list_sizes(nl).sum() == n
        h.call(f"da_approx_nn_add_{prec}", n, d, ab.ptr(Xr), ldx)
        ind4, dist4 = search(ab, h, nq, d, Qr, ldq, 2 * k, o["row"], dt)
        np.testing.assert_allclose(dist4, np.repeat(wd, 2, axis=1), rtol=eps, atol=eps,
                                   err_msg=name)
        if wi is not None:
            want = np.stack([wi, wi + n], axis=2).reshape(nq, 2 * k)
            np.testing.assert_array_equal(sort_pairs(ind4), sort_pairs(want), err_msg=name)
        assert h.list_sizes(nl).sum() == 2 * n
        h.close()


def _directions(rng, n, d, n_dirs, dt):
    dirs = rng.standard_normal((n_dirs, d))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    X = dirs[rng.integers(0, n_dirs, n)] * 3 + rng.standard_normal((n, d))
    return (X * rng.uniform(0.5, 4.0, n)[:, None]).astype(dt), dirs


@pytest.mark.parametrize("prec,order", [("s", 0), ("d", 1), ("s", 1)])
@pytest.mark.parametrize("metric", ["inner product", "cosine"])
@pytest.mark.parametrize("n_probe,k", [(3, 10), (1, 2000), (16, 50)])
def test_ivf_spherical_matches_oracle(gpu, ab, orc, prec, order, metric, n_probe, k):
    dt = np.float32 if prec == "s" else np.float64
    rng = np.random.default_rng(11 + n_probe + k)
    X, dirs = _directions(rng, 20000, 24, 16, dt)
    Q = (dirs[rng.integers(0, 16, 300)] * 3 + rng.standard_normal((300, 24))).astype(dt)
    h = ab.ApproxNN(prec, order=order, metric=metric, n_list=16, n_probe=n_probe, seed=3,
                    kmeans_iter=20)
    h.set_training_data(X).train_and_add()
    C = h.result(ab.APPROX_NN_CENTROIDS, 16 * 24)
    C = (C.reshape(16, 24) if order == ab.ROW_MAJOR else C.reshape(24, 16).T).astype(np.float64)
    np.testing.assert_allclose((C ** 2).sum(1), 1.0, atol=1e-5)
    Xs = orc.normalise_rows(X) if metric == "cosine" else X
    Qs = orc.normalise_rows(Q) if metric == "cosine" else Q
    lists = orc.ivf_lists(C, Xs, metric)
    ind, dist = h.kneighbors(Q, k)
    rind, rdist, _ = orc.ivf_kneighbors(C, Xs, Qs, k, n_probe, metric, lists)
    fin = np.isfinite(rdist)
    scale = np.abs(Xs).max() * np.abs(Qs).max() * 24
    tol = 64 * np.finfo(dt).eps * scale
    if dt == np.float64:
        np.testing.assert_array_equal(h.list_sizes(16), np.bincount(lists, minlength=16))
        assert (np.isfinite(dist) == fin).all() and ((ind == -1) == ~fin).all()
        np.testing.assert_allclose(dist[fin], rdist[fin], rtol=0, atol=tol)
        bad = ind != rind
        assert np.abs(dist[bad] - rdist[bad]).max(initial=0) <= tol
        assert bad.mean() < 0.001
    else:
        assert np.abs(h.list_sizes(16) - np.bincount(lists, minlength=16)).sum() <= 0.002 * len(X)
        ok = ind >= 0
        true = (Qs.astype(np.float64)[:, None, :] *
                Xs.astype(np.float64)[np.where(ok, ind, 0)]).sum(-1)
        if metric == "cosine":
            true = 1.0 - true
        np.testing.assert_allclose(dist[ok], true[ok], rtol=0, atol=tol)
        step = np.diff(dist.astype(np.float64), axis=1)
        both = ok[:, 1:] & ok[:, :-1]      # empty slots only at the end
        assert ((step >= -tol) if metric == "cosine" else (step <= tol))[both].all()
        assert (ok[:, 1:] <= ok[:, :-1]).all()
        hits = sum(len(set(a[a >= 0]) & set(b[b >= 0])) for a, b in zip(ind, rind))
        assert hits >= 0.98 * (rind >= 0).sum()
    if k == 2000:
        assert (~fin).any()
        # empty slots: index -1, distance -inf (inner product) / +inf (cosine)
        empty = ind == -1
        assert empty.any()
        assert (dist[empty] == (-np.inf if metric == "inner product" else np.inf)).all()
    h.close()


def test_ivf_spherical_persistence(gpu, ab, tmp_path):
    rng = np.random.default_rng(4)
    X, dirs = _directions(rng, 5000, 12, 8, np.float32)
    Q = X[:40] * 0.5
    for metric in ("inner product", "cosine"):
        h = ab.ApproxNN("s", metric=metric, n_list=8, n_probe=3, seed=1)
        h.set_training_data(X).train_and_add()
        ind, dist = h.kneighbors(Q, 5)
        f = tmp_path / f"ivf_{metric.replace(' ', '_')}.model"
        h.save_model(f)
        h2 = ab.ApproxNN.load_model(f, "s")
        ind2, dist2 = h2.kneighbors(Q, 5)
        np.testing.assert_array_equal(ind2, ind)
        np.testing.assert_array_equal(dist2, dist)
        h.close()
        h2.close()
