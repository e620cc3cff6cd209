"""The split k-means and kNN (aocl-data-analytics_b200/sharded.py) with
library shards on one GPU (several shards in one process; across processes
the only difference is the collective, which the gloo test covers): the
k-means labels, centres and iteration count must equal da_kmeans_compute_s
on the unsplit data (supplied initial centres, n_init = 1) bit for bit and
the inertia to fp64 rounding (relative 1e-12); kNN neighbours, distances
and classifier votes must equal one handle over the unsplit training set."""
import os

import numpy as np
import pytest

from conftest import PKG, _load

pytestmark = pytest.mark.gpu


def mixture(rng, n, d, comps, scale=8.0):
    means = rng.uniform(-scale, scale, (comps, d))
    sig = rng.uniform(0.5, 2.0, comps)
    lab = rng.integers(0, comps, n)
    X = means[lab] + rng.standard_normal((n, d)) * sig[lab, None]
    return X.astype(np.float32), lab


@pytest.mark.parametrize("n,d,k,mode,max_iter,tol,cuts", [
    (200_000, 48, 40, "bf16x3", 60, 1e-4, (0.31, 0.32, 0.8)),
    (150_000, 64, 256, "bf16x3", 8, 0.0, (0.5,)),
    (90_000, 33, 17, "plain", 100, 1e-6, (0.1, 0.55)),
])
def test_kmeans_shards_equal_single(gpu, ab, n, d, k, mode, max_iter, tol, cuts):
    sd = _load("aoclda_sharded", os.path.join(PKG, "sharded.py"))
    rng = np.random.default_rng(n + d + k)
    X, _ = mixture(rng, n, d, k)
    C0 = X[rng.choice(n, k, replace=False)].copy()
    km = ab.KMeans(k, "s", order=ab.ROW_MAJOR, max_iter=max_iter, n_init=1)
    km.set("convergence tolerance", tol)
    km.set("precision mode", mode)
    km.fit(X, C0)
    info = km.rinfo()
    ref_lab, ref_cen = km.labels(n), km.centres(k, d)
    km.close()

    edges = [0] + [int(c * n) for c in cuts] + [n]
    shards = [sd.DeviceKMeansShard(ab, X[a:b], k, precision_mode=mode)
              for a, b in zip(edges, edges[1:])]
    fit = sd.kmeans_fit(shards, C0, max_iter=max_iter, tol=tol)
    for sh in shards:
        sh.close()
    assert fit["n_iter"] == int(info[3])
    np.testing.assert_array_equal(fit["centres"], ref_cen)
    np.testing.assert_array_equal(np.concatenate(fit["labels"]), ref_lab)
    assert abs(fit["inertia"] - info[4]) <= 1e-12 * abs(info[4])


def test_knn_shards_equal_single(gpu, ab):
    sd = _load("aoclda_sharded", os.path.join(PKG, "sharded.py"))
    rng = np.random.default_rng(21)
    n, d, nq, k = 240_000, 64, 1_000, 50
    X, lab = mixture(rng, n, d, 64, scale=5.0)
    X[rng.integers(0, n, 2_000)] = X[rng.integers(0, n, 2_000)]   # exact ties
    y = (lab % 7).astype(np.int32)
    Q, _ = mixture(rng, nq, d, 64, scale=5.0)
    Q[:4] = X[[1, 70_000, 150_000, 239_999]]
    edges = [0, 70_000, 70_001, 150_000, n]
    shards = [sd.DeviceKNNShard(ab, X[a:b], a, y[a:b]) for a, b in zip(edges, edges[1:])]
    try:
        for metric in ("euclidean", "sqeuclidean"):
            one = ab.KNN("s", order=ab.ROW_MAJOR, metric=metric).fit(X)
            ri, rd = one.kneighbors(Q, k)
            one.close()
            si, sdist = sd.knn_kneighbors(shards, Q, k, metric=metric)
            np.testing.assert_array_equal(si, ri)
            np.testing.assert_array_equal(sdist, rd)
        for weights in ("uniform", "distance"):
            one = ab.KNN("s", order=ab.ROW_MAJOR, metric="euclidean", number_of_neighbors=k,
                         weights=weights).fit(X, y)
            rp = one.predict(Q)
            rpr = one.predict_proba(Q)
            one.close()
            _, spr = sd.knn_predict_proba(shards, Q, k, weights=weights)
            np.testing.assert_array_equal(spr, rpr)
            np.testing.assert_array_equal(sd.knn_predict(shards, Q, k, weights=weights), rp)
    finally:
        for sh in shards:
            sh.close()


def test_torch_comm_nccl_single_rank(gpu, ab):
    """The NCCL exchange (TorchComm over a one-rank process group) gives the
    single-handle results too."""
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    sd = _load("aoclda_sharded", os.path.join(PKG, "sharded.py"))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                            world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        comm = sd.TorchComm()
        rng = np.random.default_rng(3)
        n, d, k = 120_000, 40, 30
        X, lab = mixture(rng, n, d, k)
        C0 = X[rng.choice(n, k, replace=False)].copy()
        km = ab.KMeans(k, "s", order=ab.ROW_MAJOR, max_iter=40, n_init=1)
        km.fit(X, C0)
        info = km.rinfo()
        ref_lab, ref_cen = km.labels(n), km.centres(k, d)
        km.close()
        shards = [sd.DeviceKMeansShard(ab, X[:50_000], k), sd.DeviceKMeansShard(ab, X[50_000:], k)]
        fit = sd.kmeans_fit(shards, C0, comm, max_iter=40)
        for sh in shards:
            sh.close()
        assert fit["n_iter"] == int(info[3])
        np.testing.assert_array_equal(fit["centres"], ref_cen)
        np.testing.assert_array_equal(np.concatenate(fit["labels"]), ref_lab)
        assert abs(fit["inertia"] - info[4]) <= 1e-12 * abs(info[4])

        Q = X[rng.choice(n, 300, replace=False)] + np.float32(0.01)
        one = ab.KNN("s", order=ab.ROW_MAJOR, metric="euclidean").fit(X)
        ri, rd = one.kneighbors(Q, 20)
        one.close()
        kn = [sd.DeviceKNNShard(ab, X[:50_000], 0), sd.DeviceKNNShard(ab, X[50_000:], 50_000)]
        si, sdist = sd.knn_kneighbors(kn, Q, 20, comm)
        for sh in kn:
            sh.close()
        np.testing.assert_array_equal(si, ri)
        np.testing.assert_array_equal(sdist, rd)
    finally:
        dist.destroy_process_group()
