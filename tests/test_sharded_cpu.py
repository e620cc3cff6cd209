"""The exchange of the split k-means and kNN (aocl-data-analytics_b200/
sharded.py) on CPU with the host shards: two gloo processes (one holding
two shards), and several shards in one process, must give exactly what one
shard holding all rows gives -- k-means labels, centres and iteration count
bit for bit (the integer centroid sums make the reduction exact in any
order), the inertia to fp64 rounding (relative 1e-12), kNN neighbours,
distances and classifier votes bit for bit."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import sharded_worker as W  # noqa: E402


def unsplit(sd, X, y, C0, Q):
    fit = sd.kmeans_fit([sd.NumpyKMeansShard(X, C0.shape[0])], C0, max_iter=100, tol=1e-6)
    nn = [sd.NumpyKNNShard(X, 0, y)]
    ind, dist = sd.knn_kneighbors(nn, Q, 12)
    ind2, d2 = sd.knn_kneighbors(nn, Q, 12, metric="sqeuclidean")
    return {"centres": fit["centres"], "labels": fit["labels"][0], "n_iter": fit["n_iter"],
            "inertia": fit["inertia"], "converged": fit["converged"], "ind": ind, "dist": dist,
            "ind2": ind2, "d2": d2, "pu": sd.knn_predict(nn, Q, 12),
            "pd": sd.knn_predict(nn, Q, 12, weights="distance")}


def check(got, ref):
    for key in ("centres", "labels", "ind", "dist", "ind2", "d2", "pu", "pd"):
        np.testing.assert_array_equal(np.asarray(got[key]), np.asarray(ref[key]), err_msg=key)
    assert int(got["n_iter"]) == ref["n_iter"]
    assert int(got["converged"]) == ref["converged"]
    assert abs(float(got["inertia"]) - ref["inertia"]) <= 1e-12 * abs(ref["inertia"])


def test_in_process_shards_equal_unsplit():
    sd = W.load_sharded()
    X, y, C0, Q = W.data()
    ref = unsplit(sd, X, y, C0, Q)
    assert ref["n_iter"] > 2
    cuts = [0, 700, 701, 1900, X.shape[0]]
    km = [sd.NumpyKMeansShard(X[a:b], C0.shape[0]) for a, b in zip(cuts, cuts[1:])]
    fit = sd.kmeans_fit(km, C0, max_iter=100, tol=1e-6)
    nn = [sd.NumpyKNNShard(X[a:b], a, y[a:b]) for a, b in zip(cuts, cuts[1:])]
    ind, dist = sd.knn_kneighbors(nn, Q, 12)
    ind2, d2 = sd.knn_kneighbors(nn, Q, 12, metric="sqeuclidean")
    got = {"centres": fit["centres"], "labels": np.concatenate(fit["labels"]),
           "n_iter": fit["n_iter"], "inertia": fit["inertia"], "converged": fit["converged"],
           "ind": ind, "dist": dist, "ind2": ind2, "d2": d2,
           "pu": sd.knn_predict(nn, Q, 12), "pd": sd.knn_predict(nn, Q, 12, weights="distance")}
    check(got, ref)


def test_max_iter_and_k_checks():
    sd = W.load_sharded()
    X, y, C0, Q = W.data()
    one = sd.kmeans_fit([sd.NumpyKMeansShard(X, C0.shape[0])], C0, max_iter=2, tol=0.0)
    two = sd.kmeans_fit([sd.NumpyKMeansShard(X[:10], C0.shape[0]),
                         sd.NumpyKMeansShard(X[10:], C0.shape[0])], C0, max_iter=2, tol=0.0)
    assert one["n_iter"] == two["n_iter"] == 2 and one["converged"] == two["converged"] == 0
    np.testing.assert_array_equal(one["centres"], two["centres"])
    np.testing.assert_array_equal(one["labels"][0], np.concatenate(two["labels"]))
    with pytest.raises(ValueError):
        sd.knn_kneighbors([sd.NumpyKNNShard(X[:5], 0)], Q, 6)
    with pytest.raises(ValueError):
        sd.kmeans_fit([sd.NumpyKMeansShard(X, 3)], C0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_processes_equal_unsplit(tmp_path):
    sd = W.load_sharded()
    out = str(tmp_path / "sharded.npz")
    env = dict(os.environ, OMP_NUM_THREADS="1", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(HERE, "sharded_worker.py"), out]
    r = subprocess.run(cmd, env=env, timeout=300, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    got = dict(np.load(out))
    X, y, C0, Q = W.data()
    check(got, unsplit(sd, X, y, C0, Q))
