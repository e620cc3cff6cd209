"""One rank of the two-process (gloo) run of the split k-means and kNN with
the host shards: rank 0 holds the first 40% of the rows, rank 1 the rest as
two shards.  Launched by test_sharded_cpu.py under torch.distributed.run;
rank 0 writes the results to the .npz named on the command line."""
import importlib.util
import os
import sys
from datetime import timedelta

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "aocl-data-analytics_b200")


def load_sharded():
    spec = importlib.util.spec_from_file_location("aoclda_sharded", os.path.join(PKG, "sharded.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["aoclda_sharded"] = mod
    spec.loader.exec_module(mod)
    return mod


def data(seed=5, n=3001, d=7, comps=9, nq=57):
    rng = np.random.default_rng(seed)
    means = rng.uniform(-6.0, 6.0, (comps, d))
    lab = rng.integers(0, comps, n)
    X = (means[lab] + rng.standard_normal((n, d))).astype(np.float32)
    X[100:140] = X[:40]                      # exact duplicates across the split -> ties
    y = (lab % 4).astype(np.int32)
    C0 = X[rng.choice(n, comps, replace=False)].copy()
    Q = (means[rng.integers(0, comps, nq)] + rng.standard_normal((nq, d))).astype(np.float32)
    Q[:3] = X[[0, 105, 2000]]
    return X, y, C0, Q


def splits(n):
    a = int(n * 0.4)
    b = a + (n - a) // 3
    return [(0, a)], [(a, b), (b, n)]


def main(out):
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    sd = load_sharded()
    comm = sd.TorchComm()
    X, y, C0, Q = data()
    mine = splits(X.shape[0])[comm.rank]
    km = [sd.NumpyKMeansShard(X[a:b], C0.shape[0]) for a, b in mine]
    fit = sd.kmeans_fit(km, C0, comm, max_iter=100, tol=1e-6)
    nn = [sd.NumpyKNNShard(X[a:b], a, y[a:b]) for a, b in mine]
    ind, dist_ = sd.knn_kneighbors(nn, Q, 12, comm)
    ind2, d2 = sd.knn_kneighbors(nn, Q, 12, comm, metric="sqeuclidean")
    pu = sd.knn_predict(nn, Q, 12, comm)
    pd = sd.knn_predict(nn, Q, 12, comm, weights="distance")
    labels = comm.allgather_object(np.concatenate(fit["labels"]))
    if comm.rank == 0:
        np.savez(out, centres=fit["centres"], labels=np.concatenate(labels),
                 n_iter=fit["n_iter"], inertia=fit["inertia"], converged=fit["converged"],
                 ind=ind, dist=dist_, ind2=ind2, d2=d2, pu=pu, pd=pd)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
