"""k-means and kNN over a data set split row-wise across processes, one GPU
(one library handle per shard) each.

k-means (the Lloyd loop of da_kmeans_compute_s, kmeans.cpp:996-1058 and the
convergence test of kmeans.cpp:1359-1397 in the reference): every process
assigns its rows and writes its fixed-point centroid sums, counts and
label-change flag into ONE int64 device buffer; one integer all-reduce over
the processes per iteration (exact, so the result does not depend on the
order of the reduction); then every process computes the same new centres
from the reduced buffer on its device.  With the whole data set's column
maxima and row count fixing the fixed-point scales, the labels, centres and
iteration count equal da_kmeans_compute_s on the unsplit data (supplied
initial centres, n_init = 1) bit for bit; the inertia is the sum of the
shards' inertias.

kNN (da_nn_kneighbors, nearest_neighbors.cpp in the reference): every
process searches its rows for the queries' k nearest, in squared distance
with global row indices; the candidates are all-gathered and merged by
(squared distance, index) -- ties to the lower index, as the single search
orders them -- and the square root is taken last for the euclidean metric,
so the neighbours and distances equal one search over the unsplit data.  The
classifier vote of da_nn_classifier_predict (nearest_neighbors.cpp:1166-1272
and 1566-1573) runs on the merged neighbours in the same fp32 order.

The exchange goes through `Comm` (one process: no exchange) or `TorchComm`
(torch.distributed: NCCL on device tensors, gloo on host tensors).  Several
shards may also live in one process (they are reduced locally first).
Shards: `DeviceKMeansShard` / `DeviceKNNShard` drive the library; the
`Numpy*` shards are host restatements with the same interface, used to test
the exchange logic without a GPU.
"""
import contextlib
import ctypes as C

import numpy as np

# -------------------------------------------------------------- exchange --


class Comm:
    """The exchange of a single process (nothing to exchange)."""
    rank = 0
    world = 1

    def allreduce_sum(self, t):
        return t

    def allreduce_max(self, t):
        return t

    def allgather(self, t):
        return [t]

    def allgather_object(self, obj):
        return [obj]


class TorchComm(Comm):
    """torch.distributed collectives of the default (or given) process
    group; tensors move to the group's device for the collective (CUDA for
    NCCL, host for gloo) and come back to their own device."""

    def __init__(self, group=None):
        import torch
        import torch.distributed as dist
        self.torch = torch
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        nccl = dist.get_backend(group) == "nccl"
        self.device = (torch.device("cuda", torch.cuda.current_device()) if nccl
                       else torch.device("cpu"))

    def _reduce(self, t, op):
        x = t if t.device == self.device else t.to(self.device)
        self.dist.all_reduce(x, op=op, group=self.group)
        return x if x.device == t.device else x.to(t.device)

    def allreduce_sum(self, t):
        return self._reduce(t, self.dist.ReduceOp.SUM)

    def allreduce_max(self, t):
        return self._reduce(t, self.dist.ReduceOp.MAX)

    def allgather(self, t):
        x = t if t.device == self.device else t.to(self.device)
        out = [self.torch.empty_like(x) for _ in range(self.world)]
        self.dist.all_gather(out, x.contiguous(), group=self.group)
        return [o if o.device == t.device else o.to(t.device) for o in out]

    def allgather_object(self, obj):
        out = [None] * self.world
        self.dist.all_gather_object(out, obj, group=self.group)
        return out


def _torch():
    import torch
    return torch


_STREAMS = {}


def shard_stream(device=None):
    """The CUDA stream the device shards of this process share on `device`
    (created once).  The library calls, the exchange buffers and the
    collectives all go on it, so they are ordered with one another."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    if dev.index not in _STREAMS:
        _STREAMS[dev.index] = torch.cuda.Stream(dev)
    return _STREAMS[dev.index]


# --------------------------------------------------------------- k-means --

def acc_len(k, d):
    """int64 entries of a shard's exchange buffer: k*d sums, k counts, the
    label-change flag."""
    return k * d + k + 1


def fixed_point_scales(colmax, n_global):
    """2^s_f and 2^-s_f per feature: s_f = min(62 - L, 44) - E_f with
    n_global <= 2^L and colmax[f] < 2^E_f, clamped to [-126, 127] (the
    library's scales for the whole data set)."""
    L = 0
    while (1 << L) < n_global:
        L += 1
    sf = np.empty(len(colmax), dtype=np.int64)
    for f, m in enumerate(np.asarray(colmax, dtype=np.float32)):
        E = int(np.frexp(np.float64(m))[1]) if m > 0 else 0
        sf[f] = max(-126, min(127, min(62 - L, 44) - E))
    return np.ldexp(np.float32(1.0), sf).astype(np.float32), np.ldexp(1.0, -sf)


class DeviceKMeansShard:
    """One shard of the rows in a library handle (fp32, row-major).  All its
    device work runs on `stream` (a torch.cuda.Stream; by default
    shard_stream()), which every shard of the process must share: the
    exchange buffers and the collectives go on it too (`context()`)."""

    def __init__(self, ab, X, n_clusters, precision_mode="bf16x3", stream=None):
        torch = _torch()
        self.ab = ab
        self.X = np.ascontiguousarray(X, dtype=np.float32)
        self.n, self.d = self.X.shape
        self.k = int(n_clusters)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = shard_stream(self.device.index) if stream is None else stream
        self.km = ab.KMeans(self.k, "s", order=ab.ROW_MAJOR, n_init=1, max_iter=1)
        self.km.set("precision mode", precision_mode)
        self.km.set_data(self.X)
        self.km.L.da_b200_set_stream(self.km.h, C.c_void_p(self.stream.cuda_stream))

    def context(self):
        return _torch().cuda.stream(self.stream)

    def new_acc(self):
        torch = _torch()
        return torch.zeros(acc_len(self.k, self.d), dtype=torch.int64, device=self.device)

    def colmax(self):
        out = np.zeros(self.d, dtype=np.float32)
        self.km.call("da_b200_kmeans_shard_colmax_s", self.ab.ptr(out))
        return out

    def begin(self, colmax, n_global, C0):
        cm = np.ascontiguousarray(colmax, dtype=np.float32)
        c0 = np.ascontiguousarray(C0, dtype=np.float32)
        self.km.call("da_b200_kmeans_shard_begin_s", self.ab.ptr(cm), int(n_global),
                     self.ab.ptr(c0))

    def partial(self, acc):
        self.km.call("da_b200_kmeans_shard_partial_s", C.c_void_p(acc.data_ptr()))

    def finalize(self, acc):
        scal = np.zeros(2, dtype=np.float64)
        flags = np.zeros(2, dtype=np.int32)
        self.km.call("da_b200_kmeans_shard_finalize_s", C.c_void_p(acc.data_ptr()),
                     self.ab.ptr(scal), self.ab.ptr(flags))
        return scal, flags

    def inertia(self, relabel):
        v = C.c_double()
        self.km.call("da_b200_kmeans_shard_inertia_s", int(bool(relabel)), C.byref(v))
        return v.value

    def result(self):
        cen = np.zeros((self.k, self.d), dtype=np.float32)
        lab = np.zeros(self.n, dtype=np.int32)
        self.km.call("da_b200_kmeans_shard_result_s", self.ab.ptr(cen), self.ab.ptr(lab))
        return cen, lab

    def close(self):
        self.km.close()


class NumpyKMeansShard:
    """Host restatement of the shard steps (labels by fp64 distances, the
    fixed-point sums by round-to-nearest-even of x 2^s_f), for testing the
    exchange on CPU: the unsplit and split data give identical results with
    it too."""

    def __init__(self, X, n_clusters):
        self.X = np.ascontiguousarray(X, dtype=np.float32)
        self.n, self.d = self.X.shape
        self.k = int(n_clusters)

    def new_acc(self):
        torch = _torch()
        return torch.zeros(acc_len(self.k, self.d), dtype=torch.int64)

    def context(self):
        return contextlib.nullcontext()

    def colmax(self):
        if self.n == 0:
            return np.zeros(self.d, dtype=np.float32)
        return np.abs(self.X).max(axis=0).astype(np.float32)

    def begin(self, colmax, n_global, C0):
        self.scale, self.inv = fixed_point_scales(colmax, n_global)
        self.C = np.array(C0, dtype=np.float32)
        self.lab = np.zeros(self.n, dtype=np.int32)
        self.q = np.rint(self.X.astype(np.float64) * self.scale.astype(np.float64)).astype(np.int64)

    def _assign(self):
        X = self.X.astype(np.float64)
        Cd = self.C.astype(np.float64)
        dist = (X * X).sum(1)[:, None] + (Cd * Cd).sum(1)[None, :] - 2.0 * X @ Cd.T
        return np.argmin(dist, axis=1).astype(np.int32)

    def partial(self, acc):
        lab = self._assign()
        changed = bool((lab != self.lab).any())
        self.lab = lab
        k, d = self.k, self.d
        sums = np.zeros((k, d), dtype=np.int64)
        np.add.at(sums, lab, self.q)
        cnt = np.bincount(lab, minlength=k).astype(np.int64)
        a = acc.numpy()
        a[:k * d] = sums.ravel()
        a[k * d:k * d + k] = cnt
        a[k * d + k] = int(changed)

    def finalize(self, acc):
        k, d = self.k, self.d
        a = acc.numpy()
        S = a[:k * d].reshape(k, d).astype(np.float64)
        cnt = a[k * d:k * d + k]
        new = ((S * self.inv[None, :]) / np.maximum(cnt, 1)[:, None].astype(np.float64))
        new = new.astype(np.float32)
        old = self.C.astype(np.float64)
        scal = np.array([(old * old).sum(), ((old - new.astype(np.float64)) ** 2).sum()])
        self.C = new
        flags = np.array([int(a[k * d + k] != 0), int((cnt == 0).sum())], dtype=np.int32)
        return scal, flags

    def inertia(self, relabel):
        if relabel:
            self.lab = self._assign()
        diff = self.X.astype(np.float64) - self.C.astype(np.float64)[self.lab]
        return float((diff * diff).sum())

    def result(self):
        return self.C.copy(), self.lab.copy()

    def close(self):
        pass


def kmeans_fit(shards, C0, comm=None, max_iter=300, tol=1e-4, empty_clusters="ignore"):
    """Lloyd k-means over this process's shards and the other processes' (all
    processes call it with their own shards and the same C0 and options).
    Returns {"centres", "labels" (one array per local shard), "n_iter",
    "inertia", "converged" (0: max_iter reached, 1: centre shift below tol,
    2: no label changed)}."""
    if empty_clusters not in ("ignore", "error"):
        raise ValueError("empty_clusters must be 'ignore' or 'error' for split data")
    torch = _torch()
    comm = comm or Comm()
    C0 = np.ascontiguousarray(C0, dtype=np.float32)
    k, d = C0.shape
    if not shards:
        raise ValueError("every process needs at least one shard")
    for sh in shards:
        if sh.k != k or sh.d != d:
            raise ValueError("shard shapes disagree with the initial centres")
    with shards[0].context():
        return _lloyd(shards, C0, comm, max_iter, tol, empty_clusters)


def _lloyd(shards, C0, comm, max_iter, tol, empty_clusters):
    torch = _torch()
    # the whole data set's column maxima and row count
    cm = np.max(np.stack([sh.colmax() for sh in shards]), axis=0)
    cm = comm.allreduce_max(torch.from_numpy(cm.copy())).numpy()
    n_global = int(comm.allreduce_sum(torch.tensor([sum(sh.n for sh in shards)],
                                                   dtype=torch.int64)).item())
    for sh in shards:
        sh.begin(cm, n_global, C0)
    accs = [sh.new_acc() for sh in shards]
    total = accs[0] if len(shards) == 1 else torch.zeros_like(accs[0])
    converged = 0
    it = 0
    while it < max_iter:
        for sh, a in zip(shards, accs):
            sh.partial(a)
        if len(shards) > 1:
            torch.sum(torch.stack(accs), dim=0, out=total)
        g = comm.allreduce_sum(total)
        res = [sh.finalize(g) for sh in shards]
        scal, flags = res[0]
        if int(flags[1]) > 0 and empty_clusters == "error":
            raise RuntimeError(f"{int(flags[1])} empty clusters in Lloyd iteration {it}")
        conv = 0
        if it > 1 and int(flags[0]) == 0:
            conv = 2
        if conv == 0 and np.sqrt(scal[1]) < tol * np.sqrt(scal[0]):
            conv = 1
        converged = conv
        if converged > 0:
            break
        it += 1
    relabel = converged == 1 or it == max_iter
    local = sum(sh.inertia(relabel) for sh in shards)
    inertia = float(comm.allreduce_sum(torch.tensor([local], dtype=torch.float64)).item())
    out = [sh.result() for sh in shards]
    return {"centres": out[0][0], "labels": [o[1] for o in out], "n_iter": it,
            "inertia": inertia, "converged": converged}


# ------------------------------------------------------------------- kNN --

_FAR = np.iinfo(np.int64).max


class DeviceKNNShard:
    """Rows [offset, offset + n) of the training set in a library kNN handle
    (fp32, row-major, squared euclidean)."""

    def __init__(self, ab, X, offset, y=None, precision_mode="bf16x3"):
        self.ab = ab
        self.X = np.ascontiguousarray(X, dtype=np.float32)
        self.n, self.d = self.X.shape
        self.offset = int(offset)
        self.y = None if y is None else np.ascontiguousarray(y, dtype=np.int32)
        self.nn = ab.KNN("s", order=ab.ROW_MAJOR, metric="sqeuclidean",
                         precision_mode=precision_mode).fit(self.X)

    def search(self, Q, k):
        ind, d2 = self.nn.kneighbors(np.ascontiguousarray(Q, dtype=np.float32), k)
        return ind.astype(np.int64), d2

    def close(self):
        self.nn.close()


class NumpyKNNShard:
    """Host restatement of a shard's search (fp64 squared distances rounded
    to fp32, ties to the lower index), for testing the exchange on CPU."""

    def __init__(self, X, offset, y=None):
        self.X = np.ascontiguousarray(X, dtype=np.float32)
        self.n, self.d = self.X.shape
        self.offset = int(offset)
        self.y = None if y is None else np.ascontiguousarray(y, dtype=np.int32)

    def search(self, Q, k):
        Qd = np.asarray(Q, dtype=np.float64)
        Xd = self.X.astype(np.float64)
        d2 = ((Qd[:, None, :] - Xd[None, :, :]) ** 2).sum(-1).astype(np.float32)
        idx = np.broadcast_to(np.arange(self.n, dtype=np.int64), d2.shape)
        o = np.lexsort((idx, d2), axis=-1)[:, :k]
        return o.astype(np.int64), np.take_along_axis(d2, o, axis=1)

    def close(self):
        pass


def _merge(ind, d2, lab, k):
    """The k smallest (squared distance, global index) of every row."""
    o = np.lexsort((ind, d2), axis=-1)[:, :k]
    take = lambda a: None if a is None else np.take_along_axis(a, o, axis=1)  # noqa: E731
    return take(ind), take(d2), take(lab)


def knn_kneighbors(shards, Q, k, comm=None, metric="euclidean", with_labels=False):
    """The k nearest training rows (global indices, distances) of every query
    over all processes' shards; k <= the whole training set's rows.  metric:
    "euclidean" or "sqeuclidean".  With with_labels the neighbours' class
    labels come too (every shard needs y)."""
    if metric not in ("euclidean", "sqeuclidean"):
        raise ValueError("split kNN supports the euclidean and sqeuclidean metrics")
    torch = _torch()
    comm = comm or Comm()
    Q = np.ascontiguousarray(Q, dtype=np.float32)
    nq = Q.shape[0]
    parts_i, parts_d, parts_l = [], [], []
    for sh in shards:
        kk = min(k, sh.n)
        if kk == 0:
            continue
        ind, d2 = sh.search(Q, kk)
        parts_i.append(ind + sh.offset)
        parts_d.append(d2)
        if with_labels:
            parts_l.append(sh.y[ind])
    n_here = sum(sh.n for sh in shards)
    n_all = int(comm.allreduce_sum(torch.tensor([n_here], dtype=torch.int64)).item())
    if k > n_all:
        raise ValueError("k is larger than the training set")
    # pad to k per process so that the all-gather has one shape
    pad = max(0, k - sum(p.shape[1] for p in parts_i))
    parts_i.append(np.full((nq, pad), _FAR, dtype=np.int64))
    parts_d.append(np.full((nq, pad), np.inf, dtype=np.float32))
    parts_l.append(np.full((nq, pad), -1, dtype=np.int32))
    ind, d2, lab = _merge(np.concatenate(parts_i, 1), np.concatenate(parts_d, 1),
                          np.concatenate(parts_l, 1) if with_labels else None, k)
    if comm.world > 1:
        gi = comm.allgather(torch.from_numpy(np.ascontiguousarray(ind)))
        gd = comm.allgather(torch.from_numpy(np.ascontiguousarray(d2)))
        ind = np.concatenate([t.numpy() for t in gi], 1)
        d2 = np.concatenate([t.numpy() for t in gd], 1)
        if with_labels:
            gl = comm.allgather(torch.from_numpy(np.ascontiguousarray(lab)))
            lab = np.concatenate([t.numpy() for t in gl], 1)
        ind, d2, lab = _merge(ind, d2, lab, k)
    dist = np.sqrt(d2) if metric == "euclidean" else d2
    ind = ind.astype(np.int32)
    return (ind, dist.astype(np.float32), lab) if with_labels else (ind, dist.astype(np.float32))


def knn_classes(shards, comm=None):
    """Sorted class labels over all processes' shards."""
    comm = comm or Comm()
    mine = sorted(set(int(v) for sh in shards for v in np.unique(sh.y)))
    return np.array(sorted(set(v for part in comm.allgather_object(mine) for v in part)),
                    dtype=np.int32)


def knn_predict_proba(shards, Q, k, comm=None, metric="euclidean", weights="uniform"):
    """Class probabilities of the neighbour vote (fp32, the library's order of
    additions); returns (classes, proba[nq, n_classes])."""
    if weights not in ("uniform", "distance"):
        raise ValueError("weights must be 'uniform' or 'distance'")
    classes = knn_classes(shards, comm)
    ind, dist, lab = knn_kneighbors(shards, Q, k, comm, metric, with_labels=True)
    nq = ind.shape[0]
    eps = np.finfo(np.float32).eps
    if weights == "uniform":
        w = np.ones_like(dist)
    else:
        with np.errstate(divide="ignore"):
            w = np.where(dist <= eps, np.float32(1.0), np.float32(1.0) / dist).astype(np.float32)
    v = np.zeros((nq, classes.size), dtype=np.float32)
    for c, cls in enumerate(classes):
        acc = np.zeros(nq, dtype=np.float32)
        for r in range(k):
            acc = np.where(lab[:, r] == cls, acc + w[:, r], acc).astype(np.float32)
        v[:, c] = acc
    den = np.zeros(nq, dtype=np.float32)
    for c in range(classes.size):
        den = (den + v[:, c]).astype(np.float32)
    return classes, (v / den[:, None]).astype(np.float32)


def knn_predict(shards, Q, k, comm=None, metric="euclidean", weights="uniform"):
    """Predicted classes: the first class of largest probability."""
    classes, pr = knn_predict_proba(shards, Q, k, comm, metric, weights)
    return classes[np.argmax(np.abs(pr), axis=1)]
