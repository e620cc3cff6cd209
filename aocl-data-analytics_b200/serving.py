"""Request loop over device-resident kNN indexes and k-means models.

The training set of the kNN index and the centres of the k-means models stay
in device memory for the life of the server: one library handle per worker,
the kNN handles holding one shared device copy of the index
(da_b200_nn_share_data).
Requests -- a kNN search (queries, k), an approximate (IVF-flat) search
(queries, k) when the server holds an IVF-flat index, or a k-means predict
(model, queries) -- are queued as they arrive; a kNN request with more queries than one call
takes is split into parts of at most that many (each part is searched on its
own; the request completes with its last part).  Each worker thread
repeatedly takes pending requests of its kind that fit its share of the
device-memory budget and its query cap -- requests waiting longer than
`aging_ms` first, then small ones (at most `small_queries` queries), then
the rest, oldest first within each class -- (continuous batching: requests
that arrive while a batch runs join the next one) and serves them with ONE
library call.  With `fast_lane` (two kNN workers or more) the first
`fast_lanes` kNN workers take only small requests (at most
`fast_lane_max_queries` per call), on high-priority streams, so that a
small request never waits behind a large batch; the others take large
requests first and small ones when nothing else is pending or when a small
one has waited `overflow_ms` (the fast lane is behind).  For kNN the
queries are concatenated and searched with the largest k asked for; every
request gets the prefix it asked for, which is exactly its own search because
results are ordered by (distance, index).  Several kNN workers run their
batches at the same time, each on its own handle, so their device work
overlaps.  Every request records when it was submitted and completed;
`latency_summary` gives p50 / p99.

The library calls release the Python interpreter lock (ctypes), so the worker
threads' device work proceeds concurrently.

Admission: a batch's device bytes (its queries, their candidate lists and
outputs) stay within the worker's share of `hbm_budget` and of the device
memory free when the batch is formed (less `hbm_reserve`); the oldest
request is always admitted, so no request waits for ever.  A library call
that fails completes every request of its batch with `error` set (the
workers keep serving).
"""
import collections
import gc
import threading
import time

import numpy as np

# device bytes per query of a kNN batch: the query row, its candidate list of
# the tensor-core pass (16,384 entries of 8 bytes) and its outputs (k <= 256)
KNN_LIST_BYTES = 16384 * 8
KNN_OUT_BYTES = 256 * 8


class Request:
    __slots__ = ("kind", "queries", "k", "model", "t_submit", "t_start", "t_done", "result",
                 "error", "_done", "parent", "offset", "parts_left")

    def __init__(self, kind, queries, k=None, model=None):
        if kind not in ("knn", "ann", "predict"):
            raise ValueError("kind must be 'knn', 'ann' or 'predict'")
        self.kind = kind
        self.queries = np.ascontiguousarray(queries, dtype=np.float32)
        self.k = k
        self.model = model
        self.t_submit = None
        self.t_start = None  # when a worker took it into a batch
        self.t_done = None
        self.result = None
        self.error = None       # the library's error when its call failed
        self._done = threading.Event()
        self.parent = None      # for a part: the request it belongs to
        self.offset = 0         # for a part: its first query in the parent
        self.parts_left = 0

    def wait(self, timeout=None):
        return self._done.wait(timeout)

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit


class Server:
    """kNN index X (n x d, fp32, euclidean) and k-means models given as
    {name: (training rows, initial centres)}, fitted at start-up.  `workers`
    kNN worker threads (one handle each) and one predict worker.  With
    `ann` = {"n_list": .., "n_probe": ..} an IVF-flat index of X (squared
    euclidean, trained and filled at start-up) serves "ann" requests on
    one more worker."""

    def __init__(self, ab, X, models=None, workers=2, max_batch_queries=1024,
                 max_request_queries=4096, hbm_budget=16 << 30, precision_mode="bf16x3",
                 small_queries=256, aging_ms=20.0, ann=None, free_memory="auto",
                 hbm_reserve=1 << 30, fast_lane=True, overflow_ms=2.0, fast_lanes=1,
                 fast_lane_max_queries=None):
        self.ab = ab
        # admission: a batch's device bytes stay within the worker's share of
        # hbm_budget AND of the device memory free (less hbm_reserve), read
        # every free_every seconds by a monitor thread (the reading is a
        # driver call that can wait behind other device work: no worker ever
        # makes it); free_memory() -> bytes, None to use the budget only
        if free_memory == "auto":
            dm = getattr(ab, "device_memory", None)
            free_memory = (lambda: dm()[0]) if dm is not None else None  # noqa: E731
        self.free_memory = free_memory
        self.hbm_reserve = hbm_reserve
        self.free_every = 0.05
        self._free_val = None
        self.small_queries = small_queries
        self.fast_lane = bool(fast_lane) and workers >= 2
        # the first fast_lanes kNN workers are fast lanes (at least one other
        # worker takes the large requests); a fast lane's batch holds at most
        # fast_lane_max_queries queries
        self.fast_lanes = max(1, min(int(fast_lanes), workers - 1)) if self.fast_lane else 0
        self.fast_cap = int(fast_lane_max_queries or max_batch_queries)
        self.overflow = overflow_ms / 1e3
        self.aging = aging_ms / 1e3
        self.X = np.ascontiguousarray(X, dtype=np.float32)
        self.d = self.X.shape[1]
        self.max_batch_queries = max_batch_queries
        self.hbm_budget = hbm_budget
        self.cv = threading.Condition()
        self.pending = {"knn": collections.deque(), "ann": collections.deque(),
                        "predict": collections.deque()}
        self.stopping = False
        self.completed = []
        # every library call: (kind, requests, queries, seconds, largest
        # request, worker thread id)
        self.batches = []
        self.fallback_queries = 0  # kNN queries the tensor-core pass handed to the plain path
        self.knn_handles = []
        for w in range(workers):
            h = ab.KNN("s", order=ab.ROW_MAJOR, metric="euclidean",
                       precision_mode=precision_mode)
            if w < self.fast_lanes:
                # the fast lane's kernels overtake the other workers' as SMs
                # free up
                h.set_stream_priority(-100)
            if w == 0:
                h.fit(self.X)
            else:
                # one device copy of the index (rows and tensor-core copies,
                # built by the first handle's warm-up below) for every worker
                h.share(self.knn_handles[0])
            # one call of the largest batch: the device copies and every
            # per-call buffer reach their final size now, so that no request
            # waits for a device allocation (which also stalls other work);
            # then calls of the other shapes a request can take (query tile
            # widths, k), so that every kernel they launch is loaded now
            warm = max(max_batch_queries, max_request_queries)
            h.kneighbors(self.X[np.arange(warm) % self.X.shape[0]], 256)
            for nq in (1, 64, 128, 256, min(warm, 512)):
                for kk in (1, 10, 100):
                    h.kneighbors(self.X[np.arange(nq) % self.X.shape[0]], kk)
            self.knn_handles.append(h)
        self.models = {}
        for name, (Xm, C0) in (models or {}).items():
            km = ab.KMeans(C0.shape[0], "s", order=ab.ROW_MAJOR, max_iter=50, n_init=1)
            km.fit(Xm, C0)
            # one predict of the largest request: its device buffers are
            # allocated now (an allocation later would stall every stream)
            km.predict(np.zeros((max_request_queries, Xm.shape[1]), dtype=np.float32))
            self.models[name] = km
        self.ann = None
        if ann is not None:
            # euclidean, as the kNN requests (distances, not their squares)
            self.ann = ab.ApproxNN("s", order=ab.ROW_MAJOR, n_list=int(ann["n_list"]),
                                   n_probe=int(ann.get("n_probe", 1)),
                                   seed=int(ann.get("seed", 0)), metric="euclidean")
            self.ann.set_training_data(self.X).train_and_add()
            # every kernel and buffer of the request shapes, now
            for nq in (1, min(max_request_queries, 512), max_batch_queries):
                self.ann.kneighbors(self.X[np.arange(nq) % self.X.shape[0]], 256)
        self.bytes_per_query = self.d * 4 + KNN_LIST_BYTES + KNN_OUT_BYTES
        # the start-up objects (index, models, handles) leave the collector's
        # view: a full collection then never walks them while requests wait
        gc.collect()
        gc.freeze()
        self.threads = [threading.Thread(target=self._knn_worker, args=(w,), daemon=True)
                        for w in range(workers)]
        if self.free_memory is not None:
            self.refresh_free_memory()
            self.threads.append(threading.Thread(target=self._monitor, daemon=True))
        self.threads.append(threading.Thread(target=self._predict_worker, daemon=True))
        if self.ann is not None:
            self.threads.append(threading.Thread(target=self._ann_worker, daemon=True))
        for t in self.threads:
            t.start()

    # ------------------------------------------------------------ clients --
    def submit(self, req):
        if req.kind == "predict" and req.model not in self.models:
            raise KeyError(f"unknown model {req.model!r}")
        if req.kind == "ann" and self.ann is None:
            raise KeyError("the server holds no IVF-flat index")
        if req.kind in ("knn", "ann") and not (1 <= req.k <= 256):
            raise ValueError("k must be in [1, 256]")
        req.t_submit = time.perf_counter()
        parts = [req]
        nq = req.queries.shape[0]
        if req.kind in ("knn", "ann") and nq > self.max_batch_queries:
            req.result = (np.empty((nq, req.k), dtype=np.int32),
                          np.empty((nq, req.k), dtype=np.float32))
            parts = []
            for o in range(0, nq, self.max_batch_queries):
                part = Request(req.kind, req.queries[o:o + self.max_batch_queries], k=req.k)
                part.t_submit, part.parent, part.offset = req.t_submit, req, o
                parts.append(part)
            req.parts_left = len(parts)
        with self.cv:
            self.pending[req.kind].extend(parts)
            self.cv.notify_all()
        return req

    def close(self):
        with self.cv:
            self.stopping = True
            self.cv.notify_all()
        for t in self.threads:
            t.join()
        for h in self.knn_handles:
            h.close()
        for km in self.models.values():
            km.close()
        if self.ann is not None:
            self.ann.close()

    # ------------------------------------------------------------ workers --
    def _take(self, kind, cap_queries, cap_bytes, per_query_bytes, same_model=False,
              small_only=False, large_first=False):
        """Oldest pending requests of `kind` within the caps (at least one);
        blocks until one is pending, None once the server stops.  small_only:
        requests of at most small_queries queries only.  large_first (the
        other workers beside a fast lane): large requests before small ones,
        unless a small one has waited overflow_ms (the fast lane is behind)."""
        def fits(r):
            return not small_only or r.queries.shape[0] <= self.small_queries

        with self.cv:
            while not any(map(fits, self.pending[kind])) and not self.stopping:
                self.cv.wait()
            q = self.pending[kind]
            if not any(map(fits, q)):
                return None
            now = time.perf_counter()
            # aged requests, then small ones, then the rest (oldest first in each)
            def rank(r):
                wait = now - r.t_submit
                small = r.queries.shape[0] <= self.small_queries
                if large_first:
                    return (not (wait >= self.aging or (small and wait >= self.overflow)),
                            small, r.t_submit)
                return (wait < self.aging, not small, r.t_submit)
            order = sorted(filter(fits, q), key=rank)
            model = order[0].model
            batch, nq = [], 0
            for r in order:
                m = r.queries.shape[0]
                if same_model and r.model != model:
                    continue
                if batch and (nq + m > cap_queries or (nq + m) * per_query_bytes > cap_bytes):
                    break
                r.t_start = now
                batch.append(r)
                nq += m
            taken = set(map(id, batch))
            self.pending[kind] = collections.deque(r for r in q if id(r) not in taken)
            return batch

    def refresh_free_memory(self):
        """Read the free device memory now (the monitor thread does this
        every free_every seconds)."""
        try:
            self._free_val = int(self.free_memory())
        except Exception:
            self._free_val = None

    def _monitor(self):
        while not self.stopping:
            time.sleep(max(self.free_every, 0.001))
            self.refresh_free_memory()

    def _cap_bytes(self, share):
        """The device bytes a batch may use now: the worker's share of the
        budget, and of the free device memory last read, less the reserve."""
        free = self._free_val
        if self.free_memory is None or free is None:
            return share
        free -= self.hbm_reserve
        return max(0, min(share, free // max(1, len(self.knn_handles))))

    def _fail(self, kind, batch, exc):
        """A library call failed: every request of the batch completes with
        the error (its parent request too), and the worker goes on."""
        for r in batch:
            (r.parent or r).error = f"{type(exc).__name__}: {exc}"
        self._finish(kind, batch, sum(r.queries.shape[0] for r in batch), 0.0)

    def _finish(self, kind, batch, nq, secs):
        t = time.perf_counter()
        done = []
        with self.cv:
            for r in batch:
                p = r.parent
                if p is None:
                    r.t_done = t
                    done.append(r)
                    continue
                p.t_start = r.t_start if p.t_start is None else min(p.t_start, r.t_start)
                p.parts_left -= 1
                if p.parts_left == 0:
                    p.t_done = t
                    done.append(p)
            self.completed.extend(done)
            self.batches.append((kind, len(batch), nq, secs,
                                 max(r.queries.shape[0] for r in batch), threading.get_ident()))
        for r in done:
            r._done.set()

    def _knn_worker(self, w):
        h = self.knn_handles[w]
        share = self.hbm_budget // len(self.knn_handles)
        while True:
            fast = w < self.fast_lanes
            batch = self._take("knn", self.fast_cap if fast else self.max_batch_queries,
                               self._cap_bytes(share), self.bytes_per_query, small_only=fast,
                               large_first=self.fast_lane and not fast)
            if batch is None:
                return
            try:
                Q = batch[0].queries if len(batch) == 1 else np.concatenate(
                    [r.queries for r in batch])
                kmax = max(r.k for r in batch)
                t0 = time.perf_counter()
                ind, dist = h.kneighbors(Q, kmax)
                secs = time.perf_counter() - t0
                nfb = int(h.stat("knn_tc_fallback_queries"))
            except Exception as exc:  # the request fails, the worker stays
                self._fail("knn", batch, exc)
                continue
            if nfb:
                with self.cv:
                    self.fallback_queries += nfb
            self._scatter("knn", batch, Q, ind, dist, secs)

    def _ann_worker(self):
        """IVF-flat requests: one search of the batch with the largest k; a
        request's own results are the prefix (the top-k over the probed lists
        in (distance, index) order does not depend on k)."""
        while True:
            batch = self._take("ann", self.max_batch_queries, self._cap_bytes(self.hbm_budget),
                               self.bytes_per_query)
            if batch is None:
                return
            try:
                Q = batch[0].queries if len(batch) == 1 else np.concatenate(
                    [r.queries for r in batch])
                kmax = max(r.k for r in batch)
                t0 = time.perf_counter()
                ind, dist = self.ann.kneighbors(Q, kmax)
                secs = time.perf_counter() - t0
            except Exception as exc:
                self._fail("ann", batch, exc)
                continue
            self._scatter("ann", batch, Q, ind, dist, secs)

    def _scatter(self, kind, batch, Q, ind, dist, secs):
        """Every request of a search batch gets its rows and k-prefix."""
        o = 0
        for r in batch:
            m = r.queries.shape[0]
            if r.parent is None:
                r.result = (ind[o:o + m, :r.k].copy(), dist[o:o + m, :r.k].copy())
            else:  # a part: its rows of the parent's result
                pi, pd = r.parent.result
                pi[r.offset:r.offset + m] = ind[o:o + m, :r.k]
                pd[r.offset:r.offset + m] = dist[o:o + m, :r.k]
            o += m
        self._finish(kind, batch, Q.shape[0], secs)

    def _predict_worker(self):
        while True:
            batch = self._take("predict", 1 << 30, 1 << 62, 1, same_model=True)
            if batch is None:
                return
            try:
                km = self.models[batch[0].model]
                Q = batch[0].queries if len(batch) == 1 else np.concatenate(
                    [r.queries for r in batch])
                t0 = time.perf_counter()
                lab = km.predict(Q)
                secs = time.perf_counter() - t0
            except Exception as exc:
                self._fail("predict", batch, exc)
                continue
            o = 0
            for r in batch:
                m = r.queries.shape[0]
                r.result = lab[o:o + m].copy()
                o += m
            self._finish("predict", batch, Q.shape[0], secs)


def latency_summary(reqs):
    """p50 / p99 / max of submit-to-completion latency, and its two parts:
    queueing (submit to the start of its batch) and service (batch start to
    completion)."""
    done = [r for r in reqs if r.latency is not None]
    if not done:
        return {"requests": 0}
    lat = np.array([r.latency for r in done])
    wait = np.array([r.t_start - r.t_submit for r in done])
    serve = np.array([r.t_done - r.t_start for r in done])
    ms = lambda a, q: float(np.percentile(a, q) * 1e3)  # noqa: E731
    return {"requests": int(lat.size), "p50_ms": ms(lat, 50), "p99_ms": ms(lat, 99),
            "max_ms": float(lat.max() * 1e3), "queue_p50_ms": ms(wait, 50),
            "queue_p99_ms": ms(wait, 99), "service_p50_ms": ms(serve, 50),
            "service_p99_ms": ms(serve, 99)}


def replay(server, trace, rng_queries):
    """Submit requests at the trace's arrival offsets (seconds from now):
    trace = [(t, kind, size, k_or_model)], queries drawn by rng_queries(size).
    Returns the submitted requests once all are complete."""
    reqs = []
    t0 = time.perf_counter()
    for t, kind, size, arg in trace:
        # sleep (not spin) until the arrival time, leaving the interpreter
        # lock to the workers
        wait = t - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        Q = rng_queries(size)
        r = Request(kind, Q, k=arg if kind in ("knn", "ann") else None,
                    model=arg if kind == "predict" else None)
        reqs.append(server.submit(r))
    for r in reqs:
        r.wait()
    return reqs
