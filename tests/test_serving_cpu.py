"""The serving loop's host logic (aocl-data-analytics_b200/serving.py) on
CPU, over a stand-in for the library binding that answers with numpy:
requests larger than one call are split into parts and reassembled, kNN
requests batched together each get their own k-prefix, predict requests are
batched per model, and the latency summary splits queueing and service."""
import os
import threading
import time

import numpy as np

from conftest import PKG, _load


class FakeKNN:
    def __init__(self, prec, order=None, **options):
        self.calls = []

    def fit(self, X):
        self.X = np.asarray(X, dtype=np.float64)
        return self

    def share(self, source):
        self.X = source.X
        return self

    def set_stream_priority(self, priority):
        return self

    def kneighbors(self, Q, k):
        self.calls.append(Q.shape[0])
        d2 = ((np.asarray(Q, dtype=np.float64)[:, None, :] - self.X[None]) ** 2).sum(-1)
        idx = np.broadcast_to(np.arange(self.X.shape[0]), d2.shape)
        o = np.lexsort((idx, d2), axis=-1)[:, :k]
        return o.astype(np.int32), np.sqrt(np.take_along_axis(d2, o, 1)).astype(np.float32)

    def stat(self, name):
        return 0.0

    def close(self):
        pass


class FakeKMeans:
    def __init__(self, k, prec, order=None, **options):
        self.k = k

    def fit(self, X, C0):
        self.C = np.asarray(C0, dtype=np.float64)
        return self

    def predict(self, Q):
        d2 = ((np.asarray(Q, dtype=np.float64)[:, None, :] - self.C[None]) ** 2).sum(-1)
        return np.argmin(d2, axis=1).astype(np.int32)

    def close(self):
        pass


class FakeAB:
    ROW_MAJOR = 1
    KNN = FakeKNN
    KMeans = FakeKMeans


def test_serving_split_batch_and_prefixes():
    sv = _load("aoclda_serving_cpu", os.path.join(PKG, "serving.py"))
    rng = np.random.default_rng(3)
    X = rng.standard_normal((400, 5)).astype(np.float32)
    Xm = rng.standard_normal((100, 5)).astype(np.float32)
    models = {"m": (Xm, Xm[:7].copy())}
    server = sv.Server(FakeAB(), X, models=models, workers=2, max_batch_queries=16,
                       max_request_queries=64)
    try:
        reqs = []
        for i, (size, k) in enumerate([(3, 1), (40, 10), (1, 100), (16, 7), (33, 256), (5, 2)]):
            reqs.append(server.submit(sv.Request("knn", rng.standard_normal((size, 5)), k=k)))
            if i % 2:
                reqs.append(server.submit(sv.Request("predict", rng.standard_normal((size, 5)),
                                                     model="m")))
        for r in reqs:
            assert r.wait(30)
        ref_knn = FakeKNN("s").fit(X)
        ref_km = FakeKMeans(7, "s").fit(Xm, Xm[:7])
        for r in reqs:
            assert r.t_submit <= r.t_start <= r.t_done
            if r.kind == "knn":
                ind, dist = ref_knn.kneighbors(r.queries, r.k)
                np.testing.assert_array_equal(r.result[0], ind)
                np.testing.assert_array_equal(r.result[1], dist)
            else:
                np.testing.assert_array_equal(r.result, ref_km.predict(r.queries))
        # every kNN call stays within the cap; the 40- and 33-query
        # requests were served in parts
        assert max(b[2] for b in server.batches if b[0] == "knn") <= 16
        assert sum(1 for b in server.batches if b[0] == "knn") >= 6
        s = sv.latency_summary(reqs)
        assert s["requests"] == len(reqs)
        for key in ("p50_ms", "p99_ms", "queue_p99_ms", "service_p99_ms"):
            assert s[key] >= 0.0
    finally:
        server.close()


def test_serving_small_requests_first():
    """With one worker held busy, a small request submitted after a large one
    is taken first."""
    sv = _load("aoclda_serving_cpu2", os.path.join(PKG, "serving.py"))
    gate = threading.Event()

    class SlowKNN(FakeKNN):
        def kneighbors(self, Q, k):
            if Q.shape[0] == 2:  # the blocking request
                gate.wait(10)
            return super().kneighbors(Q, k)

    class AB(FakeAB):
        KNN = SlowKNN

    rng = np.random.default_rng(4)
    X = rng.standard_normal((300, 4)).astype(np.float32)
    server = sv.Server(AB(), X, workers=1, max_batch_queries=512, max_request_queries=512,
                       small_queries=8, aging_ms=10_000.0)
    try:
        block = server.submit(sv.Request("knn", rng.standard_normal((2, 4)), k=1))
        time.sleep(0.2)                        # the worker is now inside the blocking call
        large = server.submit(sv.Request("knn", rng.standard_normal((300, 4)), k=1))
        small = server.submit(sv.Request("knn", rng.standard_normal((5, 4)), k=1))
        gate.set()
        for r in (block, large, small):
            assert r.wait(30)
        assert small.t_start <= large.t_start
    finally:
        gate.set()
        server.close()


class FakeApproxNN(FakeKNN):
    """Stands in for the IVF-flat handle: an exact search (all lists probed)."""

    def __init__(self, prec, order=None, **options):
        super().__init__(prec)
        self.options = options

    def set_training_data(self, X):
        return self.fit(X)

    def train_and_add(self):
        return self


def test_serving_ann_requests():
    """IVF-flat requests are batched on their own worker, split when larger
    than one call, and each gets its k-prefix; kNN requests are unaffected."""
    sv = _load("aoclda_serving_cpu3", os.path.join(PKG, "serving.py"))

    class AB(FakeAB):
        ApproxNN = FakeApproxNN

    rng = np.random.default_rng(5)
    X = rng.standard_normal((300, 6)).astype(np.float32)
    server = sv.Server(AB(), X, workers=1, max_batch_queries=16, max_request_queries=64,
                       ann={"n_list": 8, "n_probe": 8})
    try:
        assert server.ann.options == {"n_list": 8, "n_probe": 8, "seed": 0,
                                      "metric": "euclidean"}
        reqs = [server.submit(sv.Request(kind, rng.standard_normal((size, 6)), k=k))
                for kind, size, k in (("ann", 3, 5), ("ann", 40, 2), ("knn", 5, 3),
                                      ("ann", 16, 9))]
        for r in reqs:
            assert r.wait(30)
        ref = FakeKNN("s").fit(X)
        for r in reqs:
            ind, dist = ref.kneighbors(r.queries, r.k)
            np.testing.assert_array_equal(r.result[0], ind)
            np.testing.assert_array_equal(r.result[1], dist)
        ann_batches = [b for b in server.batches if b[0] == "ann"]
        assert ann_batches and max(b[2] for b in ann_batches) <= 16
    finally:
        server.close()
    # without an index, "ann" requests are refused
    plain = sv.Server(FakeAB(), X, workers=1, max_batch_queries=16, max_request_queries=64)
    try:
        try:
            plain.submit(sv.Request("ann", X[:2], k=1))
            raise AssertionError("an ann request without an index was accepted")
        except KeyError:
            pass
    finally:
        plain.close()


def test_serving_library_error_completes_the_batch():
    """A library call that raises completes its requests with the error (and a
    split request's parent), and the worker keeps serving the next ones."""
    sv = _load("aoclda_serving_err", os.path.join(PKG, "serving.py"))

    class FailingKNN(FakeKNN):
        def kneighbors(self, Q, k):
            if k == 13:
                raise RuntimeError("da_nn_kneighbors_s: status 2 (memory_error)")
            return super().kneighbors(Q, k)

    class AB(FakeAB):
        KNN = FailingKNN

    rng = np.random.default_rng(9)
    X = rng.standard_normal((300, 4)).astype(np.float32)
    server = sv.Server(AB(), X, workers=1, max_batch_queries=8, max_request_queries=32,
                       free_memory=None)
    try:
        bad = server.submit(sv.Request("knn", rng.standard_normal((20, 4)), k=13))
        assert bad.wait(30)
        assert bad.error and "memory_error" in bad.error
        good = server.submit(sv.Request("knn", rng.standard_normal((5, 4)), k=3))
        assert good.wait(30) and good.error is None
        ind, dist = FakeKNN("s").fit(X).kneighbors(good.queries, 3)
        np.testing.assert_array_equal(good.result[0], ind)
    finally:
        server.close()


def test_serving_admission_follows_free_memory():
    """With little device memory free, batches shrink to what fits (but the
    oldest request is always taken)."""
    sv = _load("aoclda_serving_adm", os.path.join(PKG, "serving.py"))
    rng = np.random.default_rng(10)
    X = rng.standard_normal((200, 4)).astype(np.float32)
    free = {"bytes": 1 << 40}
    gate = threading.Event()
    armed = {"on": False}  # the start-up warm-up calls do not wait

    class SlowKNN(FakeKNN):
        def kneighbors(self, Q, k):
            if armed["on"]:
                gate.wait(10)
            return super().kneighbors(Q, k)

    class AB(FakeAB):
        KNN = SlowKNN

    server = sv.Server(AB(), X, workers=1, max_batch_queries=64, max_request_queries=64,
                       free_memory=lambda: free["bytes"], hbm_reserve=0)
    armed["on"] = True
    try:
        per_query = server.bytes_per_query
        first = server.submit(sv.Request("knn", rng.standard_normal((1, 4)), k=1))
        time.sleep(0.2)  # the worker holds the first batch
        free["bytes"] = 3 * per_query  # room for three queries per batch
        server.refresh_free_memory()
        later = [server.submit(sv.Request("knn", rng.standard_normal((1, 4)), k=1))
                 for _ in range(7)]
        gate.set()
        for r in [first] + later:
            assert r.wait(30)
        sizes = [b[2] for b in server.batches if b[0] == "knn"][1:]
        assert max(sizes) <= 3 and sum(sizes) == 7
    finally:
        gate.set()
        server.close()


def test_serving_fast_lane():
    """With two kNN workers the first serves only small requests (its batches
    never hold a request of more than small_queries queries); every result is
    still the request's own search."""
    sv = _load("aoclda_serving_fast", os.path.join(PKG, "serving.py"))
    rng = np.random.default_rng(8)
    X = rng.standard_normal((300, 4)).astype(np.float32)
    server = sv.Server(FakeAB(), X, workers=2, max_batch_queries=16, max_request_queries=64,
                       small_queries=4)
    try:
        reqs = [server.submit(sv.Request("knn", rng.standard_normal((int(m), 4)), k=3))
                for m in rng.choice([1, 2, 4, 9, 16, 40], 120)]
        for r in reqs:
            assert r.wait(30)
        ref = FakeKNN("s").fit(X)
        for r in reqs:
            ind, dist = ref.kneighbors(r.queries, 3)
            np.testing.assert_array_equal(r.result[0], ind)
        fast = server.threads[0].ident
        mine = [b for b in server.batches if b[0] == "knn" and b[5] == fast]
        assert mine, "the fast lane served nothing"
        assert all(b[4] <= 4 for b in mine)
        assert any(b[4] > 4 for b in server.batches if b[0] == "knn")
    finally:
        server.close()


def test_serving_two_fast_lanes_with_a_cap():
    """Two fast lanes of three kNN workers, each fast-lane call at most
    fast_lane_max_queries queries; results are every request's own search."""
    sv = _load("aoclda_serving_fast2", os.path.join(PKG, "serving.py"))
    rng = np.random.default_rng(9)
    X = rng.standard_normal((300, 4)).astype(np.float32)
    server = sv.Server(FakeAB(), X, workers=3, fast_lanes=2, fast_lane_max_queries=6,
                       max_batch_queries=16, max_request_queries=64, small_queries=4)
    try:
        reqs = [server.submit(sv.Request("knn", rng.standard_normal((int(m), 4)), k=2))
                for m in rng.choice([1, 2, 3, 4, 9, 30], 150)]
        for r in reqs:
            assert r.wait(30)
        ref = FakeKNN("s").fit(X)
        for r in reqs:
            np.testing.assert_array_equal(r.result[0], ref.kneighbors(r.queries, 2)[0])
        fast = {server.threads[0].ident, server.threads[1].ident}
        mine = [b for b in server.batches if b[0] == "knn" and b[5] in fast]
        assert mine and all(b[2] <= 6 and b[4] <= 4 for b in mine)
    finally:
        server.close()
