"""The serving loop (aocl-data-analytics_b200/serving.py): kNN and k-means
predict requests of different sizes, some arriving in a burst (so that they
are batched together) and some paced, served by two kNN workers and a predict
worker over device-resident data.  Every request's result must be exactly
what the same request gives alone (its own library call on its own handle):
a kNN request batched with others is searched with a larger k and gets the
prefix it asked for, and one larger than a call takes is served in parts."""
import numpy as np
import pytest

from conftest import PKG, _load

pytestmark = pytest.mark.gpu


def mixture(rng, n, d, comps):
    means = rng.uniform(-10.0, 10.0, (comps, d))
    lab = rng.integers(0, comps, n)
    return (means[lab] + rng.standard_normal((n, d))).astype(np.float32)


def test_serving_results_alone_and_in_the_mix(gpu, ab):
    import os
    sv = _load("aoclda_serving", os.path.join(PKG, "serving.py"))
    rng = np.random.default_rng(7)
    nx, d = 300_000, 64
    X = mixture(rng, nx, d, 128)
    models = {}
    for m in range(3):
        Xm = mixture(rng, 20_000, d, 32)
        models[f"m{m}"] = (Xm, Xm[rng.choice(Xm.shape[0], 32, replace=False)].copy())
    # calls of at most 128 queries: the larger requests are split into parts
    server = sv.Server(ab, X, models=models, workers=2, max_batch_queries=128)
    try:
        def queries(size):
            return mixture(rng, size, d, 128)

        trace = []
        for i in range(24):   # burst: all at t = 0
            size = int(np.clip(rng.lognormal(np.log(40), 1.0), 1, 300))
            if i % 4 == 3:
                trace.append((0.0, "predict", size, f"m{i % 3}"))
            else:
                trace.append((0.0, "knn", size, int(rng.choice([1, 10, 100]))))
        t = 0.0
        for i in range(40):   # paced: Poisson arrivals at 2,000 requests/s
            t += rng.exponential(1 / 2000.0)
            size = int(np.clip(rng.lognormal(np.log(20), 1.0), 1, 256))
            if i % 5 == 4:
                trace.append((t, "predict", size, f"m{i % 3}"))
            else:
                trace.append((t, "knn", size, int(rng.choice([1, 10, 100]))))
        reqs = sv.replay(server, trace, queries)
        assert all(r.result is not None for r in reqs)
        assert any(r.kind == "knn" and r.queries.shape[0] > 128 for r in reqs)
        assert max(b[1] for b in server.batches if b[0] == "knn") > 1
        summary = sv.latency_summary(reqs)
        assert summary["requests"] == len(reqs)
    finally:
        server.close()

    # the same requests, one library call each
    alone_knn = ab.KNN("s", order=ab.ROW_MAJOR, metric="euclidean").fit(X)
    alone_km = {}
    for name, (Xm, C0) in models.items():
        km = ab.KMeans(C0.shape[0], "s", order=ab.ROW_MAJOR, max_iter=50, n_init=1)
        km.fit(Xm, C0)
        alone_km[name] = km
    for r in reqs:
        if r.kind == "knn":
            ind, dist = alone_knn.kneighbors(r.queries, r.k)
            np.testing.assert_array_equal(r.result[0], ind)
            np.testing.assert_array_equal(r.result[1], dist)
        else:
            np.testing.assert_array_equal(r.result, alone_km[r.model].predict(r.queries))
    alone_knn.close()
    for km in alone_km.values():
        km.close()


def test_serving_ann_alone_and_in_the_mix(gpu, ab):
    """IVF-flat ("ann") requests served in a mix with kNN requests give, each,
    what one search of the same index gives alone: the top-k over the probed
    lists in (distance, index) order does not depend on the batch or on k."""
    import os
    sv = _load("aoclda_serving_ann", os.path.join(PKG, "serving.py"))
    rng = np.random.default_rng(12)
    nx, d = 100_000, 32
    X = mixture(rng, nx, d, 64)
    opts = {"n_list": 64, "n_probe": 8, "seed": 3}
    server = sv.Server(ab, X, workers=1, max_batch_queries=128, max_request_queries=512, ann=opts)
    try:
        trace = []
        for i in range(30):
            size = int(np.clip(rng.lognormal(np.log(20), 1.0), 1, 300))
            kind = "ann" if i % 3 else "knn"
            trace.append((0.0 if i < 10 else i * 5e-4, kind, size, int(rng.choice([1, 10, 50]))))
        reqs = sv.replay(server, trace, lambda size: mixture(rng, size, d, 64))
        assert all(r.error is None and r.result is not None for r in reqs)
        assert any(b[0] == "ann" and b[1] > 1 for b in server.batches)
    finally:
        server.close()
    lone = ab.ApproxNN("s", order=ab.ROW_MAJOR, metric="euclidean", **opts)
    lone.set_training_data(X).train_and_add()
    knn = ab.KNN("s", order=ab.ROW_MAJOR, metric="euclidean").fit(X)
    for r in reqs:
        h = lone if r.kind == "ann" else knn
        ind, dist = h.kneighbors(r.queries, r.k)
        np.testing.assert_array_equal(r.result[0], ind)
        np.testing.assert_array_equal(r.result[1], dist)
    lone.close()
    knn.close()
