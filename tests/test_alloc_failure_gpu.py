"""Device allocation failures, injected on the host: with
AOCLDA_B200_FAIL_ALLOC=N the library's N-th device allocation (counted from
the moment the variable takes that value) fails as an out-of-memory device
would.  For each public call, every allocation it makes is failed in turn
(N = 1, 2, ... until the call succeeds): the call must return
da_status_memory_error (the reference's status for a failed allocation,
utilities/da_error.hpp:163-260, metrics/partitioning_infrastructure.hpp:
206-227) and nothing else, and afterwards the same call on a fresh handle
must give the results of an undisturbed run.  No GPU fault is involved:
the failure is made before any device work that would use the memory."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMORY_ERROR = 2
ENV = "AOCLDA_B200_FAIL_ALLOC"


def sweep(ab, run, max_allocs=60):
    """run() -> result; returns (failures seen, clean result)."""
    os.environ.pop(ENV, None)
    want = run()
    failures = 0
    for n in range(1, max_allocs + 1):
        os.environ[ENV] = str(n)
        try:
            got = run()
        except ab.DAError as e:
            assert e.status == MEMORY_ERROR, f"allocation {n}: status {e.status} ({e})"
            failures += 1
            continue
        finally:
            os.environ.pop(ENV, None)
        # the n-th allocation was beyond this call's allocations: it succeeded
        _same(got, want)
        break
    else:
        pytest.fail("the call kept failing")
    # and a fresh handle afterwards gives the undisturbed results
    _same(run(), want)
    return failures, want


def _same(a, b):
    if isinstance(a, tuple):
        for x, y in zip(a, b):
            _same(x, y)
    else:
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b))


def test_alloc_failure_knn_plain_and_tensor_core(gpu, ab):
    rng = np.random.default_rng(3)
    for nx, d in ((3000, 16), (300_000, 64)):  # plain SIMT path, tensor-core pass
        X = rng.standard_normal((nx, d)).astype(np.float32)
        Q = rng.standard_normal((64, d)).astype(np.float32)

        def run():
            nn = ab.KNN("s", order=ab.ROW_MAJOR)
            try:
                nn.fit(X)
                return nn.kneighbors(Q, 10)
            finally:
                nn.close()

        failures, _ = sweep(ab, run)
        assert failures >= 2


def test_alloc_failure_kmeans_tensor_core_and_kmeanspp(gpu, ab):
    rng = np.random.default_rng(4)
    A = (rng.standard_normal((40_000, 32)) + rng.integers(0, 20, 40_000)[:, None]).astype(np.float32)

    def run():
        km = ab.KMeans(20, "s", order=ab.ROW_MAJOR, max_iter=20, n_init=1, seed=2)
        try:
            km.fit(A)
            return km.labels(A.shape[0]), km.centres(20, 32), km.rinfo()
        finally:
            km.close()

    failures, _ = sweep(ab, run)
    assert failures >= 5


def test_alloc_failure_pairwise_radius_ivf(gpu, ab):
    rng = np.random.default_rng(5)
    X = rng.standard_normal((2000, 8))
    Y = rng.standard_normal((300, 8))
    def pairwise():
        st, D = ab.pairwise_distances(X, Y, metric="euclidean", prec="d")
        if st != 0:
            raise ab.DAError(st, "da_pairwise_distances_d")
        return D

    sweep(ab, pairwise)

    def radius():
        nn = ab.KNN("d", order=ab.ROW_MAJOR)
        try:
            nn.fit(X)
            cnt, off, ind, dist = nn.radius_neighbors(Y[:20], 2.5, True, True)
            return cnt, off, ind, dist
        finally:
            nn.close()

    sweep(ab, radius)

    def ivf():
        h = ab.ApproxNN("d", order=ab.ROW_MAJOR, n_list=8, n_probe=3, seed=1)
        try:
            h.set_training_data(X).train_and_add()
            return h.kneighbors(Y, 5)
        finally:
            h.close()

    sweep(ab, ivf)


def test_alloc_failure_batched_kmeans(gpu, ab):
    rng = np.random.default_rng(6)
    Xs = [rng.standard_normal((n, d)).astype(np.float32) for n, d in ((3000, 16), (5000, 32))]
    C0s = [x[:8].copy() for x in Xs]

    def run():
        out = ab.kmeans_batched(Xs, C0s, max_iter=10, tol=1e-4)
        return tuple(np.asarray(r["labels"]) for r in out)

    failures, _ = sweep(ab, run)
    assert failures >= 1
