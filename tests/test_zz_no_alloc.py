"""da_b200_knn_euclidean_noalloc_s: the k-nearest-neighbour search for callers
that cannot allocate device memory.  Its working memory is a fixed array in
the library, so its results are checked against da_nn_kneighbors_s (the
handle path, which allocates its own buffers) and, where the oracle's search
is quick, against the oracle, on two calls in a row -- the
second call runs over what the first left in the shared array -- plus a
repeat of the first.  kNN results are compared bit for bit, as in the other
kNN tests.  This file is collected last so that it also runs after every
other test in the same process."""
import ctypes as C

import numpy as np
import pytest

STATUS_INVALID_ARRAY_DIMENSION = 17


def _entry(ab):
    f = ab.lib().da_b200_knn_euclidean_noalloc_s
    f.argtypes = [C.c_void_p, ab.da_int, C.c_void_p, ab.da_int, ab.da_int, ab.da_int, ab.da_int,
                  C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _reference(ab, X, Q, k):
    knn = ab.KNN("s", order=ab.ROW_MAJOR, metric="euclidean")
    knn.fit(X)
    ind, dist = knn.kneighbors(Q, k)
    knn.close()
    return ind, dist


@pytest.mark.gpu
def test_knn_noalloc_matches_kneighbors(ab, orc, gpu):
    import torch

    f = _entry(ab)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    # the last: one query over a million rows with k = 256, where the merge
    # fan-in cap bounds the number of partial lists
    cases = [(5000, 300, 37, 10, 11), (20000, 1000, 64, 200, 12), (5000, 300, 37, 10, 11),
             (1_000_000, 1, 32, 256, 13)]
    for n, nq, d, k, seed in cases:
        rng = np.random.default_rng(seed)
        X = rng.standard_normal((n, d)).astype(np.float32)
        Q = rng.standard_normal((nq, d)).astype(np.float32)
        X[7] = X[3]  # exact ties between training rows
        ind_ref, dist_ref = _reference(ab, X, Q, k)

        ld = (d + 3) // 4 * 4
        Xd = torch.zeros((n, ld), dtype=torch.float32, device=dev)
        Qd = torch.zeros((nq, ld), dtype=torch.float32, device=dev)
        Xd[:, :d] = torch.from_numpy(X).to(dev)
        Qd[:, :d] = torch.from_numpy(Q).to(dev)
        dist = torch.full((nq, k), -1.0, dtype=torch.float32, device=dev)
        ind = torch.full((nq, k), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize(dev)
        st = f(Xd.data_ptr(), n, Qd.data_ptr(), nq, d, ld, k, dist.data_ptr(), ind.data_ptr(),
               stream)
        assert st == 0
        torch.cuda.synchronize(dev)
        np.testing.assert_array_equal(ind.cpu().numpy(), ind_ref)
        np.testing.assert_array_equal(dist.cpu().numpy(), dist_ref)
        if n * nq <= 20_000_000:
            # and the oracle's search (the reference's arithmetic, ties to
            # the lower index)
            oind, odist = orc.knn(X, Q, k, "euclidean")
            np.testing.assert_array_equal(ind.cpu().numpy(), oind)
            np.testing.assert_array_equal(dist.cpu().numpy(), odist)


@pytest.mark.gpu
def test_knn_noalloc_rejects_oversized(ab, gpu):
    import torch

    f = _entry(ab)
    dev = torch.device("cuda:0")
    n, nq, d, k = 1000, 20000, 8, 256  # 20000 * 256 * 8 bytes > the 32 MiB scratch
    Xd = torch.zeros((n, d), dtype=torch.float32, device=dev)
    Qd = torch.zeros((nq, d), dtype=torch.float32, device=dev)
    dist = torch.zeros((nq, k), dtype=torch.float32, device=dev)
    ind = torch.zeros((nq, k), dtype=torch.int32, device=dev)
    st = f(Xd.data_ptr(), n, Qd.data_ptr(), nq, d, d, k, dist.data_ptr(), ind.data_ptr(), None)
    assert st == STATUS_INVALID_ARRAY_DIMENSION
