"""Two kNN handles over one device copy of the training data
(da_b200_nn_share_data): the sharing handle allocates none of the rows or of
their tensor-core bf16 copies again, gives exactly the results of a handle
fitted on its own (tensor-core pass and plain path, concurrently with the
source on another thread), keeps working after the source is destroyed, and
a later set_data on it gives it fresh buffers without touching the other
handle's.  Argument errors come back as the statuses of the C API."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_share_data_memory_results_lifetime(gpu, ab):
    rng = np.random.default_rng(21)
    nx, d = 400_000, 64
    X = rng.standard_normal((nx, d)).astype(np.float32)
    Q = rng.standard_normal((256, d)).astype(np.float32)
    src = ab.KNN("s", order=ab.ROW_MAJOR).fit(X)
    want = src.kneighbors(Q, 10)              # builds the tensor-core copies
    assert src.stat("tensor_core") == 1.0
    plain_want = ab.KNN("s", order=ab.ROW_MAJOR, precision_mode="plain").fit(X)
    pw = plain_want.kneighbors(Q, 10)
    plain_want.close()

    free0 = _free_bytes()
    dst = ab.KNN("s", order=ab.ROW_MAJOR).share(src)
    free1 = _free_bytes()
    rows_bytes = nx * d * 4 * 2               # fp32 rows + the bf16 pair
    assert free0 - free1 < rows_bytes // 8, (free0, free1)

    # both handles searching at the same time on their own streams
    out = {}

    def search(name, h):
        out[name] = [h.kneighbors(Q, 10) for _ in range(4)]

    ts = [threading.Thread(target=search, args=(n, h)) for n, h in (("s", src), ("d", dst))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for name in ("s", "d"):
        for ind, dist in out[name]:
            np.testing.assert_array_equal(ind, want[0])
            np.testing.assert_array_equal(dist, want[1])
    assert dst.stat("tensor_core") == 1.0

    # a plain-path handle over the same shared rows
    pl = ab.KNN("s", order=ab.ROW_MAJOR, precision_mode="plain").share(src)
    ind, dist = pl.kneighbors(Q, 10)
    np.testing.assert_array_equal(ind, pw[0])
    np.testing.assert_array_equal(dist, pw[1])
    pl.close()

    # the source goes away; the shared copy stays with dst
    src.close()
    ind, dist = dst.kneighbors(Q, 10)
    np.testing.assert_array_equal(ind, want[0])
    np.testing.assert_array_equal(dist, want[1])

    # new data on a handle that shares: its own buffers, the other unchanged
    other = ab.KNN("s", order=ab.ROW_MAJOR).share(dst)
    X2 = X[::-1].copy()
    dst.fit(X2)
    i2, _ = dst.kneighbors(Q, 10)
    ref2 = ab.KNN("s", order=ab.ROW_MAJOR).fit(X2)
    np.testing.assert_array_equal(i2, ref2.kneighbors(Q, 10)[0])
    ref2.close()
    ind, dist = other.kneighbors(Q, 10)
    np.testing.assert_array_equal(ind, want[0])
    np.testing.assert_array_equal(dist, want[1])
    other.close()
    dst.close()


def test_share_data_labels_and_errors(gpu, ab):
    rng = np.random.default_rng(22)
    X = rng.standard_normal((2000, 8))
    y = rng.integers(0, 3, 2000)
    Q = rng.standard_normal((50, 8))
    src = ab.KNN("d", order=ab.ROW_MAJOR, number_of_neighbors=5).fit(X, y)
    dst = ab.KNN("d", order=ab.ROW_MAJOR, number_of_neighbors=5).share(src)
    np.testing.assert_array_equal(dst.predict(Q), src.predict(Q))

    fresh = ab.KNN("d", order=ab.ROW_MAJOR)
    with pytest.raises(ab.DAError) as e:            # source without data
        ab.KNN("d", order=ab.ROW_MAJOR).share(fresh)
    assert e.value.status == 20                      # da_status_no_data
    with pytest.raises(ab.DAError) as e:            # precision mismatch
        ab.KNN("s", order=ab.ROW_MAJOR).share(src)
    assert e.value.status == 7                       # da_status_wrong_type
    with pytest.raises(ab.DAError) as e:            # storage order mismatch
        ab.KNN("d", order=ab.COLUMN_MAJOR).share(src)
    assert e.value.status == 4                       # da_status_invalid_input
    with pytest.raises(ab.DAError) as e:            # different number of rows
        ab.KNN("d", order=ab.ROW_MAJOR).fit(X[:100]).share(src)
    assert e.value.status == 17                      # da_status_invalid_array_dimension
    for h in (src, dst, fresh):
        h.close()
