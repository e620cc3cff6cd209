"""Model persistence (da_handle_save_model / da_handle_load_model) without a
GPU: a kNN handle with training data, labels and options set round-trips
(options, classes, and a second save of the loaded handle is byte-identical
to the first); the error paths follow the reference's statuses."""
import ctypes as C

import numpy as np

IO_ERROR, INVALID_POINTER, NO_DATA = 26, 3, 20
INVALID_FILE_DATA, VERSION_MISMATCH = 801, 802


def test_knn_model_round_trip(ab, tmp_path):
    rng = np.random.default_rng(0)
    X = rng.standard_normal((57, 6))
    y = rng.integers(0, 4, 57).astype(np.int32)
    nn = ab.KNN("d", order=ab.ROW_MAJOR, number_of_neighbors=7, metric="manhattan",
                weights="distance")
    nn.fit(X, y)
    f1 = tmp_path / "knn1.bin"
    nn.save_model(f1)
    nn2 = ab.KNN.load_model(f1, "d")
    assert nn2.get_int("number of neighbors") == 7
    assert nn2.get_string("metric") == "manhattan"
    assert nn2.get_string("weights") == "distance"
    assert nn2.order == ab.ROW_MAJOR
    np.testing.assert_array_equal(nn2.classes(), np.unique(y))
    f2 = tmp_path / "knn2.bin"
    nn2.save_model(f2)
    assert f1.read_bytes() == f2.read_bytes()
    nn.close()
    nn2.close()


def test_model_file_errors(ab, tmp_path):
    L = ab.lib()
    h = C.c_void_p()
    assert L.da_handle_load_model(C.byref(h), str(tmp_path / "missing").encode()) == IO_ERROR
    assert L.da_handle_load_model(None, b"x") == INVALID_POINTER
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"not a model file at all")
    assert L.da_handle_load_model(C.byref(h), str(bad).encode()) == INVALID_FILE_DATA
    # an untrained k-means handle cannot be saved
    km = ab.KMeans(3, "s")
    assert L.da_handle_save_model(km.h, str(tmp_path / "km.bin").encode()) == NO_DATA
    km.close()
    # nor an untrained IVF-flat handle
    ivf = ab.ApproxNN("d", n_list=2)
    assert L.da_handle_save_model(ivf.h, str(tmp_path / "ivf.bin").encode()) == NO_DATA
    ivf.close()
    assert L.da_handle_save_model(None, b"x") == INVALID_POINTER
    # a valid file, corrupted: the checksum rejects it; another format version
    rng = np.random.default_rng(1)
    nn = ab.KNN("s").fit(rng.standard_normal((20, 3)))
    good = tmp_path / "good.bin"
    nn.save_model(good)
    nn.close()
    data = bytearray(good.read_bytes())
    data[40] ^= 0xFF
    bad.write_bytes(bytes(data))
    assert L.da_handle_load_model(C.byref(h), str(bad).encode()) == INVALID_FILE_DATA
    data = bytearray(good.read_bytes())
    data[12] = 2                                  # format version 2
    body = bytes(data[:-8])
    hsum = 1469598103934665603
    for ch in body:
        hsum = ((hsum ^ ch) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    bad.write_bytes(body + hsum.to_bytes(8, "little"))
    assert L.da_handle_load_model(C.byref(h), str(bad).encode()) == VERSION_MISMATCH
    # a handle slot that is not empty
    h2 = C.c_void_p(12345)
    assert L.da_handle_load_model(C.byref(h2), str(good).encode()) == INVALID_POINTER
