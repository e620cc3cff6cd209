"""Model files written by AOCL-DA's own da_handle_save_model load through
da_handle_load_model (host part: no device needed).

The files come from tests/refmodel.py, a restatement of the reference's
serializer.  The metadata checks follow the reference's
LoadCorruptedFileMetadataValidation
(tests/unit_tests/model_persistence/handle_errors_public.cpp:209-300): a
wrong keyword, da_int size or precision is da_status_invalid_file_data, a
serialization version other than 50301 da_status_version_mismatch; a handle
type outside this library is da_status_not_implemented; a truncated or
inconsistent body is da_status_invalid_file_data."""
import ctypes as C

import numpy as np
import pytest

import refmodel as rm

SUCCESS, NOT_IMPLEMENTED, INVALID_FILE_DATA, VERSION_MISMATCH = 0, 5, 801, 802


def load_status(ab, path):
    h = C.c_void_p()
    st = ab.lib().da_handle_load_model(C.byref(h), str(path).encode())
    if st == SUCCESS:
        ab.lib().da_handle_destroy(C.byref(h))
    return st


def small_kmeans(tmp_path, prec="d", order=rm.COLUMN_MAJOR, **kw):
    rng = np.random.default_rng(3)
    C0 = rng.standard_normal((4, 3))
    lab = rng.integers(0, 4, 50)
    f = tmp_path / "km.model"
    rm.kmeans_file(f, prec, order, C0, lab, 7, 12.5, **kw)
    return f, C0, lab


def test_status_codes(ab):
    # the codes this module expects are the C API's
    import re
    import os
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "aoclda_b200.h")).read()
    for name, v in (("da_status_invalid_file_data", INVALID_FILE_DATA),
                    ("da_status_version_mismatch", VERSION_MISMATCH)):
        assert re.search(rf"{name}\s*=\s*{v}\b", hdr), name


@pytest.mark.parametrize("prec", ["s", "d"])
@pytest.mark.parametrize("order", [rm.COLUMN_MAJOR, rm.ROW_MAJOR])
def test_kmeans_model_results(ab, tmp_path, prec, order):
    f, C0, lab = small_kmeans(tmp_path, prec, order)
    km = ab.KMeans.load_model(f, prec)
    dt = np.float32 if prec == "s" else np.float64
    np.testing.assert_array_equal(km.centres(4, 3), C0.astype(dt))
    np.testing.assert_array_equal(km.labels(50), lab)
    r = km.rinfo()
    assert list(r[:4]) == [50, 3, 4, 7]
    assert r[4] == np.asarray(12.5, dtype=dt)
    assert km.get_int("n_clusters") == 4
    assert km.get_string("storage order") == ("row-major" if order == rm.ROW_MAJOR
                                              else "column-major")
    km.close()


def test_metadata_validation(ab, tmp_path):
    rng = np.random.default_rng(0)
    C0, lab = rng.standard_normal((2, 2)), np.array([0, 1, 1])
    cases = [(dict(keyword="AOCLDA_STORED_MODEX"), INVALID_FILE_DATA),
             (dict(version=50300), VERSION_MISMATCH),
             (dict(version=50302), VERSION_MISMATCH),
             (dict(int_size=2), INVALID_FILE_DATA),
             (dict(precision=2), INVALID_FILE_DATA)]
    for meta, want in cases:
        w = rm.Writer("d")
        w.metadata(rm.HANDLE_KMEANS, **meta)
        w.registry([])
        f = tmp_path / "bad.model"
        w.save(f)
        assert load_status(ab, f) == want, meta
    # a handle type this library does not provide (PCA)
    w = rm.Writer("d")
    w.metadata(2)
    w.registry([])
    f = tmp_path / "pca.model"
    w.save(f)
    assert load_status(ab, f) == NOT_IMPLEMENTED
    # truncated bodies, an unknown option, an inconsistent size
    f, _, _ = small_kmeans(tmp_path)
    data = f.read_bytes()
    for cut in (len(data) - 1, len(data) - 40, 200, 90):
        g = tmp_path / "cut.model"
        g.write_bytes(data[:cut])
        assert load_status(ab, g) == INVALID_FILE_DATA, cut
    w = rm.Writer("d")
    w.metadata(rm.HANDLE_KMEANS)
    w.registry([("no such option", "I", 1)])
    w.save(tmp_path / "opt.model")
    assert load_status(ab, tmp_path / "opt.model") == INVALID_FILE_DATA
    g = tmp_path / "lab.model"
    rm.kmeans_file(g, "d", rm.COLUMN_MAJOR, C0, np.array([0, 1, 5]), 1, 1.0)  # label >= k
    assert load_status(ab, g) == INVALID_FILE_DATA


def test_nn_and_ivf_models_load(ab, tmp_path):
    rng = np.random.default_rng(1)
    X = rng.standard_normal((40, 5))
    y = rng.integers(0, 3, 40)
    f = tmp_path / "nn.model"
    rm.nn_file(f, "d", rm.ROW_MAJOR, X, y=y, n_neighbors=4, metric="manhattan",
               algorithm="kd tree", tree_bytes=b"\x01" * 64)
    nn = ab.KNN.load_model(f, "d")
    assert nn.get_string("metric") == "manhattan" and nn.get_int("number of neighbors") == 4
    nn.close()
    # IVF-flat: two lists
    Cn = np.array([[0.0] * 5, [1.0] * 5])
    rows = [X[:25], X[25:]]
    ids = [np.arange(25), np.arange(25, 40)]
    g = tmp_path / "ivf.model"
    rm.ivf_file(g, "d", rm.COLUMN_MAJOR, Cn, rows, ids, 40, metric="inner product", n_probe=2)
    h = ab.ApproxNN.load_model(g, "d")
    assert list(h.list_sizes(2)) == [25, 15]
    got = h.result(ab.APPROX_NN_CENTROIDS, 10).reshape(5, 2).T
    np.testing.assert_array_equal(got, Cn)
    assert h.get_string("metric") == "inner product" and h.get_int("n_probe") == 2
    h.close()
