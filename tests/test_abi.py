"""C-ABI boundary tests that need no GPU: the library loads, exports every
symbol include/aoclda_b200.h declares, and reproduces the reference's host
logic (option registry, argument checks, status codes)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu


def header_functions():
    import glob
    text = "".join(open(f).read() for f in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:da_status|void)\s+(da_\w+)\s*\(", text, flags=re.M)))


def test_exports_every_declared_symbol(ab):
    lib = ab.lib()
    names = header_functions()
    assert len(names) >= 54
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_handle_lifecycle(ab):
    L = ab.lib()
    h = C.c_void_p()
    assert L.da_handle_init_d(C.byref(h), ab.HANDLE_NN) == 0
    assert h.value
    L.da_handle_destroy(C.byref(h))
    assert not h.value
    # handle types outside this path are not provided
    assert L.da_handle_init_s(C.byref(h), 1) == 5  # linmod -> not_implemented
    # null handle
    assert L.da_options_set_int(None, b"n_init", 3) == 10


def test_option_registry_semantics(ab):
    km = ab.Handle(ab.HANDLE_KMEANS, "d")
    L = km.L
    # case / whitespace insensitive names (options.hpp:192-202)
    assert L.da_options_set_int(km.h, b"  N_Clusters ", 7) == 0
    assert km.get_int("n_clusters") == 7
    assert km.get_int("max_iter") == 300 and km.get_int("n_init") == 10
    assert L.da_options_set_int(km.h, b"no such option", 1) == 400
    assert L.da_options_set_string(km.h, b"n_clusters", b"x") == 402
    assert L.da_options_set_int(km.h, b"n_clusters", 0) == 404
    assert L.da_options_set_string(km.h, b"initialization method", b"bogus") == 404
    assert L.da_options_set_string(km.h, b"initialization method", b" Supplied ") == 0
    assert km.get_string("initialization method") == "supplied"
    # precision of real options
    assert L.da_options_set_real_s(km.h, b"convergence tolerance", 1e-3) == 7
    assert L.da_options_set_real_d(km.h, b"convergence tolerance", -1.0) == 404
    assert L.da_options_set_real_d(km.h, b"convergence tolerance", 1e-6) == 0
    v = C.c_double()
    assert L.da_options_get_real_d(km.h, b"convergence tolerance", C.byref(v)) == 0
    assert v.value == 1e-6
    # string getter buffer size protocol (options_public.cpp:80-89)
    n = ab.da_int(3)
    buf = C.create_string_buffer(3)
    assert L.da_options_get_string(km.h, b"algorithm", buf, C.byref(n)) == 4
    assert n.value == len("lloyd") + 1
    key = ab.da_int(-1)
    n = ab.da_int(32)
    buf = C.create_string_buffer(32)
    assert L.da_options_get_string_key(km.h, b"storage order", buf, C.byref(n), C.byref(key)) == 0
    assert buf.value == b"column-major" and key.value == 1


def test_knn_argument_checks(ab):
    nn = ab.KNN("d")
    L = nn.L
    X = np.zeros((10, 3))
    ind = np.zeros((2, 2), dtype=np.int32)
    dist = np.zeros((2, 2))
    Q = np.zeros((2, 3))
    # no data yet
    assert L.da_nn_kneighbors_d(nn.h, 2, 3, ab.ptr(Q), 2, ab.ptr(ind), ab.ptr(dist), 2, 1) == 20
    # wrong precision
    assert L.da_nn_set_data_s(nn.h, 10, 3, ab.ptr(X.astype(np.float32)), 10) == 7
    # leading dimension / dimensions / null
    assert L.da_nn_set_data_d(nn.h, 10, 3, ab.ptr(X), 5) == 15
    assert L.da_nn_set_data_d(nn.h, 0, 3, ab.ptr(X), 10) == 17
    assert L.da_nn_set_data_d(nn.h, 10, 3, None, 10) == 3
    assert L.da_nn_set_data_d(nn.h, 10, 3, ab.ptr(np.asfortranarray(X)), 10) == 0
    # n_ind null, feature mismatch, k too large, n_dist null
    assert L.da_nn_kneighbors_d(nn.h, 2, 3, ab.ptr(Q), 2, None, ab.ptr(dist), 2, 1) == 3
    assert L.da_nn_kneighbors_d(nn.h, 2, 4, ab.ptr(Q), 2, ab.ptr(ind), ab.ptr(dist), 2, 1) == 17
    assert L.da_nn_kneighbors_d(nn.h, 2, 3, ab.ptr(Q), 2, ab.ptr(ind), ab.ptr(dist), 11, 1) == 4
    assert L.da_nn_kneighbors_d(nn.h, 2, 3, ab.ptr(Q), 2, ab.ptr(ind), None, 2, 1) == 3
    # labels of a different length
    y = np.zeros(9, dtype=np.int32)
    assert L.da_nn_set_labels_d(nn.h, 9, ab.ptr(y)) == 17
    # options locked after set_data with algorithm = auto (nearest_neighbors.cpp:429-463)
    assert nn.set("metric", "manhattan") == 0
    st = L.da_nn_kneighbors_d(nn.h, 2, 3, ab.ptr(Q), 2, ab.ptr(ind), ab.ptr(dist), 2, 1)
    assert st == 401
    # a kmeans call on a kNN handle
    assert L.da_kmeans_compute_d(nn.h) == 9


def test_kmeans_argument_checks(ab):
    km = ab.KMeans(4, "s")
    L = km.L
    assert L.da_kmeans_compute_s(km.h) == 20  # no data
    A = np.asfortranarray(np.random.default_rng(0).standard_normal((3, 2)).astype(np.float32))
    # n_clusters > n_samples is reduced with a warning (kmeans.cpp:283-289)
    st = L.da_kmeans_set_data_s(km.h, 3, 2, ab.ptr(A), 3)
    assert st == 13 and km.get_int("n_clusters") == 3
    assert km.set("initialization method", "supplied") == 0
    # supplied but no centres
    expect = 20 if True else None
    st = L.da_kmeans_compute_s(km.h)
    assert st == expect
    dim = ab.da_int(6)
    out = np.zeros(6, dtype=np.float32)
    assert L.da_handle_get_result_s(km.h, ab.RINFO, C.byref(dim), ab.ptr(out)) == 20
    # wrong result precision
    outd = np.zeros(6)
    assert L.da_handle_get_result_d(km.h, ab.RINFO, C.byref(dim), ab.ptr(outd)) == 7


@pytest.mark.skipif(has_gpu(), reason="checks the no-device behaviour")
def test_no_cpu_fallback(ab):
    """Without a GPU the compute entry points fail loudly (no CPU path)."""
    km = ab.KMeans(2, "d")
    A = np.asfortranarray(np.random.default_rng(0).standard_normal((10, 2)))
    L = km.L
    assert L.da_kmeans_set_data_d(km.h, 10, 2, ab.ptr(A), 10) == 0
    assert L.da_kmeans_compute_d(km.h) == 25  # arch_not_supported
    assert "CUDA" in km.message()
    st, _ = ab.pairwise_distances(A)
    assert st == 25
