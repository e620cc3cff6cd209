"""Spherical (cosine) k-means through the C ABI ("distance" = "cosine").

The reference's own spherical tests (kmeans_public.cpp:722-1200,
kmeans_test.py:313-337) assert properties: unit-length centres, results
invariant to scaling the data, predict / transform of scaled centres, the
same answer with "normalize data" on and off for normalised data, and
recovery of an empty cluster by splitting.  They are repeated here on their
data (tests/golden/kmeans_spherical.npz) for Lloyd and Elkan, every
initialisation and both storage orders.  Parity with the oracle
(oracle.c, orc_kmeans_sph_lloyd_*) is checked on larger sets: labels
exact unless the trajectory passes a near-tie, centres relative 1e-5 (fp32) /
1e-12 (fp64), the returned labels exactly the assignment to the returned
centres, the inertia the oracle's for those labels and centres; k-means++
chooses the oracle's rows."""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

TOL = {"s": 1e-6, "d": 1e-12}
DT = {"s": np.float32, "d": np.float64}


def unit_norms(C):
    return (C.astype(np.float64) ** 2).sum(1)


def fit(ab, A, k, prec, order, init, alg="lloyd", C0=None, **kw):
    km = ab.KMeans(k, prec, order=order, n_init=1, seed=42, distance="cosine", **kw)
    km.set("algorithm", alg)
    if C0 is None:
        km.set("initialization method", init)
    km.fit(A, C0=C0)
    return km


@pytest.mark.parametrize("prec", ["s", "d"])
@pytest.mark.parametrize("order", [0, 1])
def test_spherical_reference_properties(gpu, ab, prec, order):
    z = golden("kmeans_spherical.npz")
    A = z["A"].astype(DT[prec])
    tol = TOL[prec]
    for alg in ("lloyd", "elkan"):
        for init in ("random", "k-means++", "afk-mc2"):
            km = fit(ab, A, 3, prec, order, init, alg, normalize_data="yes")
            C = km.centres(3, 3)
            np.testing.assert_allclose(unit_norms(C), 1.0, atol=tol, err_msg=f"{alg} {init}")
            km2 = fit(ab, 2 * A, 3, prec, order, init, alg, normalize_data="yes")
            C2 = km2.centres(3, 3)
            np.testing.assert_allclose(unit_norms(C2), 1.0, atol=tol)
            np.testing.assert_allclose(C, C2, atol=tol, err_msg=f"{alg} {init} scaled")
            Xt = (2 * C2).astype(DT[prec])
            np.testing.assert_array_equal(km2.predict(Xt), np.arange(3))
            T = km2.transform(Xt, 3)
            np.testing.assert_allclose(np.diag(T), 0.0, atol=tol)
            km.close()
            km2.close()
        # unnormalised supplied centres
        km = fit(ab, A, 3, prec, order, None, alg, C0=z["C"].astype(DT[prec]))
        np.testing.assert_allclose(unit_norms(km.centres(3, 3)), 1.0, atol=tol)
        km.close()


@pytest.mark.parametrize("prec", ["s", "d"])
def test_spherical_normalise_on_off(gpu, ab, prec):
    z = golden("kmeans_spherical.npz")
    A = z["A"].astype(DT[prec])
    nrm = np.sqrt((A * A).sum(1, dtype=A.dtype))
    An = (A * (1 / nrm)[:, None]).astype(A.dtype)
    for order in (0, 1):
        for init in ("random", "k-means++", "afk-mc2"):
            on = fit(ab, An, 3, prec, order, init, normalize_data="yes")
            off = fit(ab, An, 3, prec, order, init, normalize_data="no")
            np.testing.assert_array_equal(on.labels(20), off.labels(20))
            np.testing.assert_allclose(on.centres(3, 3), off.centres(3, 3), atol=TOL[prec])


@pytest.mark.parametrize("prec", ["s", "d"])
@pytest.mark.parametrize("order", [0, 1])
def test_spherical_empty_cluster_split(gpu, ab, prec, order):
    z = golden("kmeans_spherical.npz")
    A = z["ec_A"].astype(DT[prec])
    for alg in ("lloyd", "elkan"):
        km = ab.KMeans(2, prec, order=order, distance="cosine", empty_clusters="split")
        km.set("algorithm", alg)
        km.fit(A, C0=z["ec_C"].astype(DT[prec]))
        lab = km.labels(5)
        assert set(lab) == {0, 1}
        np.testing.assert_allclose(unit_norms(km.centres(2, 2)), 1.0, atol=TOL[prec])
        # "error" reports the empty cluster (da_status_empty_clusters)
        km = ab.KMeans(2, prec, order=order, distance="cosine", empty_clusters="error")
        km.set("algorithm", alg)
        km.fit(A, C0=z["ec_C"].astype(DT[prec]), ok=(900,))


def test_spherical_python_case(gpu, ab):
    a = golden("kmeans_spherical.npz")["py_a"]
    for prec in ("s", "d"):
        km = ab.KMeans(2, prec, n_init=1, seed=42, distance="cosine", normalize_data="no")
        km.fit(a.astype(DT[prec]))
        np.testing.assert_allclose(np.linalg.norm(km.centres(2, 3).astype(np.float64), axis=1),
                                   1.0, atol=TOL[prec])


def _mixture(rng, n, d, k, dtype):
    dirs = rng.standard_normal((k, d))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    lab = rng.integers(0, k, n)
    X = dirs[lab] * 4 + rng.standard_normal((n, d))
    X *= rng.uniform(0.1, 10.0, n)[:, None]            # row norms vary widely
    return X.astype(dtype)


@pytest.mark.parametrize("prec,n,d,k,normalise",
                         [("s", 20000, 64, 37, True), ("s", 30000, 33, 100, False),
                          ("s", 5000, 200, 16, True), ("d", 8000, 12, 9, True),
                          ("d", 3000, 40, 25, False)])
def test_spherical_supplied_vs_oracle(gpu, ab, orc, prec, n, d, k, normalise):
    rng = np.random.default_rng(n + d + k)
    dt = DT[prec]
    A = _mixture(rng, n, d, k, dt)
    if not normalise:
        A = (A / np.linalg.norm(A.astype(np.float64), axis=1, keepdims=True)).astype(dt)
    C0 = A[rng.choice(n, k, replace=False)] * 3
    km = ab.KMeans(k, prec, order=1, max_iter=60, n_init=1, distance="cosine",
                   normalize_data="yes" if normalise else "no")
    km.fit(A, C0=C0)
    C, lab, nit, inertia = orc.kmeans_sph_lloyd(A, C0, 60, 1e-4, normalise)
    r = km.rinfo()
    glab = km.labels(n)
    gC = km.centres(k, d)
    rtol = 1e-5 if prec == "s" else 1e-12
    if np.array_equal(glab, lab):
        assert int(r[3]) == nit
        np.testing.assert_allclose(gC, C, rtol=rtol, atol=rtol)
    # whatever the trajectory: unit-length centres, labels = the assignment to
    # the returned centres (same fma order -> exact), inertia = the oracle's
    np.testing.assert_allclose(unit_norms(gC[np.bincount(glab, minlength=k) > 0]), 1.0,
                               atol=10 * TOL[prec])
    lab2, _ = orc.kmeans_assign_sph(A, gC)
    np.testing.assert_array_equal(glab, lab2)
    want = orc.kmeans_inertia_sph(A, glab, gC, normalise)
    assert abs(r[4] - want) <= 1e-9 * abs(want) + 1e-9


@pytest.mark.parametrize("prec", ["s", "d"])
def test_spherical_kmeanspp_rows_match_oracle(gpu, ab, orc, prec):
    rng = np.random.default_rng(5)
    dt = DT[prec]
    A = _mixture(rng, 30000, 24, 40, dt)
    for normalise in (True, False):
        km = ab.KMeans(40, prec, order=1, seed=11, distance="cosine",
                       normalize_data="yes" if normalise else "no")
        km.set("initialization method", "k-means++")
        km.set_data(A)
        got = km.init_centres(40)
        rows = orc.kmeanspp_cosine(A, 40, 11, normalise)
        want = A[rows].astype(np.float64)
        want /= np.sqrt((want ** 2).sum(1, keepdims=True))
        np.testing.assert_allclose(got, want.astype(dt), rtol=4 * TOL[prec], atol=4 * TOL[prec])


def test_spherical_predict_transform_and_persistence(gpu, ab, orc):
    rng = np.random.default_rng(9)
    A = _mixture(rng, 10000, 16, 12, np.float32)
    Y = _mixture(rng, 500, 16, 12, np.float32)
    km = ab.KMeans(12, "s", order=1, n_init=2, seed=3, distance="cosine")
    km.fit(A)
    C = km.centres(12, 16)
    lab, _ = orc.kmeans_assign_sph(Y, C)
    np.testing.assert_array_equal(km.predict(Y), lab)
    T = km.transform(Y, 12)
    y64 = Y.astype(np.float64)
    cos = (y64 @ C.astype(np.float64).T) / np.linalg.norm(y64, axis=1, keepdims=True)
    np.testing.assert_allclose(T, 1 - np.clip(cos, -1, 1), atol=2e-6)
    f = os.path.join(tempfile.mkdtemp(), "sph.model")
    km.save_model(f)
    km2 = ab.KMeans.load_model(f, "s")
    np.testing.assert_array_equal(km2.predict(Y), lab)
    np.testing.assert_array_equal(km2.transform(Y, 12), T)


def test_spherical_errors(gpu, ab):
    A = np.random.default_rng(0).standard_normal((100, 4))
    km = ab.KMeans(3, "d", distance="cosine")
    km.set("algorithm", "hartigan-wong")
    km.fit(A, ok=(13,))                      # da_status_incompatible_options
    km = ab.KMeans(3, "d", distance="cosine")
    km.set("algorithm", "macqueen")
    km.fit(A, ok=(5,))                       # not provided (da_status_not_implemented)


@pytest.mark.parametrize("n,d,k,normalise", [(100000, 64, 256, True), (33333, 37, 100, False),
                                             (20000, 128, 64, True), (5000, 200, 16, True)])
def test_spherical_tensor_core_equals_plain(gpu, ab, n, d, k, normalise):
    """The tcgen05 candidate passes (bias columns zero, error bound from
    unit-length centres) give exactly the plain fp32 path's labels, centres,
    iteration count and inertia."""
    rng = np.random.default_rng(n + k + 1)
    A = _mixture(rng, n, d, max(k // 2, 2), np.float32)
    if not normalise:
        A = (A / np.linalg.norm(A.astype(np.float64), axis=1, keepdims=True)).astype(np.float32)
    C0 = A[rng.choice(n, k, replace=False)].copy()
    out = {}
    for mode in ("plain", "bf16", "bf16x3"):
        km = ab.KMeans(k, "s", order=0, max_iter=25, n_init=1, distance="cosine",
                       normalize_data="yes" if normalise else "no")
        km.set("precision mode", mode)
        km.fit(A, C0=C0)
        out[mode] = (km.labels(n), km.centres(k, d), km.rinfo(), km.stat("tensor_core"))
    assert out["plain"][3] == 0.0
    assert out["bf16x3"][3] == (1.0 if d <= 128 else 0.0)  # d = 200: no tensor-core pass
    for mode in ("bf16", "bf16x3"):
        np.testing.assert_array_equal(out["plain"][0], out[mode][0])
        np.testing.assert_array_equal(out["plain"][1], out[mode][1])
        np.testing.assert_array_equal(out["plain"][2], out[mode][2])
