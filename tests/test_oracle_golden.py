"""Pins the CPU oracle against the reference's own known-answer tests.

The oracle (oracle/oracle.c) restates the AOCL-DA algorithms; before it is
trusted to check the GPU path it must reproduce the golden vectors
of the reference's test-suite (converted by tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from conftest import golden


def classify_mismatch(X, Q, got, want, dist64):
    """Indices that differ must be exact ties in fp64 distance."""
    bad = 0
    for q in range(len(got)):
        if np.array_equal(got[q], want[q]):
            continue
        a = np.sort(dist64[q][got[q]])
        b = np.sort(dist64[q][want[q]])
        if not np.allclose(a, b, rtol=1e-12, atol=0):
            bad += 1
    return bad


@pytest.mark.parametrize("tag", ["2092x2071x5", "2125x2068x20"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_knn_golden_csv(orc, tag, dtype):
    z = golden(f"nn_{tag}.npz")
    X = z["X_train"].astype(dtype)
    Q = z["X_test"].astype(dtype)
    ind, dist = orc.knn(X, Q, 5, "euclidean")
    eps = np.finfo(dtype).eps
    # reference tolerance: 500 * eps (nearest_neighbors_tests.hpp:636)
    np.testing.assert_allclose(dist, z["k_dist"], rtol=500 * eps, atol=500 * eps)
    d64 = np.sqrt(((Q.astype(np.float64)[:, None, :] - X.astype(np.float64)[None]) ** 2).sum(-1))
    assert classify_mismatch(X, Q, ind, z["k_ind"], d64) == 0


def test_oracle_knn_small_hand_problem(orc):
    z = golden("nn_small.npz")
    for k, ki, kd in ((3, "kind3", "kdist3"), (4, "kind4", "kdist4")):
        ind, dist = orc.knn(z["X_train"], z["X_test"], k, "euclidean")
        # expected arrays are n_queries x k column-major
        want_i = z[ki].reshape(k, 3).T
        want_d = z[kd].reshape(k, 3).T
        np.testing.assert_allclose(dist, want_d, rtol=40 * np.finfo(float).eps)
        # identical except exact ties: q2's 4th neighbour is a tie between rows
        # 0 and 2 (squared distance 38); the reference keeps the later row, the
        # oracle the lower index
        d64 = np.sqrt(((z["X_test"][:, None] - z["X_train"][None]) ** 2).sum(-1))
        assert classify_mismatch(None, None, ind, want_i, d64) == 0
        if k == 4:
            assert (ind[2, 3], want_i[2, 3]) == (0, 2)


def test_oracle_kmeans_lloyd80(orc):
    z = golden("kmeans_lloyd80.npz")
    C, lab, nit, inertia = orc.kmeans_lloyd(z["A"], z["C"], max_iter=30, tol=1e-4)
    assert nit == int(z["expected_rinfo"][3])
    np.testing.assert_array_equal(lab, z["expected_labels"])
    np.testing.assert_allclose(C, z["expected_centres"], rtol=1e-4, atol=1e-5)
    assert abs(inertia - z["expected_rinfo"][4]) < 1e-4


def test_oracle_kmeans_lloyd80_single(orc):
    z = golden("kmeans_lloyd80.npz")
    C, lab, nit, inertia = orc.kmeans_lloyd(z["A"].astype(np.float32),
                                            z["C"].astype(np.float32), max_iter=30, tol=1e-4)
    assert nit == int(z["expected_rinfo"][3])
    np.testing.assert_array_equal(lab, z["expected_labels"])
    np.testing.assert_allclose(C, z["expected_centres"], rtol=1e-4, atol=1e-4)


def test_oracle_sqeuclidean_order_matters(orc):
    """The two-accumulator order is not the naive order: pin that the oracle
    follows the reference's grouping (differs from a plain sequential sum on
    some inputs) while agreeing with fp64 to rounding."""
    rng = np.random.default_rng(3)
    X = rng.standard_normal((64, 37)).astype(np.float32) * 10
    Y = rng.standard_normal((48, 37)).astype(np.float32) * 10
    D = orc.pairwise(X, Y, "sqeuclidean")
    naive = np.zeros_like(D)
    for i in range(64):
        for j in range(48):
            g = np.float32(0)
            for t in range(37):
                dd = np.float32(X[i, t] - Y[j, t])
                g = np.float32(g + np.float32(dd * dd))
            naive[i, j] = g
    exact = ((X.astype(np.float64)[:, None] - Y.astype(np.float64)[None]) ** 2).sum(-1)
    np.testing.assert_allclose(D, exact, rtol=1e-5)
    assert not np.array_equal(D, naive)


def test_oracle_kc_slicing(orc):
    """d > KC: the slice boundary changes the summation order."""
    rng = np.random.default_rng(4)
    X = rng.standard_normal((8, 300)).astype(np.float32)
    Y = rng.standard_normal((8, 300)).astype(np.float32)
    a = orc.pairwise(X, Y, "sqeuclidean", kc=256)
    b = orc.pairwise(X, Y, "sqeuclidean", kc=64)
    exact = ((X.astype(np.float64)[:, None] - Y.astype(np.float64)[None]) ** 2).sum(-1)
    np.testing.assert_allclose(a, exact, rtol=1e-5)
    np.testing.assert_allclose(b, exact, rtol=1e-5)
    assert not np.array_equal(a, b)


def test_oracle_reference_tie_order(orc):
    """The reference's running top-k keeps the LAST of equal distances at the
    k boundary (<= replacement, nearest_neighbors_utils.hpp:206); the oracle's
    knn() breaks ties to the lower index.  Both orders are reproduced."""
    keys = np.array([5.0, 1.0, 3.0, 1.0, 3.0, 2.0])
    ref = orc.knn_reference_ties(keys, 3)
    assert list(ref) == [3, 1, 5]  # equal keys stay in buffer order
    keys2 = np.array([1.0, 2.0, 2.0, 2.0])
    assert list(orc.knn_reference_ties(keys2, 2)) == [0, 3]


def test_oracle_radius_hand_problem(orc):
    """The radius-5 neighbours of the reference's hand problem (sorted
    results): euclidean and squared euclidean."""
    z = golden("nn_small.npz")
    r = float(z["radius"][0])
    for metric, pre in (("euclidean", "rad_euc"), ("sqeuclidean", "rad_sq")):
        got = orc.radius(z["X_train"], z["X_test"], r, metric, sort=True)
        o = 0
        for q, c in enumerate(z[pre + "_cnt"]):
            np.testing.assert_array_equal(got[q][0], z[pre + "_ind"][o:o + c])
            np.testing.assert_allclose(got[q][1], z[pre + "_dist"][o:o + c],
                                       rtol=40 * np.finfo(float).eps)
            o += c


@pytest.mark.parametrize("weights", ["uniform", "distance"])
@pytest.mark.parametrize("group", ["euc", "sq"])
def test_oracle_radius_predict_hand_problem(orc, weights, group):
    """Radius-mode predict of the hand problem with the "radius" option 21
    (the reference's get_proba_radius / get_labels_radius /
    get_targets_radius)."""
    z, g = golden("nn_small.npz"), golden("nn_radius_predict.npz")
    r = float(g["hand_radius"][0])
    metric = {"euc": "euclidean", "sq": "sqeuclidean"}[group]
    X, Q, y, t = z["X_train"], z["X_test"], z["y_class"], z["y_reg"]
    pr, warn = orc.radius_predict_proba(X, y, Q, r, metric, weights=weights)
    want = g[f"hand_proba_{weights}_{group}"].reshape(3, 3).T  # column-major n_q x n_classes
    np.testing.assert_allclose(pr, want, rtol=100 * np.finfo(float).eps, atol=1e-15)
    assert not warn
    lab = orc.radius_predict(X, y, Q, r, metric, weights=weights)
    np.testing.assert_array_equal(lab, g[f"hand_labels_{weights}_{group}"].astype(np.int32))
    tg, _ = orc.radius_predict_reg(X, t, Q, r, metric, weights=weights)
    np.testing.assert_allclose(tg, g[f"hand_targets_{weights}_{group}"],
                               rtol=100 * np.finfo(float).eps)


def test_oracle_radius_predict_outliers(orc):
    """The reference's OutlierTesting: radius 4, distance weights; query 2
    has no neighbour.  "most frequent", then "manual" with label -999 (not a
    training label: zero probabilities and a warning) and target -123, then
    "manual" with label 1 and target NaN."""
    g = golden("nn_radius_predict.npz")
    X, Q, y, t = g["out_X_train"], g["out_X_test"], g["out_y_class"], g["out_y_reg"]
    tol = 10 * np.finfo(float).eps
    cases = (("most frequent", 0, 0.0, False, False),
             ("manual", -999, -123.0, True, True),
             ("manual", 1, np.nan, False, True))
    for i, (oh, lab_o, tgt_o, proba_warn, reg_warn) in enumerate(cases):
        pr, w = orc.radius_predict_proba(X, y, Q, 4.0, weights="distance", outlier=oh,
                                         outlier_label=lab_o)
        np.testing.assert_allclose(pr, g[f"out_proba_{i}"].reshape(3, 3).T, rtol=tol, atol=tol)
        assert w == proba_warn
        lab = orc.radius_predict(X, y, Q, 4.0, weights="distance", outlier=oh,
                                 outlier_label=lab_o)
        np.testing.assert_array_equal(lab, g[f"out_labels_{i}"].astype(np.int32))
        tg, w = orc.radius_predict_reg(X, t, Q, 4.0, weights="distance", outlier=oh,
                                       outlier_target=tgt_o)
        np.testing.assert_allclose(tg, g[f"out_targets_{i}"], rtol=tol, equal_nan=True)
        assert w == reg_warn
    with pytest.raises(LookupError):
        orc.radius_predict_proba(X, y, Q, 4.0, weights="distance")


def test_oracle_radius_predict_zero_rows(orc):
    """AccuracyTestingZeroData_radius: every distance is 0, so every weight
    of weights="distance" is 1."""
    g = golden("nn_radius_predict.npz")
    X, Q = np.zeros((4, 3)), np.zeros((3, 3))
    pr, _ = orc.radius_predict_proba(X, g["zero_y_class"], Q, 0.5, weights="distance")
    np.testing.assert_allclose(pr, g["zero_proba"].reshape(3, 3).T, rtol=1e-15)
    lab = orc.radius_predict(X, g["zero_y_class"], Q, 0.5, weights="distance")
    np.testing.assert_array_equal(lab, g["zero_labels"])
    tg, _ = orc.radius_predict_reg(X, g["zero_y_reg"], Q, 0.5, weights="distance")
    np.testing.assert_allclose(tg, np.full(3, g["zero_target"][0]), rtol=100 * np.finfo(float).eps)


def ann_case(z, i):
    """One IVF-flat functionality case of the reference: options, the
    training rows and queries as n x d arrays, and the expected neighbours
    as n_queries x k arrays (indices None where the reference checks only
    their validity)."""
    nl, npb, k, d, n, nq, ldx, ldq, it, row, frac, seed = z[f"c{i}_meta"]
    nl, npb, k, d, n, nq, ldx, ldq, it, row, seed = map(int, (nl, npb, k, d, n, nq, ldx, ldq, it,
                                                              row, seed))

    def mat(flat, rows, ld):
        flat = np.asarray(flat)
        if row:
            return flat.reshape(-1, ld)[:rows, :d].copy()
        return flat[:ld * d].reshape(d, ld).T[:rows, :].copy()

    X, Q = mat(z[f"c{i}_X_train"], n, ldx), mat(z[f"c{i}_X_test"], nq, ldq)
    shape = (nq, k) if row else (k, nq)
    wd = z[f"c{i}_kdist"].reshape(shape)
    wi = z[f"c{i}_kind"].reshape(shape) if f"c{i}_kind" in z.files else None
    if not row:
        wd = wd.T
        wi = None if wi is None else wi.T
    opts = dict(n_list=nl, n_probe=npb, k=k, kmeans_iter=it, row=bool(row),
                train_fraction=float(frac), seed=seed)
    return opts, X, Q, wi, wd


def test_oracle_ivf_functionality_cases(orc):
    """The reference's IVF-flat functionality cases: their expected
    neighbours are the exact ones, which the oracle's search reproduces with
    every list probed."""
    z = golden("ann_functionality.npz")
    for i in range(len(z["names"])):
        o, X, Q, wi, wd = ann_case(z, i)
        C = X.mean(0, keepdims=True)
        ind, dist, _ = orc.ivf_kneighbors(C, X, Q, o["k"], 1)
        tol = 3000 * np.finfo(float).eps
        np.testing.assert_allclose(dist, wd, rtol=tol, atol=tol, err_msg=str(z["names"][i]))
        if wi is not None:
            np.testing.assert_array_equal(ind, wi, err_msg=str(z["names"][i]))


# ----------------------------------------------------- spherical k-means --
# The reference's spherical tests (kmeans_public.cpp:722-1200,
# kmeans_test.py:313-337) assert properties rather than values; the oracle
# must satisfy each of them on the same data.
SPH_TOL = {np.float32: 1e-6, np.float64: 1e-12}


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_spherical_properties(orc, dtype):
    z = golden("kmeans_spherical.npz")
    A = z["A"].astype(dtype)
    tol = SPH_TOL[dtype]
    for C0 in (A[orc.kmeanspp_cosine(A, 3, 42)], z["C"].astype(dtype)):
        C, lab, nit, inertia = orc.kmeans_sph_lloyd(A, C0, 300, 1e-4)
        np.testing.assert_allclose((C.astype(np.float64) ** 2).sum(1), 1.0, atol=tol)
        # invariance to scaling the data: identical results (power-of-two scale)
        C2, lab2, nit2, inertia2 = orc.kmeans_sph_lloyd(2 * A, C0, 300, 1e-4)
        np.testing.assert_array_equal(C, C2)
        np.testing.assert_array_equal(lab, lab2)
        assert nit == nit2 and inertia == inertia2
        # the returned labels are the assignment to the returned centres
        np.testing.assert_array_equal(orc.kmeans_assign_sph(A, C)[0], lab)
        assert inertia == orc.kmeans_inertia_sph(A, lab, C)
        # predicting 2 x the centres gives each centre (kmeans_public.cpp:873-912)
        np.testing.assert_array_equal(orc.kmeans_assign_sph(2 * C, C)[0], np.arange(3))
    # k-means++ on the cosine distance chooses the same rows for 2 A
    np.testing.assert_array_equal(orc.kmeanspp_cosine(A, 3, 42), orc.kmeanspp_cosine(2 * A, 3, 42))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_spherical_normalise_on_off(orc, dtype):
    """Normalised data: "normalize data" yes and no give the same labels and
    centres within the reference's tolerance (kmeans_public.cpp:980-1106)."""
    z = golden("kmeans_spherical.npz")
    A = z["A"].astype(dtype)
    nrm = np.sqrt((A * A).sum(1, dtype=dtype))
    An = (A * (1 / nrm)[:, None]).astype(dtype)
    tol = SPH_TOL[dtype]
    C0 = An[orc.kmeanspp_cosine(An, 3, 42)]
    Con, lon, _, _ = orc.kmeans_sph_lloyd(An, C0, 300, 1e-4, normalise=True)
    Coff, loff, _, _ = orc.kmeans_sph_lloyd(An, C0, 300, 1e-4, normalise=False)
    np.testing.assert_array_equal(lon, loff)
    np.testing.assert_allclose(Con, Coff, atol=tol)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_spherical_python_case(orc, dtype):
    """kmeans_test.py:313-337: 6 x 3, two clusters, data used as given."""
    a = golden("kmeans_spherical.npz")["py_a"].astype(dtype)
    C0 = a[orc.kmeanspp_cosine(a, 2, 42, normalise=False)]
    C, lab, nit, _ = orc.kmeans_sph_lloyd(a, C0, 300, 1e-4, normalise=False)
    np.testing.assert_allclose(np.linalg.norm(C.astype(np.float64), axis=1), 1.0,
                               atol=SPH_TOL[dtype])
    assert set(lab) <= {0, 1}


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_ivf_spherical_cases(orc, dtype):
    """The reference's inner-product and cosine IVF-flat functionality cases
    (ann_tests.hpp): spherical k-means coarse quantiser from the seeded
    random rows, lists by -x.c, the probed lists' k best rows.  The outlier
    cases' expectations depend on the trained lists (the unprobed list holds
    the rows with the largest inner products)."""
    z = golden("ann_functionality_spherical.npz")
    for i, name in enumerate(z["names"]):
        metric = str(z["metrics"][i])
        o, X, Q, wi, wd = ann_case(z, i)
        X, Q = X.astype(dtype), Q.astype(dtype)
        C = orc.ivf_train_spherical(X, o["n_list"], o["seed"], o["kmeans_iter"], metric)
        if metric == "cosine":
            X, Q = orc.normalise_rows(X), orc.normalise_rows(Q)
        ind, dist, _ = orc.ivf_kneighbors(C.astype(np.float64), X, Q, o["k"], o["n_probe"],
                                          metric)
        tol = 3000 * np.finfo(dtype).eps
        np.testing.assert_allclose(dist, wd, rtol=tol, atol=tol, err_msg=str(name))
        if wi is not None:
            np.testing.assert_array_equal(ind, wi, err_msg=str(name))
