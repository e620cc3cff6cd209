"""Radius-mode predict (da_nn_classifier_predict_proba_? / _predict_? and
da_nn_regressor_predict_? with radius_search_mode) on the GPU: the
reference's known answers (hand problem with the "radius" option 21,
OutlierTesting, AccuracyTestingZeroData_radius; statuses included) and the
oracle restatement on seeded data for several metrics, weights and outlier
handling modes, both precisions and storage orders."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

HAND_METRICS = [("euc", m) for m in ("euclidean", "l2", "minkowski", "euclidean_gemm")] + \
               [("sq", m) for m in ("sqeuclidean", "sqeuclidean_gemm")]


@pytest.mark.parametrize("group,metric", HAND_METRICS)
@pytest.mark.parametrize("weights", ["uniform", "distance"])
@pytest.mark.parametrize("prec,order", [("d", 0), ("s", 1)])
def test_radius_predict_hand_problem(gpu, ab, group, metric, weights, prec, order):
    z, g = golden("nn_small.npz"), golden("nn_radius_predict.npz")
    dt = np.float64 if prec == "d" else np.float32
    tol = 100 * np.finfo(dt).eps
    nn = ab.KNN(prec, order=order, metric=metric, weights=weights,
                radius=float(g["hand_radius"][0]))
    nn.fit(z["X_train"], y=z["y_class"], targets=z["y_reg"])
    pr = nn.predict_proba(z["X_test"], mode=ab.RADIUS_SEARCH)
    assert nn.last_status == 0
    np.testing.assert_allclose(pr, g[f"hand_proba_{weights}_{group}"].reshape(3, 3).T,
                               rtol=tol, atol=tol)
    lab = nn.predict(z["X_test"], mode=ab.RADIUS_SEARCH)
    np.testing.assert_array_equal(lab, g[f"hand_labels_{weights}_{group}"].astype(np.int32))
    tg = nn.predict_reg(z["X_test"], mode=ab.RADIUS_SEARCH)
    np.testing.assert_allclose(tg, g[f"hand_targets_{weights}_{group}"], rtol=tol)
    nn.close()


@pytest.mark.parametrize("prec", ["d", "s"])
def test_radius_predict_outliers(gpu, ab, prec):
    """OutlierTesting: "most frequent"; "manual" with a label absent from the
    training labels (status 700 from all three calls, zero probabilities);
    "manual" with label 1 and target NaN (700 from the regressor only)."""
    g = golden("nn_radius_predict.npz")
    dt = np.float64 if prec == "d" else np.float32
    tol = 10 * np.finfo(dt).eps
    nn = ab.KNN(prec, weights="distance", radius=4.0, outlier_handling="most frequent")
    nn.fit(g["out_X_train"], y=g["out_y_class"], targets=g["out_y_reg"])
    Q = g["out_X_test"]
    cases = ((None, None, 0, 0), (-999, -123.0, 700, 700), (1, float("nan"), 0, 700))
    for i, (lab_o, tgt_o, st_cls, st_reg) in enumerate(cases):
        if lab_o is not None:
            assert nn.set("outlier handling", "manual") == 0
            assert nn.set("outlier label", lab_o) == 0
            assert nn.set("outlier target", tgt_o) == 0
        tg = nn.predict_reg(Q, mode=ab.RADIUS_SEARCH)
        assert nn.last_status == st_reg
        np.testing.assert_allclose(tg, g[f"out_targets_{i}"], rtol=tol, equal_nan=True)
        pr = nn.predict_proba(Q, mode=ab.RADIUS_SEARCH)
        assert nn.last_status == st_cls
        np.testing.assert_allclose(pr, g[f"out_proba_{i}"].reshape(3, 3).T, rtol=tol, atol=tol)
        lab = nn.predict(Q, mode=ab.RADIUS_SEARCH)
        assert nn.last_status == st_cls
        np.testing.assert_array_equal(lab, g[f"out_labels_{i}"].astype(np.int32))
    # outlier handling "none": a query without neighbours fails (status 14)
    assert nn.set("outlier handling", "none") == 0
    for call in (nn.predict_proba, nn.predict, nn.predict_reg):
        with pytest.raises(ab.DAError) as e:
            call(Q, mode=ab.RADIUS_SEARCH)
        assert e.value.status == 14
    nn.close()


def test_radius_predict_zero_rows(gpu, ab):
    g = golden("nn_radius_predict.npz")
    nn = ab.KNN("d", weights="distance", radius=0.5)
    nn.fit(np.zeros((4, 3)), y=g["zero_y_class"], targets=g["zero_y_reg"])
    Q = np.zeros((3, 3))
    np.testing.assert_allclose(nn.predict_reg(Q, mode=ab.RADIUS_SEARCH),
                               np.full(3, g["zero_target"][0]), rtol=100 * np.finfo(float).eps)
    np.testing.assert_allclose(nn.predict_proba(Q, mode=ab.RADIUS_SEARCH),
                               g["zero_proba"].reshape(3, 3).T, rtol=1e-15)
    np.testing.assert_array_equal(nn.predict(Q, mode=ab.RADIUS_SEARCH), g["zero_labels"])
    nn.close()


def data(rng, n, nq, d, dt):
    means = rng.uniform(-3, 3, (6, d))
    X = (means[rng.integers(0, 6, n)] + rng.standard_normal((n, d))).astype(dt)
    Q = (means[rng.integers(0, 6, nq)] + rng.standard_normal((nq, d))).astype(dt)
    Q[0] = X[7]          # a query on a training row (distance 0: weight 1)
    Q[1] = 40.0          # far from every row: an outlier of the radius search
    Q[2] = -40.0
    y = np.array([3, 5, 7, 11], dtype=np.int32)[rng.integers(0, 4, n)]
    t = rng.standard_normal(n).astype(dt)
    return X, Q, y, t


@pytest.mark.parametrize("metric,p,radius", [("euclidean", 2.0, 2.2), ("sqeuclidean", 2.0, 4.0),
                                              ("manhattan", 2.0, 4.5), ("cosine", 2.0, 0.08),
                                              ("minkowski", 3.0, 1.9),
                                              ("inner product", 2.0, 0.0)])
@pytest.mark.parametrize("weights", ["uniform", "distance"])
@pytest.mark.parametrize("outlier", ["manual", "most frequent"])
@pytest.mark.parametrize("prec,order", [("s", 1), ("d", 0)])
def test_radius_predict_matches_oracle(gpu, ab, orc, metric, p, radius, weights, outlier, prec,
                                       order):
    if metric == "inner product" and weights == "distance":
        pytest.skip("inner product takes uniform weights only (status 13, tested on CPU)")
    dt = np.float32 if prec == "s" else np.float64
    rng = np.random.default_rng(len(metric) + int(10 * p))
    X, Q, y, t = data(rng, 3000, 64, 7, dt)
    # cosine: the far queries point like some rows; make them outliers by sign
    if metric == "cosine":
        Q[1] = -X[:].sum(0) / 3000 * 50
        Q[2] = Q[1]
    if metric == "inner product":
        # positive rows: a mixed-sign query has the rows of dot <= 0 as
        # neighbours, a positive query none (an outlier)
        X = (np.abs(X) + 1).astype(dt)
        Q = rng.standard_normal(Q.shape).astype(dt)
        Q[1], Q[2] = 1, 2
    lab_o, tgt_o = 5, -2.5
    nn = ab.KNN(prec, order=order, metric=metric, minkowski_parameter=p, weights=weights,
                radius=radius, outlier_handling=outlier, outlier_label=lab_o,
                outlier_target=tgt_o)
    nn.fit(X, y=y, targets=t)
    # an earlier radius search's results stay as they were (the public
    # radius search refuses the inner product, status 13, as the reference)
    if metric == "inner product":
        with pytest.raises(ab.DAError) as e:
            nn.radius_neighbors(Q[:8], radius, False, False)
        assert e.value.status == 13
    else:
        cnt0, _, ind0, _ = nn.radius_neighbors(Q[:8], radius, False, False)
    ref = orc.radius(X, Q, radius, metric, p)
    n_out = sum(len(r[0]) == 0 for r in ref)
    assert n_out >= 1 and sum(len(r[0]) for r in ref) > 64
    # distances of minkowski p = 3 may differ by an ulp of pow(): looser there
    tol = (64 if metric == "minkowski" else 4) * np.finfo(dt).eps
    pr = nn.predict_proba(Q, mode=ab.RADIUS_SEARCH)
    rpr, rwarn = orc.radius_predict_proba(X, y, Q, radius, metric, p, weights, outlier, lab_o)
    np.testing.assert_allclose(pr, rpr, rtol=tol, atol=tol)
    assert nn.last_status == (700 if rwarn else 0)
    lab = nn.predict(Q, mode=ab.RADIUS_SEARCH)
    np.testing.assert_array_equal(lab, orc.radius_predict(X, y, Q, radius, metric, p, weights,
                                                          outlier, lab_o))
    tg = nn.predict_reg(Q, mode=ab.RADIUS_SEARCH)
    rtg, rw = orc.radius_predict_reg(X, t, Q, radius, metric, p, weights, outlier, tgt_o)
    np.testing.assert_allclose(tg, rtg, rtol=tol, atol=tol)
    assert nn.last_status == (700 if rw else 0)
    if metric != "inner product":
        cnt1 = nn.result_int(ab.RNN_COUNT, 9)
        np.testing.assert_array_equal(cnt0, cnt1)
        ind1 = nn.result_int(ab.RNN_INDICES, max(int(cnt1[-1]), 1))[:int(cnt1[-1])]
        np.testing.assert_array_equal(ind0, ind1)
    nn.close()
