"""Generate the golden fixtures of tests/golden/ from the AOCL-DA test assets.

Run where the AOCL-DA source tree is available, with AOCLDA_REF naming its
root directory:

    AOCLDA_REF=<path to the AOCL-DA source tree> python tests/golden/make_golden.py

It converts, without retyping any value:
  * the "large data" kNN known-answer sets of the reference's nearest-neighbour
    tests (tests/data/nn_data/*_2092x2071x5*, *_2125x2068x20*; loaded by
    tests/unit_tests/nearest_neighbors/nearest_neighbors_tests.hpp:588-760,
    tolerance 500*eps), into nn_<samples>x<queries>x<features>.npz;
  * the 6x3 / 3x3 hand-computed kNN problem of nearest_neighbors_tests.hpp
    (X_train/X_test at :450-464, expected indices and distances at :97-144,
    radius-5 neighbours at :147-160),
    parsed from the C++ initialiser lists, into nn_small.npz;
  * the radius-mode predict expectations: those of the same hand problem with
    the "radius" option 21 (get_proba_radius / get_labels_radius /
    get_targets_radius, nearest_neighbors_tests.hpp:317-424), and the
    OutlierTesting and AccuracyTestingZeroData_radius cases of
    nearest_neighbors_public.cpp (:337-432, :462-608), into
    nn_radius_predict.npz;
  * the squared-euclidean functionality cases of the IVF-flat tests
    (tests/unit_tests/approximate_neighbors/ann_tests.hpp:395-1260: data,
    n_list / n_probe / k, storage order, leading dimensions, expected
    neighbour indices and squared distances), into ann_functionality.npz,
    and its inner-product and cosine cases (with their metric) into
    ann_functionality_spherical.npz;
  * the Lloyd "larger data matrix" k-means case of
    tests/unit_tests/kmeans/kmeans_test_data.hpp:444-526 into kmeans_lloyd80.npz;
  * the data of the spherical k-means tests into kmeans_spherical.npz.
The d=130 set cannot be converted: its inputs are absent from the tree.
"""
import os
import re

import numpy as np

REF = os.environ.get("AOCLDA_REF")
if not REF:
    raise SystemExit("set AOCLDA_REF to the root of the AOCL-DA source tree")
OUT = os.path.dirname(os.path.abspath(__file__))
NN = os.path.join(REF, "tests", "data", "nn_data")
UT = os.path.join(REF, "tests", "unit_tests")


def csv(name, dtype=np.float64):
    a = np.loadtxt(os.path.join(NN, name), delimiter=",", dtype=np.float64, ndmin=2)
    return a.astype(dtype)


def nn_large(samples, queries, feats):
    tag = f"{samples}x{queries}x{feats}"
    out = dict(
        X_train=csv(f"X_train_{samples}x{feats}.csv"),
        X_test=csv(f"X_test_{queries}x{feats}.csv"),
        y_train=csv(f"y_train_{samples}x{feats}.csv").ravel(),
        k_ind=csv(f"k_ind_{tag}_5.csv").astype(np.int32),
        k_dist=csv(f"k_dist_{tag}_5.csv"),
    )
    for w in ("uniform", "distance"):
        out[f"proba_{w}"] = csv(f"proba_knn_{queries}x{feats}_{w}.csv")
        out[f"class_{w}"] = csv(f"predict_class_knn_{queries}x{feats}_{w}.csv").ravel().astype(np.int32)
        out[f"reg_{w}"] = csv(f"predict_reg_knn_{queries}x{feats}_{w}.csv").ravel()
    np.savez_compressed(os.path.join(OUT, f"nn_{tag}.npz"), **out)


def init_lists(text, name):
    """All brace initialiser lists `name{...}` in C++ source text, as float arrays."""
    res = []
    for m in re.finditer(r"\b" + re.escape(name) + r"\s*\{([^}]*)\}", text):
        body = m.group(1).replace("\n", " ")
        vals = [v.strip() for v in body.split(",") if v.strip()]
        res.append(np.array([float(v) for v in vals]))
    return res


def nn_small():
    text = open(os.path.join(UT, "nearest_neighbors", "nearest_neighbors_tests.hpp")).read()
    X_train = init_lists(text, "X_train")[0]
    X_test = init_lists(text, "X_test")[0]
    y_class = init_lists(text, "y_train_class")[0]
    y_reg = init_lists(text, "y_train_regression")[0]
    kinds = init_lists(text, "kind")
    kdists = init_lists(text, "kdist")
    # the radius-5 expectations of get_expected_radius_ind_radius_dist
    # (:147-160; sorted results): euclidean, then squared euclidean
    blk = text[text.index("void get_expected_radius_ind_radius_dist"):]
    blk = blk[:blk.index("template <typename T>")]

    def ragged(after):
        lists = []
        pat = re.escape(after) + r"\s*=\s*std::vector<std::vector<[^>]*>>\(\{(.*?)\}\);"
        for m in re.finditer(pat, blk, re.S):
            rows = re.findall(r"\{([^{}]*)\}", m.group(1))
            lists.append([[float(v) for v in r.split(",") if v.strip()] for r in rows])
        return lists

    rind, rdist = ragged("param.expected_radius_ind"), ragged("param.expected_radius_dist")

    def flat(rows):
        return np.array([v for r in rows for v in r])

    def cnts(rows):
        return np.array([len(r) for r in rows], dtype=np.int32)

    radius = dict(radius=np.array([5.0]),
                  rad_euc_ind=flat(rind[0]).astype(np.int32), rad_euc_cnt=cnts(rind[0]),
                  rad_euc_dist=flat(rdist[0]),
                  rad_sq_ind=flat(rind[1]).astype(np.int32), rad_sq_cnt=cnts(rind[1]),
                  rad_sq_dist=flat(rdist[1]))
    # the first two lists are the k=3 and k=4 euclidean expectations (:97-144)
    np.savez_compressed(
        os.path.join(OUT, "nn_small.npz"), **radius,
        X_train=X_train.reshape(3, 6).T.copy(),  # column-major 6 x 3
        X_test=X_test.reshape(3, 3).T.copy(),    # column-major 3 x 3
        y_class=y_class.astype(np.int32), y_reg=y_reg,
        kind3=kinds[0].astype(np.int32), kdist3=kdists[0],
        kind4=kinds[1].astype(np.int32), kdist4=kdists[1])


def _values(body):
    out = []
    for v in body.replace("\n", " ").split(","):
        v = v.strip()
        if v:
            out.append(np.nan if "quiet_NaN" in v else float(v))
    return np.array(out)


def assigned_lists(text, name):
    """Initialisers of `name` in declarations and assignments: `name{...}`,
    `name = {...}`, `name = std::vector<T>({...})`, in source order."""
    pat = (r"\b" + re.escape(name) +
           r"\s*(?:=\s*)?(?:std::vector<[^>]*>\s*\(\s*)?\{([^{}]*)\}")
    return [_values(m.group(1)) for m in re.finditer(pat, text)]


def nn_radius_predict():
    hpp = open(os.path.join(UT, "nearest_neighbors", "nearest_neighbors_tests.hpp")).read()
    cpp = open(os.path.join(UT, "nearest_neighbors", "nearest_neighbors_public.cpp")).read()
    out = {}
    # hand problem, "radius" option 21: uniform / distance x euclidean / squared
    rc = re.search(r"T radius_constructor = ([0-9.]+);", hpp[hpp.index("get_targets_radius"):])
    out["hand_radius"] = np.array([float(rc.group(1))])
    for fn, name, key in (("get_proba_radius", "proba", "proba"),
                          ("get_labels_radius", "expected_labels_radius", "labels"),
                          ("get_targets_radius", "expected_targets_radius", "targets")):
        blk = hpp[hpp.index("void " + fn):]
        blk = blk[:blk.index("template <typename T>")]
        lists = init_lists(blk, name)
        assert len(lists) == 4, (fn, len(lists))
        for (w, m), v in zip((("uniform", "euc"), ("uniform", "sq"), ("distance", "euc"),
                              ("distance", "sq")), lists):
            out[f"hand_{key}_{w}_{m}"] = v
    # OutlierTesting: radius 4, weights distance; most frequent, manual (-999, -123),
    # manual (1, NaN)
    blk = cpp[cpp.index("TYPED_TEST(NearestNeighborsTest, OutlierTesting)"):]
    blk = blk[:blk.index("TYPED_TEST(", 10)]
    one = lambda n: init_lists(blk, n)[0]
    out.update(out_X_train=one("X_train").reshape(3, 6).T.copy(),  # column-major 6 x 3
               out_X_test=one("X_test").reshape(3, 3).T.copy(),
               out_y_class=one("y_train_class").astype(np.int32),
               out_y_reg=one("y_train_regression"))
    for name, key in (("expected_targets", "targets"), ("expected_proba", "proba"),
                      ("expected_labels", "labels")):
        lists = assigned_lists(blk, name)
        assert len(lists) == 3, (name, len(lists))
        for i, v in enumerate(lists):
            out[f"out_{key}_{i}"] = v
    # AccuracyTestingZeroData_radius: all-zero rows, radius 0.5, weights distance
    blk = cpp[cpp.index("AccuracyTestingZeroData_radius"):]
    blk = blk[:blk.index("TYPED_TEST(")]
    out.update(zero_y_class=init_lists(blk, "y_train_class")[0].astype(np.int32),
               zero_y_reg=init_lists(blk, "y_train_regression")[0],
               zero_proba=assigned_lists(blk, "expected_proba")[0],
               zero_labels=assigned_lists(blk, "expected_labels")[0].astype(np.int32),
               zero_target=np.array([float(re.search(
                   r"expected_targets\(n_queries, ([0-9.]+)\)", blk).group(1))]))
    np.savez_compressed(os.path.join(OUT, "nn_radius_predict.npz"), **out)


def ann_functionality(metrics=("sqeuclidean",), fname="ann_functionality.npz"):
    text = open(os.path.join(UT, "approximate_neighbors", "ann_tests.hpp")).read()
    out, names, mets = {}, [], []
    for m in re.finditer(r"template <typename T> void (\w+)\(std::vector<ANNParamType<T>> &params\) \{",
                         text):
        body = text[m.end():]
        if "params.push_back(test);" not in body:
            continue
        body = body[:body.index("params.push_back(test);")]
        ctor = re.search(r'ANNParamType<T> test\((\d+), (\d+), (\d+), "([^"]+)", "([^"]+)", "([^"]+)"\)',
                         body)
        if ctor is None or ctor.group(4) not in metrics:
            continue
        nlist, nprobe, k = (int(ctor.group(i)) for i in (1, 2, 3))
        vals = {"n_features": None, "n_samples": None, "n_queries": None, "ldx_train": None,
                "ldx_test": None, "kmeans_iter": 10, "train_fraction": 1.0, "seed": 0}
        for a in re.finditer(r"test\.(\w+) = ([^;]+);", body):
            key, expr = a.group(1), a.group(2).strip()
            if key not in vals:
                continue
            ref = re.fullmatch(r"test\.(\w+)", expr)
            vals[key] = vals[ref.group(1)] if ref else float(expr)
        lists = {n: assigned_lists(body, n) for n in ("X_train", "X_test", "expected_kind",
                                                      "expected_kdist")}
        if not lists["X_train"] or not lists["X_test"] or not lists["expected_kdist"]:
            continue
        i = len(names)
        names.append(m.group(1))
        mets.append(ctor.group(4))
        row = ctor.group(6) == "row-major"
        out[f"c{i}_meta"] = np.array([nlist, nprobe, k, vals["n_features"], vals["n_samples"],
                                      vals["n_queries"], vals["ldx_train"], vals["ldx_test"],
                                      vals["kmeans_iter"], int(row), vals["train_fraction"],
                                      vals["seed"]], dtype=np.float64)
        out[f"c{i}_X_train"] = lists["X_train"][0]
        out[f"c{i}_X_test"] = lists["X_test"][0]
        out[f"c{i}_kdist"] = lists["expected_kdist"][0]
        if lists["expected_kind"]:
            out[f"c{i}_kind"] = lists["expected_kind"][0].astype(np.int32)
    out["names"] = np.array(names)
    if metrics != ("sqeuclidean",):
        out["metrics"] = np.array(mets)
    np.savez_compressed(os.path.join(OUT, fname), **out)


def kmeans_lloyd80():
    text = open(os.path.join(UT, "kmeans", "kmeans_test_data.hpp")).read()
    start = text.index("GetLargeBaseData")
    end = text.index("GetPseudoRandomBaseData")
    block = text[start:end]
    one = lambda n: init_lists(block, n)[0]
    np.savez_compressed(
        os.path.join(OUT, "kmeans_lloyd80.npz"),
        A=one("A").reshape(2, 80).T.copy(),      # column-major 80 x 2 (lda = 80)
        C=one("C").reshape(2, 16).T.copy(),      # column-major 16 x 2 (ldc = 16)
        expected_rinfo=one("expected_rinfo"),
        expected_centres=one("expected_centres").reshape(2, 16).T.copy(),
        expected_labels=one("expected_labels").astype(np.int32),
        Y=one("Y").reshape(1, 2), expected_Y_labels=one("expected_Y_labels").astype(np.int32),
        X=one("X").reshape(1, 2), expected_X_transform=one("expected_X_transform").reshape(1, 16),
        max_iter=np.array([30]), tol=np.array([1.0e-4]))


def kmeans_spherical():
    """The data of the reference's spherical k-means tests: the 20 x 3 set,
    the unnormalised supplied centres and the empty-cluster split case of
    tests/unit_tests/kmeans/kmeans_public.cpp:722-1200 (column-major
    initialisers), and the 6 x 3 array of
    python_interface/tests/kmeans_test.py:313-337.  The tests assert
    properties only (unit-length centres, invariance to scaling the data,
    predict / transform of scaled centres, normalise on = off for
    normalised data, split recovery), which the fixture's users repeat."""
    text = open(os.path.join(UT, "kmeans", "kmeans_public.cpp")).read()
    start = text.index("TYPED_TEST(KMeansTest, SphericalKMeans)")
    end = text.index("TYPED_TEST(", start + 10)
    block = text[start:end]
    a = assigned_lists(block, "A_col")[0]
    c = assigned_lists(block, "C")[0]
    ec_a = assigned_lists(block, "ec_A_col")[0]
    ec_c = assigned_lists(block, "ec_C_col")[0]
    py = open(os.path.join(REF, "python_interface", "tests", "kmeans_test.py")).read()
    ps = py.index("def test_kmeans_spherical")
    m = re.search(r"np\.array\(\[(.*?)\],\s*dtype", py[ps:], re.S)
    rows = re.findall(r"\[([^\[\]]+)\]", m.group(1))
    pa = np.array([[float(v) for v in r.split(",")] for r in rows])
    np.savez_compressed(
        os.path.join(OUT, "kmeans_spherical.npz"),
        A=a.reshape(3, 20).T.copy(),             # column-major 20 x 3
        C=c.reshape(3, 3).T.copy(),              # column-major 3 x 3 supplied centres
        ec_A=ec_a.reshape(2, 5).T.copy(),        # column-major 5 x 2
        ec_C=ec_c.reshape(2, 2).T.copy(),        # column-major 2 x 2
        py_a=pa)


if __name__ == "__main__":
    nn_large(2092, 2071, 5)
    nn_large(2125, 2068, 20)
    nn_small()
    nn_radius_predict()
    ann_functionality()
    ann_functionality(("inner product", "cosine"), "ann_functionality_spherical.npz")
    kmeans_lloyd80()
    kmeans_spherical()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
