"""Generate the golden fixtures of tests/golden/ from the AOCL-DA test assets.

Run in a container where the AOCL-DA source tree is mounted (default
/root/reference, override with AOCLDA_REF):

    python tests/golden/make_golden.py

It converts, without retyping any value:
  * the "large data" kNN known-answer sets of the reference's nearest-neighbour
    tests (tests/data/nn_data/*_2092x2071x5*, *_2125x2068x20*; loaded by
    tests/unit_tests/nearest_neighbors/nearest_neighbors_tests.hpp:588-760,
    tolerance 500*eps), into nn_<samples>x<queries>x<features>.npz;
  * the 6x3 / 3x3 hand-computed kNN problem of nearest_neighbors_tests.hpp
    (X_train/X_test at :450-464, expected indices and distances at :97-144,
    radius-5 neighbours at :147-160),
    parsed from the C++ initialiser lists, into nn_small.npz;
  * the Lloyd "larger data matrix" k-means case of
    tests/unit_tests/kmeans/kmeans_test_data.hpp:444-526 into kmeans_lloyd80.npz.
The d=130 set cannot be converted: its inputs are absent from the tree.
"""
import os
import re

import numpy as np

REF = os.environ.get("AOCLDA_REF", "/root/reference")
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


if __name__ == "__main__":
    nn_large(2092, 2071, 5)
    nn_large(2125, 2068, 20)
    nn_small()
    kmeans_lloyd80()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
