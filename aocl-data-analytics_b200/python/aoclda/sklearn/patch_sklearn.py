"""skpatch / undo_skpatch (python_package/aoclda/sklearn/patch_sklearn.py:
150-215) for the estimators of the distance / neighbour / k-means path."""
import sklearn.cluster as _cluster
import sklearn.metrics as _metrics
import sklearn.metrics.pairwise as _pairwise
import sklearn.neighbors as _neighbors

from ._kmeans import KMeans
from ._metrics import pairwise_distances
from ._neighbors import (KNeighborsClassifier, KNeighborsRegressor, NearestNeighbors,
                         RadiusNeighborsClassifier, RadiusNeighborsRegressor)

SYMBOLS = {
    name: {"packs": packs, "sk_sym": getattr(packs[0], name), "da_sym": sym}
    for name, packs, sym in (
        ("NearestNeighbors", (_neighbors,), NearestNeighbors),
        ("KNeighborsClassifier", (_neighbors,), KNeighborsClassifier),
        ("KNeighborsRegressor", (_neighbors,), KNeighborsRegressor),
        ("RadiusNeighborsClassifier", (_neighbors,), RadiusNeighborsClassifier),
        ("RadiusNeighborsRegressor", (_neighbors,), RadiusNeighborsRegressor),
        ("KMeans", (_cluster,), KMeans),
        ("pairwise_distances", (_pairwise, _metrics), pairwise_distances))
}


def _names(args):
    if not args:
        return list(SYMBOLS)
    if isinstance(args[0], str):
        return [args[0]]
    if isinstance(args[0], (list, tuple)):
        return list(args[0])
    raise TypeError("Unrecognized argument")


def _swap(args, key, print_patched, verb):
    done = []
    for name in _names(args):
        if name not in SYMBOLS:
            print(f"The package {name} was not found.")
            continue
        for pack in SYMBOLS[name]["packs"]:
            setattr(pack, name, SYMBOLS[name][key])
        done.append(name)
    if done and print_patched:
        print(f"B200 extension for scikit-learn {verb} for the following packages:")
        print(", ".join(done))
    return done


def skpatch(*args, print_patched=True):
    """Replace the named scikit-learn symbols (all when none are named) by the
    B200 ones."""
    return _swap(args, "da_sym", print_patched, "enabled")


def undo_skpatch(*args, print_patched=True):
    """Put the named scikit-learn symbols back."""
    return _swap(args, "sk_sym", print_patched, "disabled")
