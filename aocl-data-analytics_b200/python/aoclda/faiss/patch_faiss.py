"""patch_faiss / undo_patch_faiss (python_package/aoclda/faiss/
patch_faiss.py): the faiss symbols IndexFlatL2, IndexIVFFlat and Kmeans
replaced by the B200 classes in an importable faiss module."""
import importlib

from ._index import IndexFlatL2, IndexIVFFlat
from ._kmeans import Kmeans

_SYMBOLS = {"IndexFlatL2": IndexFlatL2, "IndexIVFFlat": IndexIVFFlat, "Kmeans": Kmeans}
_saved = {}


def _faiss():
    try:
        return importlib.import_module("faiss")
    except ImportError as e:
        raise ImportError("faiss is not installed; use aoclda.faiss.IndexFlatL2 / IndexIVFFlat "
                          "/ Kmeans directly") from e


def patch_faiss(*names):
    mod = _faiss()
    for n in names or tuple(_SYMBOLS):
        _saved.setdefault(n, getattr(mod, n, None))
        setattr(mod, n, _SYMBOLS[n])


def undo_patch_faiss(*names):
    mod = _faiss()
    for n in names or tuple(_SYMBOLS):
        if n in _saved:
            setattr(mod, n, _saved.pop(n))
