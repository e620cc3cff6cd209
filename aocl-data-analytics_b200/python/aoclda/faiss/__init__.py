"""faiss-compatible IndexFlatL2, IndexIVFFlat and Kmeans over the B200
handles (python_package/aoclda/faiss/*.py); patch_faiss() installs them into
an importable ``faiss`` module, undo_patch_faiss() restores it."""
from ._index import IndexFlatL2, IndexIVFFlat, METRIC_INNER_PRODUCT, METRIC_L2  # noqa: F401
from ._kmeans import Kmeans  # noqa: F401
from .patch_faiss import patch_faiss, undo_patch_faiss  # noqa: F401
