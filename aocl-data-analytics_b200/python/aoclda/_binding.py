"""The ctypes binding of libaoclda_b200.so (aoclda_b200.py beside the
library), loaded once for the package, and the array conversion of the
reference's check_convert_data (python_package/aoclda/_internal_utils.py):
float32 stays single precision, everything else becomes double; a
Fortran-ordered array stays column-major, anything else is row-major."""
import importlib.util
import os
import tempfile

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def _load():
    spec = importlib.util.spec_from_file_location("aoclda_b200",
                                                  os.path.join(_PKG, "aoclda_b200.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.lib()  # raises when the shared library is not built
    return mod


ab = _load()


def convert(X, prec=None, order=None):
    """(array, precision 's' / 'd', storage order) for the C calls; `prec` /
    `order` force those of an already fitted handle."""
    X = np.asarray(X)
    if X.ndim != 2:
        raise ValueError(f"expected a 2-D array, got shape {X.shape}")
    if prec is None:
        prec = "s" if X.dtype == np.float32 else "d"
    dt = np.float32 if prec == "s" else np.float64
    if order is None:
        order = ab.COLUMN_MAJOR if (X.flags.f_contiguous and not X.flags.c_contiguous) \
            else ab.ROW_MAJOR
    X = np.asfortranarray(X, dtype=dt) if order == ab.COLUMN_MAJOR else \
        np.ascontiguousarray(X, dtype=dt)
    return X, prec, order


def dump_model(h):
    """The bytes of da_handle_save_model for handle object `h` (pickling)."""
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "model.bin")
        h.save_model(f)
        with open(f, "rb") as fh:
            return fh.read()


def load_model(cls, data, prec):
    """A new handle object of class `cls` from bytes written by dump_model."""
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "model.bin")
        with open(f, "wb") as fh:
            fh.write(data)
        return cls.load_model(f, prec)
