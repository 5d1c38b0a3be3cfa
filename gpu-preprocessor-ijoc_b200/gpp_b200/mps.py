"""MPS input and reduced-LP export through the C ABI (gpp_mps_*, gpp_export_reduced)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .device import _raise
from .lpgen import HostLP


class MpsModel:
    """A parsed MPS model held by the library (gpp_mps_read / gpp_mps_read_string)."""

    def __init__(self, path: str | None = None, text: str | None = None):
        lib = capi.load()
        self.h = C.c_void_p()
        if (path is None) == (text is None):
            raise ValueError("give exactly one of path and text")
        if path is not None:
            _raise(lib.gpp_mps_read(path.encode(), C.byref(self.h)))
        else:
            _raise(lib.gpp_mps_read_string(text.encode(), C.byref(self.h)))
        rows, cols, nnz, obj = C.c_int32(), C.c_int32(), C.c_int64(), C.c_double()
        name = C.create_string_buffer(256)
        _raise(lib.gpp_mps_info(self.h, C.byref(rows), C.byref(cols), C.byref(nnz), C.byref(obj), name, 256))
        self.name = name.value.decode()
        self.rows, self.cols, self.nnz, self.obj_constant = rows.value, cols.value, nnz.value, obj.value
        m, n, k = self.rows, self.cols, self.nnz
        self.row_ptr, self.col_idx, self.csr_val = np.zeros(m + 1, np.int64), np.zeros(k, np.int32), np.zeros(k)
        self.col_ptr, self.row_idx, self.csc_val = np.zeros(n + 1, np.int64), np.zeros(k, np.int32), np.zeros(k)
        self.c, self.AL, self.AU, self.l, self.u = np.zeros(n), np.zeros(m), np.zeros(m), np.zeros(n), np.zeros(n)
        arrays = (self.row_ptr, self.col_idx, self.csr_val, self.col_ptr, self.row_idx, self.csc_val, self.c,
                  self.AL, self.AU, self.l, self.u)
        _raise(lib.gpp_mps_arrays(self.h, *(a.ctypes.data_as(C.c_void_p) for a in arrays)))

    def close(self):
        if self.h:
            capi.load().gpp_mps_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def host_lp(self) -> HostLP:
        """The model as the host LP type the rest of the package uses."""
        return HostLP(self.rows, self.cols, self.row_ptr.astype(np.int32), self.col_idx, self.csr_val, self.c,
                      self.AL, self.AU, self.l, self.u, self.obj_constant).ensure_transpose()

    def upload(self) -> capi.Lp:
        """gpp_mps_upload: device A and AT = A^T; release with free_lp."""
        lp = capi.Lp()
        _raise(capi.load().gpp_mps_upload(self.h, C.byref(lp)))
        return lp


def free_lp(lp: capi.Lp) -> None:
    capi.load().gpp_lp_free(C.byref(lp))


def export_reduced(summary: capi.Summary, out_dir: str, model_name: str = "") -> None:
    """gpp_export_reduced: the reduced LP in the reference's export format."""
    _raise(capi.load().gpp_export_reduced(C.byref(summary), out_dir.encode(), model_name.encode()))


def reduced_to_device(summary: capi.Summary) -> capi.Lp:
    """gpp_reduced_to_device: a solver-owned device copy of the reduced LP
    (A, its stable transpose, vectors); release with free_lp."""
    lp = capi.Lp()
    _raise(capi.load().gpp_reduced_to_device(C.byref(summary), C.byref(lp)))
    return lp


def reduced_to_host(summary: capi.Summary) -> dict:
    """gpp_reduced_to_host: the reduced LP as host arrays."""
    m, n, nnz = summary.reduced_rows, summary.reduced_cols, summary.reduced_nnz
    out = {"row_ptr": np.zeros(m + 1, np.int32), "col_idx": np.zeros(nnz, np.int32), "val": np.zeros(nnz),
           "c": np.zeros(n), "AL": np.zeros(m), "AU": np.zeros(m), "l": np.zeros(n), "u": np.zeros(n)}
    obj = C.c_double()
    _raise(capi.load().gpp_reduced_to_host(C.byref(summary), *(out[k].ctypes.data_as(C.c_void_p) for k in (
        "row_ptr", "col_idx", "val", "c", "AL", "AU", "l", "u")), C.byref(obj)))
    out["obj_constant"] = obj.value
    return out
