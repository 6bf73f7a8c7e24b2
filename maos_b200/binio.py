"""MAOS .bin files from Python, through the native reader and writer
(include/shwfs_bin.h, maos_b200/csrc/host/binio.c).

Arrays map to Python as MAOS indexes them: a dense nx x ny array becomes a
numpy array of shape (nx, ny) in Fortran order (a[ix, iy] is P(A, ix, iy));
a cell becomes a numpy object array of shape (nx, ny) holding arrays or None;
a sparse matrix becomes a ``scipy.sparse.csc_matrix``.  ``read_bin`` with
``keywords=True`` also returns the header text.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import shwfs

M_DBL, M_INT64, M_CMP, M_INT32 = 0x6402, 0x6403, 0x6404, 0x6405
M_FLT, M_ZMP, M_INT8, M_INT16 = 0x6408, 0x6409, 0x640A, 0x640B
MCC_ANY = 0x6421
M_DSP64, M_DSP32, M_SSP64, M_SSP32 = 0x6401, 0x6407, 0x6430, 0x6431
M_CSP64, M_CSP32, M_ZSP64, M_ZSP32 = 0x6400, 0x6406, 0x6432, 0x6433

_DENSE = {M_DBL: np.float64, M_INT64: np.int64, M_CMP: np.complex128, M_INT32: np.int32, M_FLT: np.float32,
          M_ZMP: np.complex64, M_INT8: np.int8, M_INT16: np.int16}
_SPARSE = {M_DSP64: np.float64, M_DSP32: np.float64, M_SSP64: np.float32, M_SSP32: np.float32,
           M_CSP64: np.complex128, M_CSP32: np.complex128, M_ZSP64: np.complex64, M_ZSP32: np.complex64}
_MAGIC = {np.dtype(v): k for k, v in _DENSE.items()}


class BinArray(C.Structure):
    pass


BinArray._fields_ = [("id", C.c_uint32), ("nx", C.c_uint64), ("ny", C.c_uint64), ("keywords", C.c_char_p),
                     ("data", C.c_void_p), ("nnz", C.c_uint64), ("pp", C.POINTER(C.c_int64)),
                     ("pi", C.POINTER(C.c_int64)), ("cells", C.POINTER(C.POINTER(BinArray)))]
_P = C.POINTER(BinArray)
_bound = False


def _lib():
    global _bound
    L = shwfs.lib()
    if not _bound:
        L.shwfs_bin_read.argtypes = [C.c_char_p, C.POINTER(_P)]
        L.shwfs_bin_read_all.argtypes = [C.c_char_p, C.POINTER(_P)]
        L.shwfs_bin_write.argtypes = [C.c_char_p, _P]
        L.shwfs_bin_free.argtypes = [_P]
        L.shwfs_bin_free.restype = None
        L.shwfs_bin_error.restype = C.c_char_p
        L.shwfs_bin_new_dense.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p, C.c_char_p]
        L.shwfs_bin_new_dense.restype = _P
        L.shwfs_bin_new_sparse.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_char_p]
        L.shwfs_bin_new_sparse.restype = _P
        L.shwfs_bin_new_cell.argtypes = [C.c_uint64, C.c_uint64, C.c_char_p]
        L.shwfs_bin_new_cell.restype = _P
        for f in ("shwfs_bin_read", "shwfs_bin_read_all", "shwfs_bin_write"):
            getattr(L, f).restype = C.c_int
        _bound = True
    return L


class BinError(RuntimeError):
    pass


def _check(rc: int):
    if rc:
        raise BinError(_lib().shwfs_bin_error().decode())


def _to_py(p):
    if not p:
        return None, None
    a = p.contents
    kw = a.keywords.decode() if a.keywords else None
    nx, ny = int(a.nx), int(a.ny)
    if a.id == MCC_ANY:
        flat = np.empty(nx * ny, dtype=object)
        for i in range(nx * ny):
            flat[i] = _to_py(a.cells[i])[0]
        return flat.reshape((nx, ny), order="F"), kw
    if a.id in _SPARSE:
        import scipy.sparse as sp
        nnz = int(a.nnz)
        dt = np.dtype(_SPARSE[a.id])
        pp = np.ctypeslib.as_array(a.pp, shape=(ny + 1,)).copy()
        pi = np.ctypeslib.as_array(a.pi, shape=(max(nnz, 1),))[:nnz].copy()
        px = np.frombuffer(C.string_at(a.data, nnz * dt.itemsize), dtype=dt).copy()
        return sp.csc_matrix((px, pi, pp), shape=(nx, ny)), kw
    dt = np.dtype(_DENSE[a.id & 0xFFFF])
    buf = C.string_at(a.data, nx * ny * dt.itemsize) if nx * ny else b""
    return np.frombuffer(buf, dtype=dt).copy().reshape((nx, ny), order="F"), kw


def read_bin(path: str, keywords: bool = False):
    """First array of a .bin / .bin.gz file (None for an empty file)."""
    L = _lib()
    p = _P()
    _check(L.shwfs_bin_read(path.encode(), C.byref(p)))
    try:
        out, kw = _to_py(p)
    finally:
        L.shwfs_bin_free(p)
    return (out, kw) if keywords else out


def read_bin_all(path: str):
    """Every top-level array of a file, as a list."""
    L = _lib()
    p = _P()
    _check(L.shwfs_bin_read_all(path.encode(), C.byref(p)))
    try:
        out, _ = _to_py(p)
    finally:
        L.shwfs_bin_free(p)
    return list(out.reshape(-1, order="F"))


def _from_py(obj, kw: Optional[str]):
    L = _lib()
    kwb = kw.encode() if kw is not None else None
    if obj is None:
        return None
    try:
        import scipy.sparse as sp
        if sp.issparse(obj):
            m = sp.csc_matrix(obj)
            m.sort_indices()
            kinds = {np.dtype(np.float64): (M_DSP32, M_DSP64), np.dtype(np.float32): (M_SSP32, M_SSP64),
                     np.dtype(np.complex128): (M_CSP32, M_CSP64), np.dtype(np.complex64): (M_ZSP32, M_ZSP64)}
            if m.dtype not in kinds:
                m = m.astype(np.float64)
            big = m.nnz > 0x7FFFFFFF or max(m.shape) > 0x7FFFFFFF
            mid = kinds[m.dtype][1 if big else 0]
            pp = np.ascontiguousarray(m.indptr, dtype=np.int64)
            pi = np.ascontiguousarray(m.indices, dtype=np.int64)
            px = np.ascontiguousarray(m.data)
            return L.shwfs_bin_new_sparse(mid, m.shape[0], m.shape[1], m.nnz, pp.ctypes.data, pi.ctypes.data,
                                          px.ctypes.data, kwb)
    except ImportError:
        pass
    if isinstance(obj, (list, tuple)) or (isinstance(obj, np.ndarray) and obj.dtype == object):
        arr = np.empty(len(obj), dtype=object) if isinstance(obj, (list, tuple)) else obj
        if isinstance(obj, (list, tuple)):
            for i, o in enumerate(obj):
                arr[i] = o
        if arr.ndim == 1:
            arr = arr.reshape(-1, 1)
        nx, ny = arr.shape
        c = L.shwfs_bin_new_cell(nx, ny, kwb)
        flat = arr.reshape(-1, order="F")
        for i in range(nx * ny):
            c.contents.cells[i] = _from_py(flat[i], None) if flat[i] is not None else _P()
        return c
    a = np.asarray(obj)
    if a.dtype not in _MAGIC:
        a = a.astype(np.float64)
    if a.ndim == 0:
        a = a.reshape(1, 1)
    if a.ndim == 1:
        a = a.reshape(-1, 1)
    if a.ndim != 2:
        raise BinError("only 1-D and 2-D arrays have a .bin form")
    buf = np.asfortranarray(a)
    return L.shwfs_bin_new_dense(_MAGIC[a.dtype], a.shape[0], a.shape[1], buf.ctypes.data, kwb)


def write_bin(path: str, obj, keywords: Optional[str] = None):
    """Write an array, a sparse matrix or a cell (list / object array) to a
    .bin file (gzip when the name ends in .gz)."""
    L = _lib()
    p = _from_py(obj, keywords)
    try:
        _check(L.shwfs_bin_write(path.encode(), p if p is not None else _P()))
    finally:
        if p:
            L.shwfs_bin_free(p)
