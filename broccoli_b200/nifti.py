"""NIfTI-1 reading and writing through libbroccoli_b200 (include/broccoli_nifti.h).

``read(path)`` returns a ``NiftiImage`` whose ``data`` is float32 shaped
(T, D, H, W) for 4D images and (D, H, W) otherwise (x fastest, as the
library's volumes); ``write(path, data, like)`` writes FLOAT32 under the
header of ``like`` (another ``NiftiImage``) or a minimal header.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L


class _Nifti(ctypes.Structure):
    _fields_ = [("header", ctypes.c_ubyte * 348), ("dim", ctypes.c_int * 8), ("pixdim", ctypes.c_float * 8),
                ("datatype", ctypes.c_int), ("data", ctypes.POINTER(ctypes.c_float))]


class NiftiImage:
    def __init__(self, data: np.ndarray, header: bytes, pixdim, datatype: int):
        self.data = data
        self.header = header
        self.pixdim = np.asarray(pixdim, np.float32)
        self.datatype = datatype

    @property
    def voxel_size(self):
        return tuple(float(v) for v in self.pixdim[1:4])


def _fns():
    lib = L.lib()
    lib.brc_nifti_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Nifti)]
    lib.brc_nifti_read.restype = ctypes.c_int
    lib.brc_nifti_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Nifti), ctypes.c_void_p] + [ctypes.c_int] * 4
    lib.brc_nifti_write.restype = ctypes.c_int
    lib.brc_nifti_free.argtypes = [ctypes.POINTER(_Nifti)]
    lib.brc_nifti_free.restype = None
    lib.brc_nifti_error.argtypes = []
    lib.brc_nifti_error.restype = ctypes.c_char_p
    return lib


def read(path: str) -> NiftiImage:
    lib = _fns()
    img = _Nifti()
    s = lib.brc_nifti_read(path.encode(), ctypes.byref(img))
    if s != L.BRC_OK:
        raise L.BrcError(s, lib.brc_nifti_error().decode())
    try:
        nd = img.dim[0]
        shape = [img.dim[k] for k in range(1, nd + 1)]
        n = int(np.prod(shape))
        flat = np.ctypeslib.as_array(img.data, shape=(n,)).copy()
    finally:
        lib.brc_nifti_free(ctypes.byref(img))
    # x fastest: reverse the NIfTI dimension order
    data = flat.reshape(shape[::-1]) if nd > 1 else flat
    if nd > 4:
        data = data.reshape((-1,) + tuple(shape[:3][::-1]))
    return NiftiImage(data, bytes(img.header), list(img.pixdim), img.datatype)


def write(path: str, data: np.ndarray, like: NiftiImage | None = None) -> None:
    lib = _fns()
    a = np.ascontiguousarray(data, np.float32)
    if a.ndim == 3:
        T, (D, H, W) = 1, a.shape
    elif a.ndim == 4:
        T, D, H, W = a.shape
    else:
        raise ValueError("write: (D, H, W) or (T, D, H, W) data")
    ref = None
    if like is not None:
        ref = _Nifti()
        ctypes.memmove(ref.header, like.header, 348)
    s = lib.brc_nifti_write(path.encode(), ctypes.byref(ref) if ref is not None else None,
                            a.ctypes.data_as(ctypes.c_void_p), W, H, D, T)
    if s != L.BRC_OK:
        raise L.BrcError(s, lib.brc_nifti_error().decode())
