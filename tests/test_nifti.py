"""NIfTI-1 reading and writing (include/broccoli_nifti.h) on the CPU.

The files of the read tests are packed here from the NIfTI-1 header layout
(348 bytes, magic "n+1", data at vox_offset), so the reader is checked
against an independent writer: every datatype the reference's tools convert
(UINT8, INT16, UINT16, FLOAT32; MotionCorrection.cpp:422-460) plus INT8,
INT32, UINT32 and FLOAT64, both byte orders, plain and gzip files."""
import gzip
import os
import struct

import numpy as np
import pytest

from broccoli_b200 import _lib as L
from broccoli_b200 import nifti

CODES = {np.uint8: 2, np.int16: 4, np.int32: 8, np.float32: 16, np.float64: 64, np.int8: 256, np.uint16: 512,
         np.uint32: 768}


def pack_nifti(data: np.ndarray, pixdim=(2.0, 2.5, 3.0), big_endian=False, vox_offset=352, magic=b"n+1\0",
               scl_slope=1.0) -> bytes:
    e = ">" if big_endian else "<"
    shape = data.shape[::-1]  # x fastest
    h = bytearray(348)
    struct.pack_into(e + "i", h, 0, 348)
    dims = [len(shape)] + list(shape) + [1] * (7 - len(shape))
    struct.pack_into(e + "8h", h, 40, *dims)
    dt = data.dtype.type
    struct.pack_into(e + "h", h, 70, CODES[dt])
    struct.pack_into(e + "h", h, 72, data.dtype.itemsize * 8)
    struct.pack_into(e + "8f", h, 76, 1.0, *pixdim, 1.0, 1.0, 1.0, 1.0)
    struct.pack_into(e + "f", h, 108, float(vox_offset))
    struct.pack_into(e + "f", h, 112, scl_slope)
    struct.pack_into(e + "h", h, 252, 1)  # qform_code
    struct.pack_into(e + "6f", h, 256, 0.1, 0.2, 0.3, -10.0, -20.0, -30.0)
    h[148:148 + 11] = b"test header"
    h[344:348] = magic
    body = np.ascontiguousarray(data).astype(data.dtype.newbyteorder(e)).tobytes()
    return bytes(h) + b"\0" * (vox_offset - 348) + body


@pytest.mark.parametrize("dtype", list(CODES))
@pytest.mark.parametrize("big_endian", [False, True])
def test_read_every_datatype_and_byte_order(tmp_path, dtype, big_endian):
    rng = np.random.default_rng(5)
    info = np.iinfo(dtype) if np.issubdtype(dtype, np.integer) else None
    lo, hi = (max(info.min, -30000), min(info.max, 30000)) if info else (-1e3, 1e3)
    vol = rng.uniform(lo, hi, (3, 4, 5)).astype(dtype)
    path = os.path.join(tmp_path, "v.nii")
    open(path, "wb").write(pack_nifti(vol, big_endian=big_endian))
    img = nifti.read(path)
    assert img.data.shape == (3, 4, 5) and img.data.dtype == np.float32
    assert np.array_equal(img.data, vol.astype(np.float32))
    assert img.voxel_size == (2.0, 2.5, 3.0)
    assert img.datatype == CODES[dtype]


def test_read_gzip_4d_and_extensions(tmp_path):
    vols = np.arange(2 * 3 * 4 * 5, dtype=np.int16).reshape(2, 3, 4, 5) - 50
    path = os.path.join(tmp_path, "s.nii.gz")
    with gzip.open(path, "wb") as f:
        f.write(pack_nifti(vols, vox_offset=368))  # 16 bytes of extension space
    img = nifti.read(path)
    assert img.data.shape == (2, 3, 4, 5)
    assert np.array_equal(img.data, vols.astype(np.float32))


def test_scaling_is_not_applied(tmp_path):
    vol = np.full((2, 2, 2), 7, np.int16)
    path = os.path.join(tmp_path, "s.nii")
    open(path, "wb").write(pack_nifti(vol, scl_slope=3.0))
    assert np.all(nifti.read(path).data == 7.0)  # plain cast, as the reference's tools


@pytest.mark.parametrize("name", ["out.nii", "out.nii.gz"])
def test_write_round_trip_keeps_header(tmp_path, name):
    vol = np.random.default_rng(1).standard_normal((3, 4, 5)).astype(np.int16)
    src = os.path.join(tmp_path, "in.nii")
    open(src, "wb").write(pack_nifti(vol, big_endian=True))
    like = nifti.read(src)
    data = np.random.default_rng(2).standard_normal((2, 3, 4, 5)).astype(np.float32)
    dst = os.path.join(tmp_path, name)
    nifti.write(dst, data, like)
    back = nifti.read(dst)
    assert np.array_equal(back.data, data)
    assert back.datatype == 16 and back.voxel_size == like.voxel_size
    h = back.header
    assert struct.unpack_from("<8h", h, 40)[:5] == (4, 5, 4, 3, 2)
    assert struct.unpack_from("<f", h, 124)[0] == data.max() and struct.unpack_from("<f", h, 128)[0] == data.min()
    assert h[148:159] == b"test header" and struct.unpack_from("<h", h, 252)[0] == 1
    assert struct.unpack_from("<6f", h, 256) == struct.unpack_from("<6f", like.header, 256)
    raw = gzip.open(dst).read() if name.endswith(".gz") else open(dst, "rb").read()
    assert len(raw) == 352 + data.nbytes and raw[344:348] == b"n+1\0"


def test_write_without_template(tmp_path):
    data = np.ones((2, 3, 4), np.float32)
    dst = os.path.join(tmp_path, "plain.nii")
    nifti.write(dst, data)
    back = nifti.read(dst)
    assert np.array_equal(back.data, data) and back.voxel_size == (1.0, 1.0, 1.0)


def test_errors(tmp_path):
    bad = os.path.join(tmp_path, "bad.nii")
    open(bad, "wb").write(b"\0" * 400)
    with pytest.raises(L.BrcError) as e:
        nifti.read(bad)
    assert e.value.status == L.BRC_ERR_INVALID
    pair = os.path.join(tmp_path, "pair.nii")
    open(pair, "wb").write(pack_nifti(np.zeros((2, 2, 2), np.float32), magic=b"ni1\0"))
    with pytest.raises(L.BrcError) as e:
        nifti.read(pair)
    assert e.value.status == L.BRC_ERR_UNSUPPORTED
    trunc = os.path.join(tmp_path, "trunc.nii")
    open(trunc, "wb").write(pack_nifti(np.zeros((4, 4, 4), np.float32))[:500])
    with pytest.raises(L.BrcError) as e:
        nifti.read(trunc)
    assert e.value.status == L.BRC_ERR_INVALID
    with pytest.raises(L.BrcError):
        nifti.read(os.path.join(tmp_path, "missing.nii"))
    with pytest.raises(L.BrcError):
        nifti.read(os.path.join(tmp_path, "x.hdr"))
