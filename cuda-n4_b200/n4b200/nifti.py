"""Minimal NIfTI-1 (.nii / .nii.gz) reader and writer.

Replaces the ITK image I/O of the reference (``itkLoadVolume.h``).  The
reference reads a volume into a buffer with x fastest (``itkLoadVolume.h:116``,
``c + r*C + d*C*R``) and passes ``fx = size[2]`` (the slowest NIfTI axis) to
``testN4`` (``main.cpp:153-155``), so its ``[fx][fy][fz]`` array with fz
fastest is the NIfTI data read as a C-ordered ``(nz, ny, nx)`` array.  That is
what ``load`` returns; ``save`` writes such an array back with the header
(dimensions, voxel sizes, orientation) of a reference image.
"""
from __future__ import annotations

import gzip
import struct
from dataclasses import dataclass

import numpy as np

__all__ = ["NiftiImage", "load", "save"]

_DTYPES = {2: np.uint8, 4: np.int16, 8: np.int32, 16: np.float32, 64: np.float64,
           256: np.int8, 512: np.uint16, 768: np.uint32}


@dataclass
class NiftiImage:
    data: np.ndarray          # C order (nz, ny, nx): the reference's [fx][fy][fz]
    header: bytes             # the 348-byte header it was read with
    spacing: tuple            # voxel sizes (x, y, z)


def _open(path, mode):
    return gzip.open(path, mode) if str(path).endswith(".gz") else open(path, mode)


def load(path) -> NiftiImage:
    with _open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 348:
        raise ValueError(f"{path}: not a NIfTI-1 file")
    endian = "<"
    if struct.unpack("<i", raw[:4])[0] != 348:
        endian = ">"
        if struct.unpack(">i", raw[:4])[0] != 348:
            raise ValueError(f"{path}: bad NIfTI-1 header size")
    hdr = raw[:348]
    dim = struct.unpack(endian + "8h", hdr[40:56])
    datatype, = struct.unpack(endian + "h", hdr[70:72])
    pixdim = struct.unpack(endian + "8f", hdr[76:108])
    vox_offset, = struct.unpack(endian + "f", hdr[108:112])
    slope, inter = struct.unpack(endian + "2f", hdr[112:120])
    if dim[0] < 3:
        raise ValueError(f"{path}: expected a 3-D volume")
    if datatype not in _DTYPES:
        raise ValueError(f"{path}: unsupported NIfTI datatype {datatype}")
    nx, ny, nz = dim[1], dim[2], dim[3]
    dt = np.dtype(_DTYPES[datatype]).newbyteorder(endian)
    off = int(vox_offset) if vox_offset >= 348 else 352
    count = nx * ny * nz
    arr = np.frombuffer(raw, dtype=dt, count=count, offset=off).astype(np.float32)
    if slope not in (0.0, 1.0) or inter != 0.0:
        arr = arr * (slope if slope != 0.0 else 1.0) + inter
    return NiftiImage(arr.reshape(nz, ny, nx), bytes(hdr) if endian == "<" else _swap_header(hdr),
                      (pixdim[1], pixdim[2], pixdim[3]))


def _swap_header(hdr: bytes) -> bytes:
    """Re-encode the fields this module writes back in little-endian order."""
    out = bytearray(_blank_header())
    dim = struct.unpack(">8h", hdr[40:56])
    pixdim = struct.unpack(">8f", hdr[76:108])
    out[40:56] = struct.pack("<8h", *dim)
    out[76:108] = struct.pack("<8f", *pixdim)
    return bytes(out)


def _blank_header() -> bytes:
    h = bytearray(348)
    struct.pack_into("<i", h, 0, 348)
    h[344:348] = b"n+1\0"
    return bytes(h)


def save(path, data: np.ndarray, like: NiftiImage | None = None, spacing=(1.0, 1.0, 1.0)):
    """Write a float32 volume given as C-ordered (nz, ny, nx)."""
    data = np.ascontiguousarray(np.asarray(data, dtype=np.float32))
    if data.ndim != 3:
        raise ValueError("expected a 3-D array")
    nz, ny, nx = data.shape
    h = bytearray(like.header if like is not None else _blank_header())
    struct.pack_into("<i", h, 0, 348)
    struct.pack_into("<8h", h, 40, 3, nx, ny, nz, 1, 1, 1, 1)
    struct.pack_into("<h", h, 70, 16)       # float32
    struct.pack_into("<h", h, 72, 32)       # bitpix
    if like is None:
        struct.pack_into("<8f", h, 76, 1.0, *spacing, 1.0, 1.0, 1.0, 1.0)
    struct.pack_into("<f", h, 108, 352.0)   # vox_offset
    struct.pack_into("<2f", h, 112, 1.0, 0.0)
    h[344:348] = b"n+1\0"
    with _open(path, "wb") as f:
        f.write(bytes(h))
        f.write(b"\0\0\0\0")                # extension flag: none
        f.write(data.tobytes())
