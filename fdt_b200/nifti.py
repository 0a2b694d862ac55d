"""Minimal NIfTI-1 single-file reader/writer (.nii, .nii.gz) for the bedpostx driver.

Covers what the path reads and writes: 3-D/4-D volumes of the common data types, the header
geometry (dims, pixdim, units, qform/sform) carried over from an input image to the outputs,
scaling (scl_slope/scl_inter) on read, and the display range (cal_min/cal_max) the reference
sets on its outputs (merge_parts_gpu.cc: setDisplayMaximumMinimum).  Data are stored with x
fastest (Fortran order), so a masked voxel list is taken in x-fastest order, as FSL's
volume4D::matrix(mask) / setmatrix(mask) do.
"""
from __future__ import annotations

import dataclasses
import gzip
import struct

import numpy as np

_DTYPES = {2: np.uint8, 4: np.int16, 8: np.int32, 16: np.float32, 64: np.float64, 256: np.int8, 512: np.uint16,
           768: np.uint32, 1024: np.int64, 1280: np.uint64}
_CODES = {np.dtype(v): k for k, v in _DTYPES.items()}
HDR_SIZE = 348


@dataclasses.dataclass
class Header:
    """The header fields the driver keeps (the rest are written as zeros)."""

    dim: tuple
    pixdim: tuple = (1.0,) * 8
    xyzt_units: int = 10  # mm, s
    qform_code: int = 0
    sform_code: int = 0
    quatern: tuple = (0.0,) * 6  # b, c, d, qoffset x, y, z
    srow: tuple = ((1.0, 0.0, 0.0, 0.0), (0.0, 1.0, 0.0, 0.0), (0.0, 0.0, 1.0, 0.0))
    cal_min: float = 0.0
    cal_max: float = 0.0
    descrip: str = ""


def _open(path: str, mode: str):
    return gzip.open(path, mode) if path.endswith(".gz") else open(path, mode)


def read(path: str) -> tuple[np.ndarray, Header]:
    """(array with shape dim[1..dim[0]] (x fastest in memory order 'F'), header)."""
    with _open(path, "rb") as f:
        raw = f.read()
    if len(raw) < HDR_SIZE:
        raise ValueError(f"{path}: too short for a NIfTI-1 header")
    endian = "<"
    if struct.unpack("<i", raw[:4])[0] != HDR_SIZE:
        endian = ">"
        if struct.unpack(">i", raw[:4])[0] != HDR_SIZE:
            raise ValueError(f"{path}: not a NIfTI-1 file (sizeof_hdr != 348)")
    magic = raw[344:348]
    if magic not in (b"n+1\x00", b"ni1\x00"):
        raise ValueError(f"{path}: bad NIfTI-1 magic {magic!r}")
    if magic == b"ni1\x00":
        raise ValueError(f"{path}: two-file NIfTI (.hdr/.img) is not supported")
    dim = struct.unpack(endian + "8h", raw[40:56])
    datatype, bitpix = struct.unpack(endian + "2h", raw[70:74])
    pixdim = struct.unpack(endian + "8f", raw[76:108])
    vox_offset = int(struct.unpack(endian + "f", raw[108:112])[0])
    slope, inter = struct.unpack(endian + "2f", raw[112:120])
    xyzt_units = raw[123]
    cal_max, cal_min = struct.unpack(endian + "2f", raw[124:132])
    descrip = raw[148:228].split(b"\x00")[0].decode(errors="replace")
    qform_code, sform_code = struct.unpack(endian + "2h", raw[252:256])
    quatern = struct.unpack(endian + "6f", raw[256:280])
    srow = tuple(struct.unpack(endian + "4f", raw[280 + 16 * r : 296 + 16 * r]) for r in range(3))
    if datatype not in _DTYPES:
        raise ValueError(f"{path}: unsupported NIfTI datatype {datatype}")
    nd = dim[0]
    if not 1 <= nd <= 7:
        raise ValueError(f"{path}: bad dim[0] = {nd}")
    shape = tuple(int(d) for d in dim[1 : nd + 1])
    if any(d < 1 for d in shape):
        raise ValueError(f"{path}: bad dimensions {shape}")
    dt = np.dtype(_DTYPES[datatype]).newbyteorder(endian)
    count = int(np.prod(shape))
    if vox_offset < HDR_SIZE or vox_offset + count * dt.itemsize > len(raw):
        raise ValueError(f"{path}: truncated: {count} voxels of {dt.itemsize} bytes from offset {vox_offset} "
                         f"need {vox_offset + count * dt.itemsize} bytes, the file has {len(raw)}")
    data = np.frombuffer(raw, dtype=dt, count=count, offset=vox_offset).reshape(shape, order="F")
    if slope != 0.0 and not (slope == 1.0 and inter == 0.0):
        data = data.astype(np.float32) * np.float32(slope) + np.float32(inter)
    hdr = Header(dim=tuple(dim), pixdim=tuple(pixdim), xyzt_units=xyzt_units, qform_code=qform_code,
                 sform_code=sform_code, quatern=tuple(quatern), srow=srow, cal_min=cal_min, cal_max=cal_max,
                 descrip=descrip)
    return np.asarray(data), hdr


def write(path: str, data: np.ndarray, like: Header | None = None, cal: tuple | None = None,
          descrip: str = "") -> None:
    """Writes `data` (3-D or 4-D, float32 unless integer) as single-file NIfTI-1 with the
    geometry of `like` (pixdim of the spatial axes, units, qform/sform)."""
    a = np.asarray(data)
    if a.dtype not in _CODES:
        a = a.astype(np.float32)
    nd = a.ndim
    if not 1 <= nd <= 7:
        raise ValueError("data must have 1..7 dimensions")
    dim = [nd] + list(a.shape) + [1] * (7 - nd)
    pix = list(like.pixdim) if like else [1.0] * 8
    pix[0] = pix[0] if pix[0] in (-1.0, 1.0) else 1.0
    for i in range(nd + 1, 8):
        pix[i] = 1.0
    h = bytearray(HDR_SIZE)
    struct.pack_into("<i", h, 0, HDR_SIZE)
    struct.pack_into("<8h", h, 40, *dim)
    code = _CODES[a.dtype]
    struct.pack_into("<2h", h, 70, code, a.dtype.itemsize * 8)
    struct.pack_into("<8f", h, 76, *pix)
    struct.pack_into("<f", h, 108, 352.0)
    struct.pack_into("<2f", h, 112, 1.0, 0.0)
    h[123] = like.xyzt_units if like else 10
    cmin, cmax = cal if cal is not None else (0.0, 0.0)
    struct.pack_into("<2f", h, 124, float(cmax), float(cmin))
    d = (descrip or (like.descrip if like else "")).encode()[:79]
    h[148 : 148 + len(d)] = d
    if like:
        struct.pack_into("<2h", h, 252, like.qform_code, like.sform_code)
        struct.pack_into("<6f", h, 256, *like.quatern)
        for r in range(3):
            struct.pack_into("<4f", h, 280 + 16 * r, *like.srow[r])
    h[344:348] = b"n+1\x00"
    with _open(path, "wb") as f:
        f.write(bytes(h))
        f.write(b"\x00\x00\x00\x00")  # no extensions
        f.write(np.ascontiguousarray(a.astype(a.dtype.newbyteorder("<")).reshape(-1, order="F")).tobytes())


def mask_indices(mask: np.ndarray) -> np.ndarray:
    """Linear (x-fastest) indices of the voxels where mask != 0, in FSL's matrix(mask) order."""
    return np.flatnonzero(np.asarray(mask).reshape(-1, order="F") != 0)


def to_matrix(vol4: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """[nvox][nt] values of a 4-D volume at the mask's voxels (nt = 1 for a 3-D volume)."""
    v = np.asarray(vol4)
    if v.ndim == 3:
        v = v[..., None]
    flat = v.reshape(-1, v.shape[3], order="F")
    return flat[mask_indices(mask)]


def from_matrix(mat: np.ndarray, mask: np.ndarray, fill: float = 0.0) -> np.ndarray:
    """Inverse of to_matrix: [nvox] or [nvox][nt] -> 3-D or 4-D volume of the mask's shape."""
    m = np.asarray(mat)
    idx = mask_indices(mask)
    if m.shape[0] != idx.size:
        raise ValueError("matrix rows do not match the mask's voxel count")
    nt = 1 if m.ndim == 1 else m.shape[1]
    out = np.full((int(np.prod(mask.shape)), nt), fill, dtype=np.float32)
    out[idx] = m.reshape(idx.size, nt)
    vol = out.reshape(tuple(mask.shape) + (nt,), order="F")
    return vol[..., 0] if m.ndim == 1 else vol
