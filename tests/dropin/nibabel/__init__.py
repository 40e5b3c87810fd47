"""Stand-in for the part of nibabel the reference's Python layer uses: NIfTI-1 read / write
(the header parsed with gzip + struct) and affines.apply_affine."""
import gzip
import struct

import numpy as np

from . import affines  # noqa: F401

_DTYPES = {2: np.uint8, 4: np.int16, 8: np.int32, 16: np.float32, 64: np.float64, 256: np.int8,
           512: np.uint16, 768: np.uint32}
_CODES = {np.dtype(v): k for k, v in _DTYPES.items()}


class Nifti1Image:
    def __init__(self, dataobj, affine, header=None):
        self._data = np.asarray(dataobj)
        self.affine = np.asarray(affine, np.float64) if affine is not None else np.eye(4)
        self.header = header

    @property
    def shape(self):
        return self._data.shape

    def get_fdata(self):
        return np.asarray(self._data, np.float64)


def _open(path):
    with open(path, "rb") as f:
        raw = f.read()
    return gzip.decompress(raw) if raw[:2] == b"\x1f\x8b" else raw


def load(path):
    b = _open(str(path))
    end = "<" if struct.unpack("<i", b[:4])[0] == 348 else ">"
    dim = struct.unpack(end + "8h", b[40:56])
    datatype = struct.unpack(end + "h", b[70:72])[0]
    vox_offset = int(struct.unpack(end + "f", b[108:112])[0])
    slope, inter = struct.unpack(end + "2f", b[112:120])
    pixdim = struct.unpack(end + "8f", b[76:108])
    qform_code, sform_code = struct.unpack(end + "2h", b[252:256])
    shape = tuple(int(d) for d in dim[1:1 + dim[0]])
    dt = np.dtype(_DTYPES[datatype]).newbyteorder(end)
    n = int(np.prod(shape))
    data = np.frombuffer(b, dt, n, vox_offset).reshape(shape, order="F").astype(np.float64)
    if slope not in (0.0, 1.0) or inter != 0.0:
        data = data * (slope if slope != 0.0 else 1.0) + inter
    if sform_code > 0:
        srow = np.array(struct.unpack(end + "12f", b[280:328]), np.float64).reshape(3, 4)
        aff = np.vstack([srow, [0, 0, 0, 1]])
    elif qform_code > 0:
        qb, qc, qd, qx, qy, qz = struct.unpack(end + "6f", b[256:280])
        qa = np.sqrt(max(0.0, 1.0 - (qb * qb + qc * qc + qd * qd)))
        R = np.array([[qa * qa + qb * qb - qc * qc - qd * qd, 2 * (qb * qc - qa * qd),
                       2 * (qb * qd + qa * qc)],
                      [2 * (qb * qc + qa * qd), qa * qa + qc * qc - qb * qb - qd * qd,
                       2 * (qc * qd - qa * qb)],
                      [2 * (qb * qd - qa * qc), 2 * (qc * qd + qa * qb),
                       qa * qa + qd * qd - qc * qc - qb * qb]])
        qfac = -1.0 if pixdim[0] < 0 else 1.0
        R = R @ np.diag([pixdim[1], pixdim[2], pixdim[3] * qfac])
        aff = np.eye(4)
        aff[:3, :3] = R
        aff[:3, 3] = (qx, qy, qz)
    else:
        aff = np.diag([pixdim[1], pixdim[2], pixdim[3], 1.0])
    return Nifti1Image(data, aff)


def save(img, path):
    """NIfTI-1 single file, FP64 data, sform = the image's affine (gzip when the name ends .gz)"""
    data = np.asarray(img.get_fdata(), np.float64)
    hdr = bytearray(352)
    struct.pack_into("<i", hdr, 0, 348)
    dims = [data.ndim] + list(data.shape) + [1] * (7 - data.ndim)
    struct.pack_into("<8h", hdr, 40, *dims)
    struct.pack_into("<h", hdr, 70, 64)      # FLOAT64
    struct.pack_into("<h", hdr, 72, 64)      # bitpix
    struct.pack_into("<8f", hdr, 76, 1.0, *np.sqrt((img.affine[:3, :3] ** 2).sum(0)), 1, 1, 1, 1)
    struct.pack_into("<f", hdr, 108, 352.0)  # vox_offset
    struct.pack_into("<2f", hdr, 112, 1.0, 0.0)
    struct.pack_into("<2h", hdr, 252, 0, 1)  # qform 0, sform 1
    struct.pack_into("<12f", hdr, 280, *img.affine[:3, :].ravel())
    hdr[344:348] = b"n+1\x00"
    payload = bytes(hdr) + data.astype("<f8").tobytes(order="F")
    path = str(path)
    with open(path, "wb") as f:
        f.write(gzip.compress(payload) if path.endswith(".gz") else payload)
