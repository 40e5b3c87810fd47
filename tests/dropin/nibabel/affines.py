import numpy as np


def apply_affine(aff, pts):
    """points [..., 3] mapped by the 4 x 4 affine (nibabel.affines.apply_affine)"""
    aff = np.asarray(aff, np.float64)
    pts = np.asarray(pts, np.float64)
    shape = pts.shape
    p = pts.reshape(-1, shape[-1])
    out = p @ aff[:-1, :-1].T + aff[:-1, -1]
    return out.reshape(shape)
