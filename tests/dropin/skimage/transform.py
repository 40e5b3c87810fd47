"""skimage.transform.resize (order 1) and warp with a coordinate array, on scipy.ndimage (the
published semantics of skimage 0.19+: anti-aliasing Gaussian when down-sampling, grid-mode zoom
with mirror boundaries, output clipped to the input range)."""
import numpy as np
from scipy import ndimage


def resize(image, output_shape, order=1, mode="reflect", cval=0, clip=True,
           preserve_range=False, anti_aliasing=None, anti_aliasing_sigma=None):
    image = np.asarray(image, np.float64)
    output_shape = tuple(output_shape)
    if len(output_shape) < image.ndim:
        output_shape = output_shape + image.shape[len(output_shape):]
    factors = np.divide(image.shape, output_shape)
    if anti_aliasing is None:
        anti_aliasing = np.any(factors > 1)
    if anti_aliasing:
        sigma = np.maximum(0, (factors - 1) / 2)
        image = ndimage.gaussian_filter(image, sigma, cval=cval, mode="mirror")
    zoom = [o / i for o, i in zip(output_shape, image.shape)]
    out = ndimage.zoom(image, zoom, order=order, mode="mirror", cval=cval, grid_mode=True)
    if clip:
        out = np.clip(out, image.min(), image.max())
    return out


def warp(image, inverse_map, map_args=None, output_shape=None, order=None, mode="constant",
         cval=0.0, clip=True, preserve_range=False):
    image = np.asarray(image, np.float64)
    coords = np.asarray(inverse_map, np.float64)
    order = 1 if order is None else order
    out = ndimage.map_coordinates(image, coords, order=order, mode="constant", cval=cval,
                                  prefilter=order > 1)
    if clip:
        lo, hi = min(image.min(), cval), max(image.max(), cval)
        out = np.clip(out, lo, hi)
    return out
