"""Stand-in for skimage.transform (resize, warp) on scipy.ndimage."""
