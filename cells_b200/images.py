"""Images of sampled fields, written on the host (there is no graphics pipeline on the device).

The reference colours its slices with a colour map on the GPU (src/shaders/render3d.ts:179-183,
solid nodes in grey 0.35); here Solver3D.sampleSlice returns the colour-map input (0..1, NaN on
solids) and these helpers turn it into a binary PPM with a piecewise-linear ramp of this package.
"""
from __future__ import annotations

import numpy as np

# ramp anchors: position in [0, 1] and an 8-bit RGB colour (dark blue, blue, teal, green, pale yellow)
_ANCHORS = np.array([0.0, 0.25, 0.5, 0.75, 1.0])
_COLOURS = np.array([[22, 18, 64], [38, 86, 170], [36, 158, 150], [150, 206, 84], [250, 238, 150]], dtype=np.float64)
SOLID_GREY = 89  # 0.35 * 255, the reference's solid colour


def colourise(values: np.ndarray) -> np.ndarray:
    """(rows, cols) field values -> (rows, cols, 3) uint8: values clamped to [0, 1] on the ramp,
    NaN (solid) in grey."""
    v = np.asarray(values, dtype=np.float64)
    solid = np.isnan(v)
    t = np.clip(np.where(solid, 0.0, v), 0.0, 1.0)
    rgb = np.stack([np.interp(t, _ANCHORS, _COLOURS[:, c]) for c in range(3)], axis=-1)
    rgb[solid] = SOLID_GREY
    return np.rint(rgb).astype(np.uint8)


def write_ppm(path: str, values: np.ndarray, flip_vertical: bool = True) -> None:
    """Writes a field slice as a binary PPM; row 0 of the slice is the bottom of the image unless
    flip_vertical is False."""
    rgb = colourise(values)
    if flip_vertical:
        rgb = rgb[::-1]
    h, w = rgb.shape[:2]
    with open(path, "wb") as f:
        f.write(f"P6\n{w} {h}\n255\n".encode("ascii"))
        f.write(np.ascontiguousarray(rgb).tobytes())
