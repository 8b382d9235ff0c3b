"""Contrast-limited adaptive histogram equalisation (mirror of
ebsdtorch/preprocessing/clahe.py:17-130).

`clahe_grayscale` keeps the reference's signature and result: per image,
tile histograms of floor(x (n_bins - 1)) over the bottom/right
reflect-padded image, clipped at max(clip_limit * tile_pixels // n_bins, 1)
with the excess redistributed, cumulated into CDFs and read back per pixel by
trilinear interpolation over (tile row, tile column, bin) with grid_sample's
align_corners=False / border rules. All of it is one kernel launch
(`ebsd_clahe`, one CTA per image, the image staged in shared memory).
"""

from __future__ import annotations

from typing import Tuple

from torch import Tensor

from .._capi import call, ptr
from .patterns import _stream, device_rows
from .._device import on_data_device


@on_data_device
def clahe_grayscale(x: Tensor, clip_limit: float = 40.0, n_bins: int = 64,
                    grid_shape: Tuple[int, int] = (4, 4)) -> Tensor:
    """CLAHE of images (..., H, W) with values in [0, 1]; returns the same
    shape on the input's device (FP32)."""
    h, w = x.shape[-2:]
    rows, back = device_rows(x, h * w)
    out = rows.new_empty(rows.shape)
    if rows.shape[0]:
        call("ebsd_clahe", ptr(rows), rows.shape[0], h, w, rows.stride(0), None, 0, float(clip_limit), int(n_bins),
             int(grid_shape[0]), int(grid_shape[1]), 0, ptr(out), out.stride(0), _stream(rows))
    return back(out).view(x.shape)
