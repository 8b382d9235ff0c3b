"""Circular detector mask (mirror of ebsdtorch/preprocessing/radial_mask.py:5-40)."""

from __future__ import annotations

from typing import Optional, Tuple

import torch


def get_radial_mask(shape: Tuple[int, int], radius: Optional[float] = None,
                    center: Tuple[float, float] = (0.5, 0.5)) -> torch.Tensor:
    """Boolean (h, w) mask of pixels strictly inside a circle of `radius`
    (default half the smaller side) centred at fractional `center`."""
    h, w = shape
    if radius is None:
        radius = min(h, w) / 2.0
    ii = torch.arange(h, dtype=torch.float32).view(-1, 1)
    jj = torch.arange(w, dtype=torch.float32).view(1, -1)
    d2 = (ii - center[0] * (h - 1)) ** 2 + (jj - center[1] * (w - 1)) ** 2
    return d2 < radius**2
