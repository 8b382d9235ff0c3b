"""Whole-scan pattern passes behind ExperimentPatterns' preprocessing methods
(mirror of ebsdtorch/ebsd/experiment_pats.py:223-297).

Every function takes patterns of shape (..., H, W) on any device, computes
in FP32 on the GPU (host tensors go to the current CUDA device and back) and
returns the result with the input's shape on the input's device. CUDA FP32
contiguous inputs are processed in place, as the reference's ``-=`` / ``/=``
updates do; other inputs (integer counts, FP64, strided) are converted to
FP32 first.
"""

from __future__ import annotations

from typing import Callable, Tuple

import torch
from torch import Tensor

from .._capi import call, ptr
from .._device import on_data_device

NORM_MODES = {"minmax": 0, "zeromean": 1, "standard": 2}


def device_rows(x: Tensor, n_cols: int) -> Tuple[Tensor, Callable[[Tensor], Tensor]]:
    """(rows, back): `x` as contiguous FP32 CUDA rows of `n_cols` values and
    a function that moves a result back to `x`'s device."""
    if x.device.type == "cuda":
        rows = x.reshape(-1, n_cols)
        if rows.dtype != torch.float32 or not rows.is_contiguous():
            rows = rows.float().contiguous()
        return rows, (lambda y: y)
    if not torch.cuda.is_available():
        raise RuntimeError("ebsdtorch_b200 preprocessing runs on CUDA (sm_100) devices only; no GPU is visible")
    dev = torch.device("cuda", torch.cuda.current_device())
    rows = x.reshape(-1, n_cols).to(dev, dtype=torch.float32).contiguous()
    return rows, (lambda y: y.to(x.device))


def _stream(t: Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


@on_data_device
def pattern_mean(rows: Tensor) -> Tensor:
    """Mean over the rows of a (N, P) FP32 CUDA tensor, summed in FP64."""
    n, n_pix = rows.shape
    sms = torch.cuda.get_device_properties(rows.device).multi_processor_count
    col_blocks = (n_pix + 255) // 256
    n_splits = max(1, min((n + 31) // 32, -(-4 * sms // col_blocks), 65535))
    partial = torch.empty((n_splits, n_pix), dtype=torch.float64, device=rows.device)
    mean = torch.empty(n_pix, dtype=torch.float32, device=rows.device)
    call("ebsd_pattern_mean", ptr(rows), n, n_pix, rows.stride(0), ptr(partial), n_splits, ptr(mean), _stream(rows))
    return mean


@on_data_device
def subtract_overall_background(patterns: Tensor) -> Tensor:
    """patterns minus the scan's mean pattern (experiment_pats.py:223-232)."""
    h, w = patterns.shape[-2:]
    rows, back = device_rows(patterns, h * w)
    if rows.shape[0] == 0:
        return patterns
    mean = pattern_mean(rows)
    call("ebsd_subtract_pattern", ptr(rows), rows.shape[0], h * w, rows.stride(0), ptr(mean), _stream(rows))
    return back(rows).view(patterns.shape)


@on_data_device
def normalize_per_pattern(patterns: Tensor, norm_type: str = "minmax") -> Tensor:
    """Per-pattern "minmax", "zeromean" or "standard" normalisation
    (experiment_pats.py:255-285)."""
    if norm_type not in NORM_MODES:
        raise ValueError(
            f"Invalid normalization method. Got {norm_type} but expected 'minmax', 'zeromean', or 'standard'.")
    h, w = patterns.shape[-2:]
    rows, back = device_rows(patterns, h * w)
    if rows.shape[0] == 0:
        return patterns
    call("ebsd_normalize_patterns", ptr(rows), rows.shape[0], h * w, rows.stride(0), NORM_MODES[norm_type],
         _stream(rows))
    return back(rows).view(patterns.shape)


@on_data_device
def standard_clean(patterns: Tensor, clip_limit: float = 40.0, tile_grid_size: int = 4, n_bins: int = 64) -> Tensor:
    """Background subtraction, min-max, CLAHE, min-max
    (experiment_pats.py:287-297): one mean pass and one fused CLAHE pass
    (each pattern read once and written once)."""
    h, w = patterns.shape[-2:]
    rows, back = device_rows(patterns, h * w)
    if rows.shape[0] == 0:
        return patterns
    mean = pattern_mean(rows)
    call("ebsd_clahe", ptr(rows), rows.shape[0], h, w, rows.stride(0), ptr(mean), 1, float(clip_limit), int(n_bins),
         int(tile_grid_size), int(tile_grid_size), 1, ptr(rows), rows.stride(0), _stream(rows))
    return back(rows).view(patterns.shape)
