"""Experimental-pattern container and result sink (mirror of
ebsdtorch/ebsd/experiment_pats.py).

Patterns may live on a CUDA device or in (preferably pinned) host memory;
dictionary indexing streams host-resident patterns to the GPU chunk by chunk.
Indexing results are stored exactly as the reference stores them
(``raw_indexing_results[phase] = (quaternions (N, k, 4), metrics (N, k))``,
then ``orientations``, ``best_metrics``, ``phases``).
"""

from __future__ import annotations

from typing import List, Optional

import torch
from torch import Tensor
from torch.nn import Module

from .. import kernels
from ..preprocessing import patterns as _pre
from ..preprocessing.clahe import clahe_grayscale
from ..preprocessing.nlpar import nlpar


class ExperimentPatterns(Module):
    """patterns: (SCAN_H, SCAN_W, H, W), (N_PATS, H, W) or (H, W)
    (experiment_pats.py:19-56)."""

    def __init__(self, patterns: Tensor):
        super().__init__()
        if len(patterns.shape) < 2:
            raise ValueError("'patterns' requires >= 2 dimensions (B, H, W) or (H, W)")
        if len(patterns.shape) < 3:
            patterns = patterns.unsqueeze(0)
        if len(patterns.shape) > 4:
            raise ValueError(
                "3D Volume not yet supported... 'patterns' requires dimensions: "
                "(SCAN_H, SCAN_W, H, W), (N_PATS, H, W), or (H, W)"
            )
        self.pattern_shape = patterns.shape[-2:]
        self.spatial_shape = patterns.shape[:-2] if len(patterns.shape) > 2 else (1, 1)
        self.patterns = patterns.reshape(-1, *patterns.shape[-2:])
        self.n_patterns = self.patterns.shape[0]
        self.n_pixels = self.pattern_shape[0] * self.pattern_shape[1]
        self.phases = None
        self.orientations = None
        self.best_metrics = None
        self.spatial_coords = None

    def set_spatial_coords(self, spatial_coords: Tensor, indices: Optional[Tensor] = None):
        if indices is None:
            if spatial_coords.shape[0] != self.n_patterns:
                raise ValueError(
                    "Spatial coordinates must have the same number of patterns as the ExperimentPatterns object. "
                    f"Got {spatial_coords.shape[0]} spatial coordinates and {self.n_patterns} patterns.")
            self.spatial_coords = spatial_coords
        else:
            if spatial_coords.shape[0] != indices.shape[0]:
                raise ValueError(
                    "Spatial coordinates must have the same number of patterns as the indices. "
                    f"Got {spatial_coords.shape[0]} spatial coordinates and {indices.shape[0]} indices.")
            self.spatial_coords[indices] = spatial_coords

    def get_spatial_coords(self, indices: Optional[Tensor] = None) -> Tensor:
        if self.spatial_coords is None:
            raise ValueError("Spatial coordinates must be set before retrieving them.")
        return self.spatial_coords if indices is None else self.spatial_coords[indices]

    def set_orientations(self, orientations: Tensor, indices: Optional[Tensor] = None):
        if len(orientations.shape) != 2:
            raise ValueError(f"Orientations must be quaternions (N_ORI, 4). Got {orientations.shape}.")
        if orientations.shape[1] != 4:
            raise ValueError(f"Orientations must be quaternions (w, x, y, z). Got {orientations.shape[1]}.")
        if indices is None:
            if orientations.shape[0] != self.n_patterns:
                raise ValueError(
                    "Orientations must have the same number of patterns as the ExperimentPatterns object. "
                    f"Got {orientations.shape[0]} orientations and {self.n_patterns} patterns.")
            self.orientations = orientations
        else:
            if len(indices.shape) != 1:
                raise ValueError(f"Indices must be (N_ORI,). Got {indices.shape}.")
            if orientations.shape[0] != indices.shape[0]:
                raise ValueError(
                    "Orientations must have the same number of patterns as the indices. "
                    f"Got {orientations.shape[0]} orientations and {indices.shape[0]} indices.")
            self.orientations[indices] = orientations

    def get_orientations(self, indices: Optional[Tensor] = None) -> Tensor:
        return self.orientations if indices is None else self.orientations[indices]

    # ---- preprocessing (experiment_pats.py:223-316): GPU passes in FP32;
    # integer or FP64 patterns become FP32, host patterns stay on the host

    def subtract_overall_background(self) -> None:
        """Subtract the scan's mean pattern from every pattern."""
        self.patterns = _pre.subtract_overall_background(self.patterns)

    def contrast_enhance_clahe(self, clip_limit: float = 40.0, tile_grid_size: int = 4, n_bins: int = 64) -> None:
        """CLAHE of every pattern (clahe_grayscale)."""
        self.patterns = clahe_grayscale(self.patterns, clip_limit=clip_limit, n_bins=n_bins,
                                        grid_shape=(tile_grid_size, tile_grid_size))

    def normalize_per_pattern(self, norm_type: str = "minmax") -> None:
        """"minmax", "zeromean" or "standard" normalisation of every pattern."""
        self.patterns = _pre.normalize_per_pattern(self.patterns, norm_type)

    def standard_clean(self) -> None:
        """Background subtraction, min-max, CLAHE, min-max, fused into one
        pass over the patterns after the mean pattern."""
        self.patterns = _pre.standard_clean(self.patterns)

    def do_nlpar(self, k_rad: int = 3, coeff: float = 0.375) -> None:
        """Non-local pattern averaging over the 2D scan."""
        if len(self.spatial_shape) != 2:
            raise ValueError(f"NLPAR only supported for 2D EBSD scans, got {self.spatial_shape}")
        self.patterns = nlpar(self.patterns.reshape(tuple(self.spatial_shape) + tuple(self.pattern_shape)),
                              k_rad=k_rad, coeff=coeff).reshape(-1, *self.pattern_shape)

    def get_patterns(self, indices: Tensor, binning: int):
        """Patterns at `indices`, b x b average pooled (experiment_pats.py:318-346)."""
        pats = self.patterns[indices]
        if binning > 1:
            if pats.device.type == "cuda":
                pats = kernels.avg_pool(pats.contiguous().float(), int(binning))
            else:
                pats = torch.nn.functional.avg_pool2d(pats, binning)
        return pats

    def get_indices_per_phase(self) -> List[Tensor]:
        if self.phases is None:
            raise ValueError("Phases must be indexed before retrieving indices per phase.")
        return [torch.nonzero(self.phases == i, as_tuple=False).squeeze()
                for i in range(int(self.phases.max().item()) + 1)]

    def set_raw_indexing_results(self, quaternions: Tensor, metrics: Tensor, phase_id: int):
        """Store one phase's top-k results (experiment_pats.py:367-385)."""
        if not hasattr(self, "raw_indexing_results"):
            self.raw_indexing_results = {phase_id: (quaternions, metrics)}
        else:
            self.raw_indexing_results[phase_id] = (quaternions, metrics)

    def combine_indexing_results(self, higher_is_better: bool) -> None:
        """Best top-1 result over phases (experiment_pats.py:387-451). With
        several phases the reference raises a TypeError (it calls torch.full
        with an int size); this version implements the intended selection."""
        if not hasattr(self, "raw_indexing_results"):
            raise ValueError("Raw indexing results must be set before combining.")
        res = self.raw_indexing_results
        first_q = next(iter(res.values()))[0]
        dev = first_q.device
        if len(res) > 1:
            fill = float("-inf") if higher_is_better else float("inf")
            best = torch.full((self.n_patterns,), fill, device=dev)
            phase_ids = torch.full((self.n_patterns,), 255, dtype=torch.uint8, device=dev)
            ori = torch.zeros((self.n_patterns, 4), device=dev)
            for pid, (q, m) in res.items():
                m0 = m[:, 0].float()
                sel = (m0 > best) if higher_is_better else (m0 < best)
                best[sel] = m0[sel]
                phase_ids[sel] = pid
                ori[sel] = q[sel, 0].to(ori.dtype)
            self.phases, self.orientations, self.best_metrics = phase_ids, ori, best
        else:
            pid = next(iter(res.keys()))
            self.phases = torch.full((self.n_patterns,), fill_value=pid, dtype=torch.uint8, device=dev)
            self.orientations = res[pid][0][:, 0]
            self.best_metrics = res[pid][1][:, 0]
