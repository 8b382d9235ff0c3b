"""Master-pattern container (mirror of ebsdtorch/ebsd/master_pattern.py).

Holds the (H, 2W) side-by-side modified-Lambert master pattern (northern
hemisphere left, southern right; master_pattern.py:22-92) and its Laue group.
``interpolate`` and ``bin`` run on the CUDA kernels of this package.
"""

from __future__ import annotations

from typing import Optional, Tuple, Union

import torch
from torch import Tensor
from torch.nn import Module

from .. import kernels
from ..utils.symmetry_classes import point_group_to_laue, space_group_to_laue


class MasterPattern(Module):
    """Constructor arguments as master_pattern.py:40-92: a 2-D tensor (or a
    (north, south) tuple concatenated along the last dimension) and exactly
    one of laue_group, point_group or space_group."""

    def __init__(
        self,
        master_pattern: Union[Tensor, Tuple[Tensor, Tensor]],
        laue_group: Optional[int] = None,
        point_group: Optional[str] = None,
        space_group: Optional[int] = None,
    ):
        super().__init__()
        given = [v is not None for v in (laue_group, point_group, space_group)]
        if not any(given):
            raise ValueError("At least one of laue_groups, point_groups, or space_groups must be provided")
        if sum(given) > 1:
            raise ValueError("Only one of laue_groups, point_groups, or space_groups should be provided")
        if isinstance(master_pattern, tuple):
            if len(master_pattern[0].shape) != 2 or len(master_pattern[1].shape) != 2:
                raise ValueError("Both tensors in 'master_pattern' must be 2D tensors when provided as a tuple")
            master_pattern = torch.cat(master_pattern, dim=-1)
        if len(master_pattern.shape) != 2:
            raise ValueError(f"'master_pattern' must be a 2D tensor, got shape {master_pattern.shape}")
        self.register_buffer("master_pattern", master_pattern)
        if laue_group is not None:
            self.laue_group = int(laue_group)
        elif point_group is not None:
            self.laue_group = point_group_to_laue(point_group)
        else:
            self.laue_group = space_group_to_laue(space_group)
        self.master_pattern_binned = None

    def _apply(self, fn, *args, **kwargs):
        out = super()._apply(fn, *args, **kwargs)
        if self.master_pattern_binned is not None:
            self.master_pattern_binned = fn(self.master_pattern_binned)
        return out

    def bin(self, binning_factor: int) -> None:
        """b x b average pooled copy in ``master_pattern_binned``
        (master_pattern.py:94-113)."""
        self.master_pattern_binned = kernels.avg_pool(self.master_pattern.contiguous().float(), int(binning_factor))

    def normalize(self, norm_type: str) -> None:
        """In-place normalisation (master_pattern.py:115-139)."""
        mp = self.master_pattern
        if norm_type == "minmax":
            lo, hi = torch.min(mp), torch.max(mp)
            mp -= lo
            mp /= 1e-4 + hi - lo
        elif norm_type == "zeromean":
            mp -= torch.mean(mp)
        elif norm_type == "standard":
            mp -= torch.mean(mp)
            mp /= torch.std(mp)
        else:
            raise ValueError(
                f"Invalid normalization method. Got {norm_type} but expected 'minmax', 'zeromean', or 'standard'.")

    def interpolate(self, coords_3D: Tensor, mode: str = "bilinear", padding_mode: str = "border",
                    align_corners: bool = False, normalize_coords: bool = True, virtual_binning: int = 1) -> Tensor:
        """Master-pattern values at (..., 3) sphere points (master_pattern.py:141-209).
        Supported: bilinear, border padding, align_corners=False (the
        dictionary-indexing settings)."""
        if mode != "bilinear" or padding_mode != "border" or align_corners:
            raise NotImplementedError("only mode='bilinear', padding_mode='border', align_corners=False are supported")
        if virtual_binning > 1:
            if self.master_pattern_binned is None:
                self.bin(virtual_binning)
            mp = self.master_pattern_binned
        else:
            mp = self.master_pattern
        xyz = coords_3D.reshape(-1, 3).float().contiguous()
        out = kernels.sample_master_pattern(mp.contiguous().float(), xyz, normalize_coords)
        return out.view(coords_3D.shape[:-1])
