"""Orientation fundamental-zone dictionaries (mirror of
ebsdtorch/s2_and_so3/laue_fz_ori.py:486-557), generated by the FP64 CUDA grid
kernel.

Permutation convention: like the reference, the FZ points are shuffled with
``torch.randperm(n)`` drawn from the global CPU generator, so seeding torch
before a call reproduces the reference's dictionary order exactly.
"""

from __future__ import annotations

import torch
from torch import Tensor

from .. import kernels

LAUE_MULTS = [2, 4, 8, 8, 16, 6, 12, 12, 24, 24, 48]


def get_laue_mult(laue_group: int) -> int:
    """Group order including inversion (laue_generators.py:14-51)."""
    if not 1 <= int(laue_group) <= 11:
        raise ValueError(f"Laue group {laue_group} is not supported")
    return LAUE_MULTS[int(laue_group) - 1]


def edge_length_for_resolution(laue_id: int, angular_resolution_deg: float) -> int:
    """Cubochoric edge length of the reference's empirical resolution fit
    (laue_fz_ori.py:540-547)."""
    n_so3 = (2 * 131.97049 / (angular_resolution_deg - 0.03732) + 1) ** 3
    return int((n_so3 / (0.5 * get_laue_mult(laue_id))) ** (1.0 / 3.0) + 1.0)


def _finish(q: Tensor, permute: bool) -> Tensor:
    if permute and q.shape[0] > 1:
        perm = torch.randperm(q.shape[0]).to(q.device)
        q = kernels.gather_rows(q, perm)
    return q


def sample_ori_fz_laue_angle(laue_id: int, angular_resolution_deg: float, device: torch.device,
                             permute: bool = True) -> Tensor:
    """(n, 4) float32 FZ quaternions (w, x, y, z), w >= 0, for a target
    resolution (laue_fz_ori.py:516-557)."""
    get_laue_mult(laue_id)
    edge = edge_length_for_resolution(laue_id, angular_resolution_deg)
    q, _ = kernels.grid_fz(laue_id, edge, device)
    return _finish(q, permute)


def sample_ori_fz_laue(laue_id: int, target_n_samples: int, device: torch.device, permute: bool = True) -> Tensor:
    """FZ quaternions for a target sample count (laue_fz_ori.py:486-513)."""
    edge = int((target_n_samples * 0.5 * get_laue_mult(laue_id)) ** (1.0 / 3.0))
    q, _ = kernels.grid_fz(laue_id, edge, device)
    return _finish(q, permute)
