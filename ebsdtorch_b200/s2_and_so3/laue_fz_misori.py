"""Disorientation angle (mirror of ebsdtorch/s2_and_so3/laue_fz_misori.py:148-203)."""

from __future__ import annotations

import torch
from torch import Tensor

from .. import kernels


def disori_angle_laue(quats1: Tensor, quats2: Tensor, laue_id_1: int, laue_id_2: int) -> Tensor:
    """Disorientation angle in radians between orientations of one phase."""
    if quats1.shape != quats2.shape:
        raise ValueError(
            f"quats1 and quats2 must have the same data shape, but got {quats1.shape} and {quats2.shape}")
    if laue_id_1 != laue_id_2:
        raise NotImplementedError("disorientation between two different Laue groups is not implemented")
    q1 = quats1.reshape(-1, 4).float().contiguous()
    q2 = quats2.reshape(-1, 4).float().contiguous()
    return kernels.disori_angle(q1, q2, laue_id_1).view(quats1.shape[:-1])
