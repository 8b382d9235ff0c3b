"""Detector <-> sample geometry (mirror of ebsdtorch/ebsd/geometry.py).

Only what dictionary indexing consumes is provided: the Bruker pattern-centre
convention (geometry.py:31-92), the optional SE(3) correction
(geometry.py:257-280) and the sample-frame pixel coordinates
(``get_coords_sample_frame``, geometry.py:422-503). These are a one-time
(P, 3) set-up computed in float64 on the host and returned as a tensor on the
module's device; the per-orientation work happens in the CUDA projector.
"""

from __future__ import annotations

import math
from typing import Optional, Tuple

import numpy as np
import torch
from torch import Tensor
from torch.nn import Module


def bruker_geometry_to_SE3(pattern_center, primary_tilt_deg: float, secondary_tilt_deg: float,
                           detector_shape: Tuple[int, int]):
    """Rotation (3, 3) and translation (3,) of the detector-to-sample map for a
    Bruker pattern centre (geometry.py:31-92), float64 numpy."""
    pcx, pcy, pcz = (float(v) for v in pattern_center)
    rows, cols = float(detector_shape[0]), float(detector_shape[1])
    d, sx = math.radians(primary_tilt_deg), math.radians(secondary_tilt_deg)
    sd, cd, ss, cs = math.sin(d), math.cos(d), math.sin(sx), math.cos(sx)
    rot = np.array([[-sd, -ss * cd, cs * cd], [0.0, cs, ss], [-cd, ss * sd, -sd * cs]])
    t = np.array([
        pcx * cols * ss * cd + pcy * rows * sd + pcz * rows * cs * cd - ss * cd / 2 - sd / 2,
        -cols * pcx * cs + pcz * rows * ss + cs / 2,
        -cols * pcx * ss * sd + pcy * rows * cd - pcz * rows * sd * cs + ss * sd / 2 - cd / 2,
    ])
    return rot, t


def se3_exp(vec) -> np.ndarray:
    """4x4 matrix exponential of an se(3) vector (rx, ry, rz, tx, ty, tz),
    closed form (Rodrigues for the rotation, V matrix for the translation);
    the same map as lie_algebra/se3.py:363-382."""
    v = np.asarray(vec, dtype=np.float64).reshape(6)
    w, tau = v[:3], v[3:]
    th = float(np.linalg.norm(w))
    K = np.array([[0.0, -w[2], w[1]], [w[2], 0.0, -w[0]], [-w[1], w[0], 0.0]])
    K2 = K @ K
    if th > 1e-3:
        a, b, c = math.sin(th) / th, (1 - math.cos(th)) / th**2, (th - math.sin(th)) / th**3
    else:
        a, b, c = 1 - th**2 / 6, 0.5 - th**2 / 24, 1 / 6 - th**2 / 120
    R = np.eye(3) + a * K + b * K2
    V = np.eye(3) + b * K + c * K2
    out = np.eye(4)
    out[:3, :3] = R
    out[:3, 3] = V @ tau
    return out


class EBSDGeometry(Module):
    """Detector geometry with the reference's constructor
    (geometry.py:139-229): detector_shape (H, W), tilts_degrees
    (sample x tilt, sample y tilt, detector tilt), proj_center (Bruker),
    optional se3_vector and optimisation masks."""

    def __init__(
        self,
        detector_shape: Tuple[int, int],
        tilts_degrees: Optional[Tuple[float, float, float]] = (0.0, 70.0, 0.0),
        proj_center: Optional[Tuple[float, float, float]] = (0.5, 0.5, 0.5),
        se3_vector: Optional[Tensor] = None,
        opt_rots: Tuple[bool, bool, bool] = (False, False, False),
        opt_shifts: Tuple[bool, bool, bool] = (False, False, False),
    ):
        super().__init__()
        self.detector_shape = tuple(int(v) for v in detector_shape)
        self.tilts_degrees = tuple(float(v) for v in tilts_degrees)
        self.proj_center = tuple(float(v) for v in proj_center)
        rot, t = bruker_geometry_to_SE3(self.proj_center, self.tilts_degrees[2] - self.tilts_degrees[1],
                                        self.tilts_degrees[0], self.detector_shape)
        pc = np.eye(4)
        pc[:3, :3], pc[:3, 3] = rot, t
        self.register_buffer("pc_SE3_matrix", torch.from_numpy(pc).float().view(1, 4, 4))
        vec = torch.zeros(1, 6) if se3_vector is None else se3_vector.detach().reshape(1, 6).float()
        self.se3_vector = torch.nn.Parameter(vec)
        self.register_buffer("mask", torch.tensor(list(opt_rots) + list(opt_shifts), dtype=torch.bool))
        self._pc64 = pc

    def set_optimizable_se3_params(self, opt_rots=None, opt_shifts=None):
        if opt_rots is not None:
            self.mask[:3] = torch.tensor(opt_rots, dtype=torch.bool)
        if opt_shifts is not None:
            self.mask[3:] = torch.tensor(opt_shifts, dtype=torch.bool)

    def _detector2sample64(self) -> np.ndarray:
        vec = (self.se3_vector.detach().double().cpu() * self.mask.cpu().double()).numpy()
        return self._pc64 @ se3_exp(vec)

    def get_detector2sample(self) -> Tuple[Tensor, Tensor]:
        m = torch.from_numpy(self._detector2sample64()).float().to(self.pc_SE3_matrix.device)
        return m[:3, :3], m[:3, 3]

    def get_coords_sample_frame(self, binning: Tuple[int, int], dtype: Optional[torch.dtype] = torch.float32
                                ) -> Tensor:
        """Sample-frame coordinates (P, 3) of the (binned) detector pixels,
        un-normalised, row-major over (i, j) (geometry.py:422-503)."""
        h, w = self.detector_shape
        if h % binning[0] != 0:
            raise ValueError(
                f"A height binning of {binning[0]} does not evenly divide the detector height of {h}.")
        if w % binning[1] != 0:
            raise ValueError(
                f"A width binning of {binning[1]} does not evenly divide the detector width of {w}.")
        bh, bw = h // binning[0], w // binning[1]
        ii = np.linspace(0.5 * (binning[0] - 1), h - 0.5 * (binning[0] - 1), bh)
        jj = np.linspace(0.5 * (binning[1] - 1), w - 0.5 * (binning[1] - 1), bw)
        pix = np.stack(np.meshgrid(ii, jj, indexing="ij"), axis=-1).reshape(-1, 2)
        m = self._detector2sample64()
        coords = pix @ m[:3, :2].T + m[:3, 3]
        return torch.from_numpy(coords).to(dtype=dtype, device=self.pc_SE3_matrix.device)

    def unit_rays_soa(self, binning: int, signal_mask: Optional[Tensor] = None, device=None) -> Tensor:
        """Unit rays of the (masked) binned pixels as a (3, P') float32 tensor,
        the projector's input layout (normalised in float64, indexing.py:106)."""
        h, w = self.detector_shape
        coords = self.get_coords_sample_frame((binning, binning), dtype=torch.float64).cpu()
        coords = coords / coords.norm(dim=-1, keepdim=True)
        if signal_mask is not None:
            coords = coords[signal_mask.reshape(-1).cpu().bool()]
        dev = self.pc_SE3_matrix.device if device is None else device
        return coords.t().contiguous().float().to(dev)
