"""Orientation grid refinement after dictionary indexing (mirror of
ebsdtorch/ebsd/refining.py:13-244).

`orientation_grid_refinement` keeps the reference's signature and behaviour:
per phase, every pattern's orientation is moved over `n_iter` iterations to
the best point of a local cubochoric grid around it, the grid shrinking by
`shrink_factor` for patterns whose centre stayed best; orientations are
updated in place and the per-iteration best dot products are returned. All
iterations of all patterns of a phase run in one kernel launch
(`ebsd_refine_grid`: one CTA per pattern, simulations generated on the fly,
no dictionary), instead of the reference's batches of simulated pattern
tensors.

Differences, by design: scores are FP32 (`match_dtype`, FP16 by default in
the reference, is accepted and ignored); `batch_size` is accepted and ignored
(a launch covers a phase in chunks of `query_chunk` patterns).
`fz_reduction="left"` (keyword-only) moves candidates to the fundamental zone
by the left product g q, which keeps the simulated pattern; the default
"reference" reproduces the reference's right product q g (laue_fz_ori.py:
36-81), which changes the simulated pattern of candidates that leave the
fundamental zone.
"""

from __future__ import annotations

import math
from typing import List, Union

import torch
from torch import Tensor

from .. import kernels
from .._capi import call, ptr
from ..kernels import RowBuffers
from .indexing import _device, _master_pattern_tensor
from .._device import on_data_device


def get_local_orientation_grid(semi_edge_in_degrees: float, kernel_radius_in_steps: int,
                               axial_grid_dimension: int = 3) -> Tensor:
    """(G, 3) cubochoric offsets of the local grid (refining.py:13-68): a
    (2r + 1)^3 cube of semi-edge `semi_edge_in_degrees` * pi^(2/3) / 360,
    all points (3), the points with a zero coordinate (2) or on the axes (1)."""
    semi = semi_edge_in_degrees * math.pi ** (2.0 / 3.0) / 360.0
    c = torch.linspace(-semi, semi, 2 * kernel_radius_in_steps + 1)
    cu = torch.stack(torch.meshgrid(c, c, c, indexing="ij"), dim=-1).reshape(-1, 3)
    if axial_grid_dimension == 3:
        pass
    elif axial_grid_dimension == 2:
        cu = cu[torch.any(cu == 0, dim=-1)]
    elif axial_grid_dimension == 1:
        cu = cu[torch.sum(cu == 0, dim=-1) >= 2]
    else:
        raise ValueError("axial_grid_dimension must be 1, 2, or 3.")
    return cu


@on_data_device
def orientation_grid_refinement(
    master_patterns,
    geometry,
    experiment_patterns,
    grid_semi_edge_in_degrees: float,
    batch_size: int,
    virtual_binning: int = 1,
    n_iter: int = 3,
    axial_grid_dimension: int = 3,
    kernel_radius_in_steps: int = 1,
    shrink_factor: float = 0.5,
    average_pattern_center: bool = True,
    match_dtype: torch.dtype = torch.float16,
    *,
    fz_reduction: str = "reference",
    device=None,
    query_chunk: int = 65536,
) -> List[Tensor]:
    """Refine the orientations of indexed patterns in place (refining.py:71-244).
    Returns one (n_patterns, n_iter) tensor of best dot products per phase."""
    if getattr(experiment_patterns, "orientations", None) is None:
        raise ValueError("The experiment patterns must be indexed before refinement.")
    if fz_reduction not in ("reference", "left"):
        raise ValueError("fz_reduction must be 'reference' or 'left'")
    if not isinstance(master_patterns, (list, tuple)):
        master_patterns = [master_patterns]
    b = int(virtual_binning)
    grid_cpu = get_local_orientation_grid(grid_semi_edge_in_degrees, kernel_radius_in_steps, axial_grid_dimension)
    n_grid = grid_cpu.shape[0]
    coords = geometry.get_coords_sample_frame(binning=(b, b)).detach().reshape(-1, 3).double().cpu()
    offsets_all = None
    if average_pattern_center:
        coords = coords / coords.norm(dim=-1, keepdim=True)
    else:
        offsets_all = experiment_patterns.get_spatial_coords().detach().float()
    n_pix = coords.shape[0]
    phase_indices = experiment_patterns.get_indices_per_phase()
    all_dots = []
    for i, indices in enumerate(phase_indices):
        mp = master_patterns[i]
        dev = _device(mp, device)
        indices = indices.reshape(-1).to(experiment_patterns.orientations.device)
        dots = torch.zeros((experiment_patterns.n_patterns, n_iter), device=dev)
        rays = coords.t().contiguous().float().to(dev)
        mp_t = _master_pattern_tensor(mp, b, dev)
        grid = grid_cpu.float().contiguous().to(dev)
        for c0 in range(0, indices.numel(), query_chunk):
            idx = indices[c0:c0 + query_chunk]
            nq = idx.numel()
            pats = experiment_patterns.patterns[idx.to(experiment_patterns.patterns.device)]
            pats = pats.to(dev, non_blocking=pats.is_pinned())
            if pats.dtype not in kernels.PATTERN_DTYPES:
                pats = pats.float()
            rows = torch.empty((nq, n_pix), dtype=torch.float32, device=dev)
            kernels.prep_patterns(pats.contiguous(), RowBuffers(f32=rows), binning=b)
            q = experiment_patterns.get_orientations(idx).detach().to(dev).float().contiguous()
            q_out = torch.empty_like(q)
            d_out = torch.empty((nq, n_iter), dtype=torch.float32, device=dev)
            off = offsets_all[idx.to(offsets_all.device)].to(dev).contiguous() if offsets_all is not None else None
            call("ebsd_refine_grid", ptr(mp_t), mp_t.shape[0], mp_t.shape[1], ptr(rays), n_pix, ptr(off), ptr(rows),
                 rows.stride(0), ptr(q), nq, ptr(grid), n_grid, int(mp.laue_group), int(fz_reduction == "left"),
                 int(n_iter), float(shrink_factor), ptr(q_out), ptr(d_out),
                 torch.cuda.current_stream(dev).cuda_stream)
            dots[idx.to(dev)] = d_out
            experiment_patterns.set_orientations(q_out.to(experiment_patterns.orientations.device), idx)
        all_dots.append(dots)
    return all_dots
