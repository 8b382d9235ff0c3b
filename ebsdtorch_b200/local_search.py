"""Learned-proposal dictionary indexing: CNN proposals, local search in the
global dictionary around each proposal, and plain DI as the fallback.

Per phase the dictionary is built exactly as for plain DI (same grid, same
permutation, same projected rows) and kept resident; a proposal within the
search radius of the plain-DI answer therefore reproduces that answer. A
pattern whose best local score falls below `fallback_ratio` times the map's
median local score (or that finds no candidate) is re-indexed by full plain
DI against the same resident rows. No counterpart in the reference.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass
from typing import Optional

import torch

from . import kernels
from ._capi import call, ptr
from .engine import RowSet, Searcher, SearchConfig
from .kernels import LP_DTYPES, TILE_D, RowBuffers
from .s2_and_so3.laue_fz_ori import edge_length_for_resolution


def _stream(dev) -> int:
    return torch.cuda.current_stream(dev).cuda_stream


class PhaseDictionary:
    """One phase's dictionary resident on the GPU: permuted FZ quaternions,
    the cubochoric cell -> row map, zero-mean FP32 rows and unit
    low-precision rows + norms (the plain-DI layout)."""

    def __init__(self, master_pattern: torch.Tensor, rays_soa: torch.Tensor, laue_id: int, resolution_deg: float,
                 precision: str = "bf16", permute: bool = True):
        dev = master_pattern.device
        self.laue = int(laue_id)
        self.edge = edge_length_for_resolution(laue_id, resolution_deg)
        q, _, cells = kernels.grid_fz(self.laue, self.edge, dev, want_cells=True)
        n = q.shape[0]
        perm = torch.randperm(n).to(dev) if permute else None
        self.quats = kernels.gather_rows(q, perm) if permute else q
        self.cell_to_row = torch.empty(self.edge ** 3, dtype=torch.int32, device=dev)
        call("ebsd_cell_to_row", ptr(cells), ptr(perm), n, self.edge ** 3, ptr(self.cell_to_row), _stream(dev))
        self.n_pix = rays_soa.shape[1]
        self.rows = RowSet(n, self.n_pix, TILE_D, LP_DTYPES[precision], True, dev)
        kernels.project(master_pattern, rays_soa, self.quats, self.rows.buffers(0, n))
        self.n = n

    def default_radius(self, max_angle_deg: float) -> int:
        """Grid cells that contain every dictionary point within the angle
        (measured: within 3 deg needs 4 cells on the 0.5 deg, edge-199 grid)."""
        return min(8, int(math.ceil(max_angle_deg * (4.0 / 3.0) * self.edge / 199.0)) + 1)


def local_search(pd: PhaseDictionary, q_f32: torch.Tensor, proposals: torch.Tensor, max_angle_deg: float = 3.0,
                 radius_cells: Optional[int] = None, max_candidates: int = 1024):
    """Best dictionary row near each proposal: (index int64, exact FP32 score,
    candidate count int32), -1 / -inf when no candidate lies in the radius."""
    Q = q_f32.shape[0]
    dev = q_f32.device
    idx = torch.empty(Q, dtype=torch.int64, device=dev)
    score = torch.empty(Q, dtype=torch.float32, device=dev)
    ncand = torch.empty(Q, dtype=torch.int32, device=dev)
    r = pd.default_radius(max_angle_deg) if radius_cells is None else radius_cells
    call("ebsd_local_search", ptr(q_f32), q_f32.stride(0), Q, ptr(proposals.contiguous()), pd.laue, pd.edge,
         ptr(pd.cell_to_row), ptr(pd.quats), ptr(pd.rows.f32), pd.rows.f32.stride(0), pd.n, pd.n_pix, r,
         math.radians(max_angle_deg), max_candidates, ptr(idx), ptr(score), ptr(ncand), _stream(dev))
    return idx, score, ncand


@dataclass
class LearnedStats:
    n_patterns: int
    n_fallback: int
    median_local_score: float
    mean_candidates: float
    seconds: dict


def learned_dictionary_index(master_pattern, geometry, experiment_patterns, model, dictionary_resolution_degrees=0.5,
                             max_angle_deg: float = 8.0, coarse_resolution_deg: Optional[float] = 2.0,
                             fallback_ratio: float = 0.9, batch: int = 1024, precision: str = "bf16",
                             rescore_k: int = 32, device=None,
                             phase_dictionary: Optional[PhaseDictionary] = None) -> LearnedStats:
    """Top-1 indexing of one phase by learned proposal + local search with
    plain-DI fallback. With coarse_resolution_deg the search runs in two
    stages: within max_angle_deg of the proposal on a coarse dictionary, then
    within 1.5 coarse spacings of the coarse winner on the full-resolution
    dictionary (without it: one stage within max_angle_deg). Writes
    raw_indexing_results / orientations like dictionary_index_orientations and
    returns timing and fallback counts."""
    from .ebsd.indexing import _device, _master_pattern_tensor, _unit_rays_soa

    sec = {}
    dev = _device(master_pattern, device)
    t0 = time.perf_counter()
    rays = _unit_rays_soa(geometry, 1, None, dev)
    mp_t = _master_pattern_tensor(master_pattern, 1, dev)
    pd = phase_dictionary or PhaseDictionary(mp_t, rays, master_pattern.laue_group, dictionary_resolution_degrees,
                                             precision)
    coarse = None
    if coarse_resolution_deg is not None and coarse_resolution_deg > dictionary_resolution_degrees:
        coarse = PhaseDictionary(mp_t, rays, master_pattern.laue_group, coarse_resolution_deg, precision,
                                 permute=False)
    torch.cuda.synchronize(dev)
    sec["dictionary"] = time.perf_counter() - t0
    pats = experiment_patterns.patterns
    Q = pats.shape[0]
    H, W = pats.shape[-2:]
    P = H * W
    if (H, W) != (model.H, model.W):
        raise ValueError(f"the network was built for {model.H}x{model.W} patterns, got {H}x{W}")
    t0 = time.perf_counter()
    q_f32 = torch.empty((Q, P), dtype=torch.float32, device=dev)
    q_norm = torch.empty(Q, dtype=torch.float32, device=dev)
    proposals = torch.empty((Q, 4), dtype=torch.float32, device=dev)
    for b0 in range(0, Q, batch):
        b1 = min(Q, b0 + batch)
        chunk = pats[b0:b1].to(dev, non_blocking=True).float().contiguous()
        kernels.prep_patterns(chunk, RowBuffers(f32=q_f32[b0:b1], norm=q_norm[b0:b1]))
        nb = b1 - b0
        nb_pad = -(-nb // 128) * 128
        x = torch.zeros((nb_pad, H, W), dtype=torch.float32, device=dev)
        x[:nb] = (q_f32[b0:b1] * (math.sqrt(P) / q_norm[b0:b1].clamp_min(1e-12))[:, None]).view(nb, H, W)
        proposals[b0:b1] = model.predict_quaternions(x)[:nb]
    torch.cuda.synchronize(dev)
    sec["proposals"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    if coarse is not None:
        cidx, _, _ = local_search(coarse, q_f32, proposals, max_angle_deg)
        found = cidx >= 0
        refined = torch.where(found[:, None], kernels.gather_rows(coarse.quats, cidx.clamp_min(0)), proposals)
        idx, score, ncand = local_search(pd, q_f32, refined.contiguous(), 1.5 * coarse_resolution_deg)
        idx = torch.where(found, idx, torch.full_like(idx, -1))
    else:
        idx, score, ncand = local_search(pd, q_f32, proposals, max_angle_deg)
    valid = idx >= 0
    med = torch.median(score[valid]) if bool(valid.any()) else torch.tensor(0.0, device=dev)
    fb = (~valid) | (score < fallback_ratio * med)
    fb_rows = torch.nonzero(fb).reshape(-1)
    torch.cuda.synchronize(dev)
    sec["local_search"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    n_fb = int(fb_rows.numel())
    if n_fb:
        sub = kernels.gather_rows(q_f32, fb_rows)

        def fill_q(a, b, bufs):
            kernels.prep_patterns(sub[a:b].reshape(b - a, 1, P), bufs, subtract_mean=False)

        cfg = SearchConfig(precision=precision, rescore_k=rescore_k)
        s = Searcher(pd.n, n_fb, P, 1, cfg, dev)
        fi, fv = s.run(None, fill_q, resident=pd.rows)
        idx[fb_rows] = fi[:, 0]
        score[fb_rows] = fv[:, 0]
    torch.cuda.synchronize(dev)
    sec["fallback"] = time.perf_counter() - t0
    quats = kernels.gather_rows(pd.quats, idx).reshape(Q, 1, 4)
    experiment_patterns.set_raw_indexing_results(quats, score.reshape(Q, 1), phase_id=0)
    experiment_patterns.raw_indexing_indices = {0: idx.reshape(Q, 1)}
    experiment_patterns.dictionaries = {0: pd.quats}
    experiment_patterns.proposals = proposals
    experiment_patterns.combine_indexing_results(higher_is_better=True)
    return LearnedStats(Q, n_fb, float(med), float(ncand.float().mean()), sec)
