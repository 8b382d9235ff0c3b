"""Tensor-level wrappers over the C-ABI kernels.

Each function checks devices, dtypes and layouts, allocates outputs with
PyTorch (the library itself allocates nothing), passes raw pointers plus the
current CUDA stream to ``libebsd_b200.so`` and returns tensors. All work is
stream-ordered on ``torch.cuda.current_stream()``; nothing here synchronises
except ``grid_fz`` (it must read the fundamental-zone point count).
"""

from __future__ import annotations

from typing import Optional

import torch

from . import _capi
from ._capi import DT_BF16, DT_E4M3, call, ptr

LP_DTYPES = {"bf16": DT_BF16, "fp8": DT_E4M3}
LP_TORCH = {DT_BF16: torch.bfloat16, DT_E4M3: torch.float8_e4m3fn}
LP_KMULT = {DT_BF16: 64, DT_E4M3: 128}
TILE_Q, TILE_D = 128, 256


def round_up(n: int, m: int) -> int:
    return (n + m - 1) // m * m


def _stream(dev: torch.device) -> int:
    return torch.cuda.current_stream(dev).cuda_stream


def _cuda(t: torch.Tensor, name: str, dtype=None, contiguous=True) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise RuntimeError(f"{name} must be a CUDA tensor (ebsdtorch_b200 runs on sm_100 GPUs only)")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if contiguous and not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


# ---------------------------------------------------------------- A1/A2 grid


def grid_fz(laue_id: int, edge_length: int, device, want_f64: bool = False, want_cells: bool = False):
    """FZ quaternions of the edge^3 cubochoric grid in reference order.
    Returns (q_f32 (n, 4), q_f64 (n, 4) or None), plus the int32 grid cell of
    each point when want_cells."""
    device = torch.device(device)
    lib = _capi.load()
    nbytes = int(lib.ebsd_grid_workspace_bytes(int(edge_length)))
    if nbytes == 0:
        raise ValueError(f"grid edge length {edge_length} must be positive")
    ws = torch.empty(nbytes, dtype=torch.uint8, device=device)
    cnt = torch.zeros(1, dtype=torch.int64, device=device)
    s = _stream(device)
    call("ebsd_grid_fz_count", int(laue_id), int(edge_length), ptr(ws), nbytes, ptr(cnt), s)
    n = int(cnt.item())
    q32 = torch.empty((n, 4), dtype=torch.float32, device=device)
    q64 = torch.empty((n, 4), dtype=torch.float64, device=device) if want_f64 else None
    cells = torch.empty(n, dtype=torch.int32, device=device) if want_cells else None
    if n:
        call("ebsd_grid_fz_write", int(laue_id), int(edge_length), ptr(ws), nbytes, ptr(q32), ptr(q64), ptr(cells), s)
    if want_cells:
        return q32, q64, cells
    return q32, q64


def gather_rows(src: torch.Tensor, index: torch.Tensor) -> torch.Tensor:
    """out[i] = src[index[i]] for float32 rows."""
    _cuda(src, "src", torch.float32)
    _cuda(index, "index", torch.int64)
    src2 = src.reshape(src.shape[0], -1)
    out = torch.empty((index.numel(), src2.shape[1]), dtype=torch.float32, device=src.device)
    call("ebsd_gather_rows", ptr(src2), src2.shape[0], src2.shape[1], ptr(index), index.numel(), ptr(out),
         _stream(src.device))
    return out.reshape((index.numel(),) + tuple(src.shape[1:]))


# ------------------------------------------------------- A4-A8 row producers


class RowBuffers:
    """Destination of the projector / pattern preparation for a block of rows.
    Any field may be None (not written)."""

    def __init__(self, f32=None, lp=None, lp_dtype=DT_BF16, norm=None, lp_scale=None):
        self.f32, self.lp, self.lp_dtype, self.norm, self.lp_scale = f32, lp, lp_dtype, norm, lp_scale

    def args(self, n_pix: int):
        ld_f32 = self.f32.stride(0) if self.f32 is not None else 0
        ld_lp = self.lp.stride(0) if self.lp is not None else 0
        return (ptr(self.f32), ld_f32, ptr(self.lp), self.lp_dtype, ld_lp, ptr(self.norm), ptr(self.lp_scale))


def project(master_pattern: torch.Tensor, rays_soa: torch.Tensor, quats: torch.Tensor, out: RowBuffers,
            subtract_mean: bool = True) -> None:
    """K1: simulated dictionary rows for `quats` into `out` (row i <- quats[i])."""
    _cuda(master_pattern, "master_pattern", torch.float32)
    _cuda(rays_soa, "rays_soa", torch.float32)
    _cuda(quats, "quats", torch.float32)
    if rays_soa.dim() != 2 or rays_soa.shape[0] != 3:
        raise ValueError("rays_soa must be (3, n_pix)")
    n_pix = rays_soa.shape[1]
    call("ebsd_project_dictionary", ptr(master_pattern), master_pattern.shape[0], master_pattern.shape[1],
         ptr(rays_soa), n_pix, ptr(quats), quats.shape[0], int(bool(subtract_mean)), *out.args(n_pix),
         _stream(quats.device))


PATTERN_DTYPES = {torch.float32: 0, torch.uint16: 1, torch.uint8: 2, torch.float16: 3}


def prep_patterns(patterns: torch.Tensor, out: RowBuffers, binning: int = 1,
                  pix_index: Optional[torch.Tensor] = None, n_pix: Optional[int] = None,
                  subtract_mean: bool = True) -> None:
    """K2: (n, H, W) patterns (fp32, uint16 / uint8 counts or fp16; row stride
    may exceed H*W) -> rows in `out`."""
    if patterns.dtype not in PATTERN_DTYPES:
        raise TypeError(f"patterns must be float32, uint16, uint8 or float16, got {patterns.dtype}")
    _cuda(patterns, "patterns", patterns.dtype, contiguous=False)
    if patterns.dim() == 2:
        patterns = patterns.unsqueeze(1)
    n, h, w = patterns.shape
    if patterns.stride(2) != 1 or patterns.stride(1) != w:
        raise ValueError("each pattern must be a contiguous (H, W) image")
    if pix_index is not None:
        _cuda(pix_index, "pix_index", torch.int32)
        n_pix = pix_index.numel()
    elif n_pix is None:
        n_pix = (h // binning) * (w // binning)
    call("ebsd_prep_patterns_typed", ptr(patterns), PATTERN_DTYPES[patterns.dtype], n, h, w, patterns.stride(0),
         int(binning), ptr(pix_index), int(n_pix), int(bool(subtract_mean)), *out.args(n_pix),
         _stream(patterns.device))


def sample_master_pattern(master_pattern: torch.Tensor, xyz: torch.Tensor, normalize: bool) -> torch.Tensor:
    _cuda(master_pattern, "master_pattern", torch.float32)
    _cuda(xyz, "coords", torch.float32)
    out = torch.empty(xyz.shape[:-1], dtype=torch.float32, device=xyz.device)
    call("ebsd_sample_master_pattern", ptr(master_pattern), master_pattern.shape[0], master_pattern.shape[1],
         ptr(xyz), out.numel(), int(bool(normalize)), ptr(out), _stream(xyz.device))
    return out


def avg_pool(x: torch.Tensor, binning: int) -> torch.Tensor:
    """b x b average pooling over the last two axes."""
    _cuda(x, "input", torch.float32)
    h, w = x.shape[-2:]
    lead = x.shape[:-2]
    n = x.numel() // (h * w) if x.numel() else 0
    out = torch.empty(lead + (h // binning, w // binning), dtype=torch.float32, device=x.device)
    call("ebsd_avg_pool", ptr(x), n, h, w, int(binning), ptr(out), _stream(x.device))
    return out


# ---------------------------------------------------------- A9/A10 matching


def set_match_pairs(on: bool) -> bool:
    """Run the eligible top-k matches that follow as CTA pairs (two CTAs of
    a cluster share one M = 256 tcgen05.mma.cta_group::2 and each stages half
    of every dictionary tile); returns the previous setting."""
    return bool(_capi.load().ebsd_set_match_pairs(1 if on else 0))


def match_pairs() -> bool:
    """Whether eligible top-k matches run as CTA pairs."""
    return bool(_capi.load().ebsd_set_match_pairs(-1))


def set_match_dual(mode) -> int:
    """Which eligible top-k matches that follow take two query tiles per CTA
    (two MMAs per K step share one staged dictionary tile): 0 / False none,
    1 / True all, 2 those of e4m3 rows (the default). Returns the previous
    mode."""
    return int(_capi.load().ebsd_set_match_dual(int(mode)))


def match_dual() -> int:
    """The current two-tile mode (see set_match_dual)."""
    return int(_capi.load().ebsd_set_match_dual(-1))


def takes_tile_pairs(lp_dtype: int) -> bool:
    """Whether match launches of lp_dtype rows with an even number of query
    tiles run a variant that takes the tiles two at a time."""
    mode = match_dual()
    return match_pairs() or mode == 1 or (mode == 2 and lp_dtype == DT_E4M3)


def auto_splits(n_queries_pad: int, n_dict_pad: int, lp_dtype: int = DT_BF16) -> int:
    return int(_capi.load().ebsd_match_auto_splits_typed(n_queries_pad, n_dict_pad, lp_dtype))


def match_topk(q_lp, d_lp, n_dict_valid: int, lp_dtype: int, col_scale, n_cand: int, splits: int,
               part_val, part_idx, part_slots: int, slot_base: int, index_base: int, status, tile_n: int = 0,
               max_ctas: int = 0, col_bias=None, row_scale=None) -> None:
    """K3 match; tile_n / max_ctas choose the launch shape (0, 0: 256-row
    tiles, one CTA per work unit); col_bias / row_scale add
    col_bias[d] * row_scale[q] to the scores (euclidean ranking)."""
    if tile_n == 0 and max_ctas == 0 and col_bias is None:
        call("ebsd_match_topk", ptr(q_lp), q_lp.shape[0], ptr(d_lp), d_lp.shape[0], int(n_dict_valid),
             q_lp.shape[1], lp_dtype, ptr(col_scale), int(n_cand), int(splits), ptr(part_val), ptr(part_idx),
             int(part_slots), int(slot_base), int(index_base), ptr(status), _stream(q_lp.device))
        return
    call("ebsd_match_topk_tiled", ptr(q_lp), q_lp.shape[0], ptr(d_lp), d_lp.shape[0], int(n_dict_valid),
         q_lp.shape[1], lp_dtype, ptr(col_scale), ptr(col_bias), ptr(row_scale), int(n_cand), int(splits),
         ptr(part_val), ptr(part_idx),
         int(part_slots), int(slot_base), int(index_base), int(tile_n), int(max_ctas), ptr(status),
         _stream(q_lp.device))


def manhattan_topk(q_f32, n_queries: int, n_queries_pad: int, d_f32, n_pix: int, n_cand: int, splits: int,
                   part_val, part_idx, part_slots: int, slot_base: int, index_base: int) -> None:
    """L1-distance candidates (score -L1) of FP32 query rows against FP32
    dictionary rows, in the candidate layout of match_topk."""
    _cuda(q_f32, "q_f32", torch.float32, contiguous=False)
    _cuda(d_f32, "d_f32", torch.float32, contiguous=False)
    call("ebsd_manhattan_topk", ptr(q_f32), q_f32.stride(0), int(n_queries), int(n_queries_pad), ptr(d_f32),
         d_f32.stride(0), d_f32.shape[0], int(n_pix), int(n_cand), int(splits), ptr(part_val), ptr(part_idx),
         int(part_slots), int(slot_base), int(index_base), _stream(q_f32.device))


def rescore_gate(lp_dtype: int, k_pad: int, n_pix: int) -> float:
    """Bound on |s' - s| / w for unit low-precision rows (see
    ebsd_merge_rescore_gated), or 0 (no gate) for e4m3, whose bound is too
    wide to exclude candidates. bf16 rounding of both unit rows (unit
    roundoff u = 2^-8): factor (1 + u)^2; FP32 accumulation of k_pad exact
    products, counted twice to allow truncating adders: 2 k_pad 2^-24; the
    FP32 re-score of the n_pix-term dot itself: 2 n_pix 2^-24 (so that no
    candidate left out could have ranked in by re-score rounding); 1e-6 for
    the FP32 normalisation of the rows."""
    if lp_dtype != DT_BF16:
        return 0.0
    u, u32 = 2.0 ** -8, 2.0 ** -24
    return (1.0 + u) ** 2 * (1.0 + 2.0 * k_pad * u32) - 1.0 + 2.0 * n_pix * u32 + 1e-6


def merge_rescore(part_val, part_idx, n_queries: int, part_slots: int, n_cand: int, q_f32, d_f32, d_index_base: int,
                  n_pix: int, q_norm, d_norm, q_lp_scale, similarity: int, n_rescore: int, k_out: int, run_val,
                  run_idx, out_val, out_idx, gate_rel: float = 0.0, n_rescored=None) -> None:
    """K4. gate_rel > 0 re-scores only the candidates that can reach the exact
    top k_out (rescore_gate); n_rescored: optional uint64 device counter of
    the rows re-scored."""
    call("ebsd_merge_rescore_gated", ptr(part_val), ptr(part_idx), int(n_queries), int(part_slots), int(n_cand),
         ptr(q_f32), q_f32.stride(0) if q_f32 is not None else 0, ptr(d_f32),
         d_f32.stride(0) if d_f32 is not None else 0, int(d_index_base),
         d_f32.shape[0] if d_f32 is not None else 1, int(n_pix), ptr(q_norm), ptr(d_norm),
         ptr(q_lp_scale),
         int(similarity), int(n_rescore), int(k_out), ptr(run_val), ptr(run_idx), ptr(out_val), ptr(out_idx),
         float(gate_rel), ptr(n_rescored), _stream(part_val.device))


# ------------------------------------------------------------------ A11/A12


def gemm_nt(A, B, out, alpha: float = 1.0, accumulate: bool = False, m_valid=None, n_valid=None, status=None,
            lp_dtype: int = DT_BF16, splits: int = 0) -> torch.Tensor:
    """out[:m_valid, :n_valid] = alpha * A @ B.T (+ out). splits <= 0: one
    256-row tile of B per work unit; else each unit streams 1/splits of B."""
    _cuda(A, "A")
    _cuda(B, "B")
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=A.device)
    m_valid = A.shape[0] if m_valid is None else m_valid
    n_valid = B.shape[0] if n_valid is None else n_valid
    call("ebsd_gemm_nt", ptr(A), A.shape[0], ptr(B), B.shape[0], A.shape[1], lp_dtype, float(alpha),
         int(bool(accumulate)), ptr(out), out.stride(0), int(m_valid), int(n_valid), int(splits),
         ptr(status), _stream(A.device))
    return status


def gemm_f32(A: torch.Tensor, B: torch.Tensor, out: torch.Tensor, alpha: float = 1.0, accumulate: bool = False,
             status=None, splits: int = 0) -> torch.Tensor:
    """out[:m, :n] = alpha * A @ B.T (+ out) from FP32 rows read as TF32
    (ebsd_gemm_f32); A (m x k), B (n x k) with unit column stride."""
    _cuda(A, "A", torch.float32, contiguous=False)
    _cuda(B, "B", torch.float32, contiguous=False)
    if A.stride(1) != 1 or B.stride(1) != 1 or out.stride(1) != 1:
        raise ValueError("gemm_f32 needs rows with unit column stride")
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=A.device)
    call("ebsd_gemm_f32", ptr(A), A.stride(0), A.shape[0], ptr(B), B.stride(0), B.shape[0], A.shape[1],
         float(alpha), int(bool(accumulate)), ptr(out), out.stride(0), int(splits), ptr(status), _stream(A.device))
    return status


def col_mean(X: torch.Tensor) -> torch.Tensor:
    _cuda(X, "X", torch.float32, contiguous=False)
    out = torch.empty(X.shape[1], dtype=torch.float32, device=X.device)
    call("ebsd_col_mean", ptr(X), X.shape[0], X.shape[1], X.stride(0), ptr(out), _stream(X.device))
    return out


def split3(X: torch.Tensor, pattern: int, transpose: bool, seg_len: int, out_rows_pad: int, ld_out: int,
           shift: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Three-term bf16 split (see ebsd_split3_bf16); returns (out_rows_pad, ld_out) bf16 with
    rows beyond the data zero-filled."""
    _cuda(X, "X", torch.float32, contiguous=False)
    n_rows, n_cols = X.shape
    rows = n_cols if transpose else n_rows
    out = torch.empty((out_rows_pad, ld_out), dtype=torch.bfloat16, device=X.device)
    if out_rows_pad > rows:
        out[rows:].zero_()
    call("ebsd_split3_bf16", ptr(X), n_rows, n_cols, X.stride(0), ptr(shift), int(bool(transpose)), int(pattern),
         ptr(out), ld_out, int(seg_len), _stream(X.device))
    return out


# ---------------------------------------------------------------------- A14


def disori_angle(q1: torch.Tensor, q2: torch.Tensor, laue_id: int) -> torch.Tensor:
    _cuda(q1, "quats1", torch.float32)
    _cuda(q2, "quats2", torch.float32)
    if q1.shape != q2.shape or q1.shape[-1] != 4:
        raise ValueError(f"quats1 and quats2 must have the same (..., 4) shape, got {q1.shape} and {q2.shape}")
    out = torch.empty(q1.shape[:-1], dtype=torch.float32, device=q1.device)
    call("ebsd_disori_angle", ptr(q1), ptr(q2), out.numel(), int(laue_id), ptr(out), _stream(q1.device))
    return out
