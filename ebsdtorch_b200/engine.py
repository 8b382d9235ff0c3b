"""Dictionary-indexing engine: the GPU pipeline behind the drop-in functions.

Data layout in HBM (one phase):
  dictionary  lp rows   (D_pad x K_pad)  bf16 / e4m3, unit L2 norm, zero padded
              f32 rows  (D x P')         zero-mean FP32 rows (the reference's vectors)
              norm, lp scale (D_pad)     per-row L2 norm, e4m3 dequant scale
  query chunk the same three for Qc rows, plus candidate lists
              (Qc_pad x splits x n_cand) and the final (Q x k) results.
Per query chunk: prepare (K2) -> tcgen05 contraction with streaming top-k
(K3) -> merge + FP32 re-score (K4). When the dictionary does not fit the
memory budget it is processed in chunks and each chunk's exact top-k is
merged into a running result.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import Callable, Optional

import torch

from . import kernels
from ._capi import DEVICE_TIMEOUT, SIM_COSINE, SIM_DOT, SIM_EUCLIDEAN, SIM_MANHATTAN
from .kernels import LP_DTYPES, LP_KMULT, LP_TORCH, TILE_D, TILE_Q, RowBuffers, round_up

MAX_CAND = 64
MAX_MERGE_CANDIDATES = 4096  # per query, ebsd_merge_rescore's limit

# When set to a list, Searcher.run appends (start, end, flops) CUDA-event
# triples around every tensor-core match launch (measurement only).
MATCH_TIMERS: Optional[list] = None
# When set to a one-element int64 device tensor, the merge kernels add the
# number of rows they re-score in FP32 to it (measurement only).
RESCORE_COUNTER: Optional[torch.Tensor] = None
# When set to a list, Searcher.run appends (start, end) CUDA-event pairs
# around every merge + re-score launch (measurement only).
MERGE_TIMERS: Optional[list] = None
# NVTX ranges around the phases of Searcher.run (dictionary chunk fill,
# query chunk preparation, match wave, merge) for timeline profilers; off
# unless EBSD_NVTX=1 in the environment.
NVTX = os.environ.get("EBSD_NVTX", "0") == "1"


class _Range:
    """NVTX range when NVTX is on, else nothing."""

    def __init__(self, name: str):
        self.name = name

    def __enter__(self):
        if NVTX:
            torch.cuda.nvtx.range_push(self.name)

    def __exit__(self, *exc):
        if NVTX:
            torch.cuda.nvtx.range_pop()
        return False


@dataclass
class SearchConfig:
    """precision: element type of the tensor-core contraction ("bf16" | "fp8").
    rescore_k: candidates per query re-scored in FP32 (0 = report the
    low-precision score). similarity: "dot" is the reference's angular metric
    (raw dot of zero-mean rows, knn.py:96-97); "cosine" divides it by both
    norms; "euclidean" is the reference's squared euclidean distance of the
    zero-mean rows (knn.py:85-91), smallest first; "manhattan" their L1
    distance (knn.py:92-93), exact FP32 on the CUDA cores, smallest first.
    workspace_bytes: device-memory budget (default: 90 % of free memory)."""

    precision: str = "bf16"
    rescore_k: int = 32
    similarity: str = "dot"
    workspace_bytes: Optional[int] = None
    query_chunk: Optional[int] = None
    dict_chunk: Optional[int] = None
    # upper bound on the planned query chunk (host-resident patterns stream in
    # several chunks so that copies overlap the matching)
    max_query_chunk: Optional[int] = None
    # match launch shape (the batch autotuner sets these): dictionary rows per
    # CTA tile (0 = 256), dictionary ranges per query tile (0 = automatic),
    # query tiles per launch (0 = one wave), or one persistent launch per
    # query chunk with one CTA per SM
    tile_n: int = 0
    splits: int = 0
    wave_tiles: int = 0
    persistent: bool = False
    # re-score in FP32 only the candidates whose bf16 score, widened by a
    # rigorous rounding bound, can still reach the exact top-k (same results)
    rescore_gate: bool = True

    def validate(self):
        if self.precision not in LP_DTYPES:
            raise ValueError(f"precision must be one of {sorted(LP_DTYPES)}, got {self.precision!r}")
        if self.similarity not in ("dot", "cosine", "euclidean", "manhattan"):
            raise ValueError(f"similarity must be 'dot', 'cosine', 'euclidean' or 'manhattan', "
                             f"got {self.similarity!r}")
        if not 0 <= self.rescore_k <= 128:
            raise ValueError("rescore_k must be in [0, 128]")
        if self.tile_n not in (0, 128, 256):
            raise ValueError("tile_n must be 0, 128 or 256")
        if self.splits < 0 or self.wave_tiles < 0:
            raise ValueError("splits and wave_tiles must be >= 0")


def _pow2_at_least(n: int) -> int:
    return 1 << max(0, math.ceil(math.log2(max(1, n))))


class RowSet:
    """Low-precision + FP32 rows of a dictionary (or query) block on the GPU."""

    def __init__(self, n_rows: int, n_pix: int, pad_rows: int, lp_dtype: int, keep_f32: bool, device,
                 storage: Optional[torch.Tensor] = None):
        """storage: optional uint8 device tensor of at least
        storage_bytes(...) bytes to carve the buffers from (re-used between
        dictionaries of different shapes); its padding rows are zeroed here."""
        self.n_rows, self.n_pix, self.lp_dtype = n_rows, n_pix, lp_dtype
        self.k_pad = round_up(n_pix, LP_KMULT[lp_dtype])
        rows_pad = round_up(max(n_rows, 1), pad_rows)
        lp_t = LP_TORCH[lp_dtype]
        if storage is None:
            self.lp = torch.zeros((rows_pad, self.k_pad), dtype=lp_t, device=device)
            self.f32 = torch.empty((n_rows, n_pix), dtype=torch.float32, device=device) if keep_f32 else None
            self.norm = torch.zeros(rows_pad, dtype=torch.float32, device=device)
            self.lp_scale = torch.ones(rows_pad, dtype=torch.float32, device=device) \
                if lp_dtype != kernels.DT_BF16 else None
            return
        need = RowSet.storage_bytes(n_rows, n_pix, pad_rows, lp_dtype, keep_f32)
        if storage.dtype != torch.uint8 or storage.numel() < need:
            raise ValueError(f"row storage holds {storage.numel()} bytes, {need} needed")
        views, off = [], 0
        for shape, dt in RowSet._layout(n_rows, n_pix, pad_rows, lp_dtype, keep_f32):
            nbytes = math.prod(shape) * torch.empty((), dtype=dt).element_size()
            views.append(storage[off:off + nbytes].view(dt).view(shape) if nbytes else None)
            off = round_up(off + nbytes, 256)
        self.lp, self.f32, self.norm, self.lp_scale = views
        if not keep_f32:
            self.f32 = None
        if lp_dtype == kernels.DT_BF16:
            self.lp_scale = None
        else:
            self.lp_scale.fill_(1.0)
        # rows beyond n_rows take part in the tensor-core tiles: zero them
        self.lp[n_rows:].zero_()
        self.norm[n_rows:].zero_()

    @staticmethod
    def _layout(n_rows: int, n_pix: int, pad_rows: int, lp_dtype: int, keep_f32: bool):
        k_pad = round_up(n_pix, LP_KMULT[lp_dtype])
        rows_pad = round_up(max(n_rows, 1), pad_rows)
        return [((rows_pad, k_pad), LP_TORCH[lp_dtype]), ((n_rows if keep_f32 else 0, n_pix), torch.float32),
                ((rows_pad,), torch.float32), ((rows_pad if lp_dtype != kernels.DT_BF16 else 0,), torch.float32)]

    @staticmethod
    def storage_bytes(n_rows: int, n_pix: int, pad_rows: int, lp_dtype: int, keep_f32: bool) -> int:
        """Bytes of `storage` a RowSet of this shape needs (256-byte aligned parts)."""
        off = 0
        for shape, dt in RowSet._layout(n_rows, n_pix, pad_rows, lp_dtype, keep_f32):
            off = round_up(off + math.prod(shape) * torch.empty((), dtype=dt).element_size(), 256)
        return off

    def buffers(self, r0: int, r1: int, with_f32: bool = True) -> RowBuffers:
        return RowBuffers(
            f32=self.f32[r0:r1] if (self.f32 is not None and with_f32) else None,
            lp=self.lp[r0:r1],
            lp_dtype=self.lp_dtype,
            norm=self.norm[r0:r1],
            lp_scale=self.lp_scale[r0:r1] if self.lp_scale is not None else None,
        )

    @staticmethod
    def bytes_per_row(n_pix: int, lp_dtype: int, keep_f32: bool) -> int:
        k_pad = round_up(n_pix, LP_KMULT[lp_dtype])
        return k_pad * (2 if lp_dtype == kernels.DT_BF16 else 1) + (4 * n_pix if keep_f32 else 0) + 8


def _col_scale(rows: RowSet, similarity: str) -> Optional[torch.Tensor]:
    """Per-dictionary-row factor of the tensor-core score: |d| (dot metric),
    2 |d| (euclidean), times the e4m3 dequant scale."""
    if similarity == "dot":
        return rows.norm if rows.lp_scale is None else rows.norm * rows.lp_scale
    if similarity == "euclidean":
        return 2.0 * rows.norm if rows.lp_scale is None else 2.0 * rows.norm * rows.lp_scale
    return rows.lp_scale


def _col_bias(rows: RowSet, similarity: str) -> Optional[torch.Tensor]:
    """Per-dictionary-row term of the euclidean score, -|d|^2: with the
    per-query factor 1 / (|q| e4m3-scale) the tensor-core score ranks like
    2 q.d - |d|^2, i.e. by the smallest |q - d|^2."""
    return -(rows.norm * rows.norm) if similarity == "euclidean" else None


def _row_scale(rows: RowSet, similarity: str) -> Optional[torch.Tensor]:
    if similarity != "euclidean":
        return None
    n = rows.norm if rows.lp_scale is None else rows.norm * rows.lp_scale
    return torch.where(n > 0, 1.0 / n.clamp_min(1e-30), torch.zeros_like(n))


def wave_query_tiles(device, row_bytes: int = 0) -> int:
    """Query tiles per match launch, so that with the automatic dictionary
    ranges (SMs / tiles) one launch is one wave of one-CTA-per-SM units.
    Every dictionary tile meets the launch's whole query set; while that set
    (tiles x 128 rows x row_bytes) fits in about two thirds of L2 next to
    the dictionary tiles in flight, a quarter of the SMs is used (37 tiles x
    4 ranges on a 148-SM B200), otherwise an eighth (18 x 8 = 144 CTAs).
    Measured at 128 x 128 px: bf16 rows (32 KB; 37 tiles are 151 MB) read
    4.9x their operand bytes from DRAM per launch with 37 tiles and 2.1x
    with 18; in alternating runs of the full bench on one GPU the two shapes
    came within about 1 % (18 tiles: 30 MHz more SM clock under the power
    cap, four SMs idle), so the one that moves less data is used. e4m3 rows
    (16 KB, 76 MB for 37 tiles) were ~2 % slower with 18 tiles (no traffic
    to save). row_bytes 0 (unknown) takes the smaller count."""
    props = torch.cuda.get_device_properties(device)
    return wave_tiles_for(props.multi_processor_count, getattr(props, "L2_cache_size", 0) or (126 << 20), row_bytes)


def wave_tiles_for(sms: int, l2_bytes: int, row_bytes: int = 0, tile_pairs: bool = False) -> int:
    """The rule of wave_query_tiles for a device of `sms` SMs and `l2_bytes`
    of L2. tile_pairs: the launch variant takes query tiles two at a time
    (two-tile CTAs or CTA pairs), so an odd count is rounded down to an even
    one (an odd count runs the one-tile kernel)."""
    quarter = max(1, sms // 4)
    if row_bytes > 0 and quarter * TILE_Q * row_bytes <= (2 * l2_bytes) // 3:
        tiles = quarter
    else:
        tiles = max(1, sms // 8)
    return even_tiles(tiles, tile_pairs)


def even_tiles(tiles: int, tile_pairs: bool) -> int:
    """An odd query-tile count rounded down to an even one for launch
    variants that take the tiles two at a time."""
    return tiles - 1 if tile_pairs and tiles > 1 and tiles % 2 else tiles


def default_budget(device) -> int:
    free, _ = torch.cuda.mem_get_info(device)
    return int(free * 0.9)


# A query provider fills rows [q0, q1) of a RowSet: fn(q0, q1, buffers)
QueryFill = Callable[[int, int, RowBuffers], None]
# A dictionary provider fills rows [d0, d1): fn(d0, d1, buffers)
DictFill = Callable[[int, int, RowBuffers], None]


class Searcher:
    """Top-k dictionary search for one phase."""

    def __init__(self, n_dict: int, n_queries: int, n_pix: int, k: int, cfg: SearchConfig, device):
        cfg.validate()
        if k < 1:
            raise ValueError("top_k must be >= 1")
        if k > n_dict:
            raise ValueError(f"top_k ({k}) exceeds the dictionary size ({n_dict})")
        if k > MAX_CAND:
            raise ValueError(f"top_k above {MAX_CAND} is not supported")
        self.n_dict, self.n_queries, self.n_pix, self.k, self.cfg = n_dict, n_queries, n_pix, k, cfg
        self.device = torch.device(device)
        self.lp_dtype = LP_DTYPES[cfg.precision]
        self.manhattan = cfg.similarity == "manhattan"
        # manhattan candidates are exact FP32 distances: nothing to re-score,
        # but the FP32 rows are the kernel's input
        self.rescore = cfg.rescore_k > 0 and not self.manhattan
        self.keep_f32 = self.rescore or self.manhattan
        self.n_cand = min(MAX_CAND, _pow2_at_least(max(k, cfg.rescore_k if self.rescore else k)))
        self.n_rescore = max(k, cfg.rescore_k) if self.rescore else k
        self.sim = {"dot": SIM_DOT, "cosine": SIM_COSINE, "euclidean": SIM_EUCLIDEAN,
                    "manhattan": SIM_MANHATTAN}[cfg.similarity]
        self._plan()

    def _plan(self):
        budget = self.cfg.workspace_bytes or default_budget(self.device)
        drow = RowSet.bytes_per_row(self.n_pix, self.lp_dtype, self.keep_f32)
        qrow_base = RowSet.bytes_per_row(self.n_pix, self.lp_dtype, self.keep_f32)
        qrow = qrow_base + self.k * 12
        q_min = min(round_up(self.n_queries, TILE_Q), 16384)
        if self.cfg.dict_chunk:
            dchunk = round_up(self.cfg.dict_chunk, TILE_D)
        elif self.n_dict * drow + q_min * qrow <= budget:
            dchunk = round_up(self.n_dict, TILE_D)
        else:
            dchunk = max(TILE_D, (budget // 2) // drow // TILE_D * TILE_D)
        self.dict_chunk = min(dchunk, round_up(self.n_dict, TILE_D))
        left = budget - self.dict_chunk * drow
        if self.cfg.query_chunk:
            qchunk = round_up(self.cfg.query_chunk, TILE_Q)
        else:
            qchunk = max(TILE_Q, left // qrow // TILE_Q * TILE_Q)
            if self.cfg.max_query_chunk:
                qchunk = min(qchunk, round_up(self.cfg.max_query_chunk, TILE_Q))
        self.query_chunk = min(qchunk, round_up(self.n_queries, TILE_Q))
        if left < self.query_chunk * qrow and not self.cfg.query_chunk:
            raise MemoryError(
                f"dictionary indexing needs more device memory than the budget of {budget / 2**30:.1f} GiB")

    def run(self, fill_dict: Optional[DictFill], fill_queries: QueryFill, resident: Optional[RowSet] = None,
            check: bool = True, status: Optional[torch.Tensor] = None):
        """Search all queries against all dictionary rows.
        `resident`: an already filled RowSet holding the whole dictionary (then
        fill_dict is not called). Returns (indices (Q, k) int64, scores (Q, k)
        float32) on the device. With check=False nothing synchronises (for
        CUDA-graph capture): the caller reads `status` (a device int32 word,
        non-zero after a kernel timeout) later with check_status()."""
        dev, Q, D, k = self.device, self.n_queries, self.n_dict, self.k
        out_val = torch.empty((Q, k), dtype=torch.float32, device=dev)
        out_idx = torch.empty((Q, k), dtype=torch.int64, device=dev)
        if status is None:
            status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.status = status
        if resident is not None:
            if resident.n_rows != D or resident.lp_dtype != self.lp_dtype or (self.keep_f32 and resident.f32 is None):
                raise ValueError("resident dictionary rows do not match the search")
            self.dict_chunk = D
            dict_rows = resident
        else:
            dict_rows = RowSet(self.dict_chunk, self.n_pix, TILE_D, self.lp_dtype, self.keep_f32, dev)
        qc = self.query_chunk
        q_rows = RowSet(qc, self.n_pix, TILE_Q, self.lp_dtype, self.keep_f32, dev)
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        cfg = self.cfg
        split_cap = MAX_MERGE_CANDIDATES // self.n_cand
        if cfg.persistent:
            # one launch per query chunk; each of the SMs' CTAs loops over units
            qm, max_ctas = round_up(qc, TILE_Q), sms
            max_splits = min(cfg.splits or 4, split_cap)
        else:
            # launches of one wave of (query tile, dictionary range) units
            row_bytes = q_rows.k_pad * q_rows.lp.element_size()
            # launch variants that take query tiles two at a time get an even
            # count (an odd one runs the one-tile kernel)
            tiles = cfg.wave_tiles or even_tiles(wave_query_tiles(dev, row_bytes),
                                                 kernels.takes_tile_pairs(self.lp_dtype))
            qm, max_ctas = tiles * TILE_Q, 0
            max_splits = min(cfg.splits or max(1, sms), split_cap)
        part_val = torch.empty((min(qm, round_up(qc, TILE_Q)) * max_splits * self.n_cand,), dtype=torch.float32,
                               device=dev)
        part_idx = torch.empty(part_val.shape, dtype=torch.int32, device=dev)
        n_dchunks = (D + self.dict_chunk - 1) // self.dict_chunk
        gate = kernels.rescore_gate(self.lp_dtype, q_rows.k_pad, self.n_pix) \
            if (self.rescore and cfg.rescore_gate and cfg.similarity != "euclidean") else 0.0
        for ci, d0 in enumerate(range(0, D, self.dict_chunk)):
            d1 = min(D, d0 + self.dict_chunk)
            nd = d1 - d0
            if resident is None:
                if nd < dict_rows.n_rows:
                    dict_rows.lp[nd:].zero_()
                    dict_rows.norm[nd:].zero_()
                with _Range(f"ebsd dictionary rows [{d0}, {d1})"):
                    fill_dict(d0, d1, dict_rows.buffers(0, nd))
            col_scale = _col_scale(dict_rows, self.cfg.similarity)
            col_bias = _col_bias(dict_rows, self.cfg.similarity)
            nd_pad = round_up(nd, TILE_D)
            d_lp = dict_rows.lp[:nd_pad]
            for q0 in range(0, Q, qc):
                q1 = min(Q, q0 + qc)
                nq = q1 - q0
                with _Range(f"ebsd query rows [{q0}, {q1})"):
                    fill_queries(q0, q1, q_rows.buffers(0, nq))
                row_scale = _row_scale(q_rows, self.cfg.similarity)
                # the next chunk's host-to-device copy runs under this chunk's matching
                prefetch = getattr(fill_queries, "prefetch", None)
                if prefetch is not None:
                    if q1 < Q:
                        prefetch(q1, min(Q, q1 + qc))
                    elif ci + 1 < n_dchunks and qc < Q:
                        prefetch(0, min(Q, qc))
                for s0 in range(0, nq, qm):
                    s1 = min(nq, s0 + qm)
                    ns = s1 - s0
                    ns_pad = round_up(ns, TILE_Q)
                    tile = cfg.tile_n or 256
                    auto = max_splits if cfg.persistent else kernels.auto_splits(ns_pad, nd_pad, self.lp_dtype)
                    splits = max(1, min(cfg.splits or auto, max_splits, split_cap, nd_pad // tile))
                    timers = MATCH_TIMERS
                    if timers is not None:
                        ev0 = torch.cuda.Event(enable_timing=True)
                        ev1 = torch.cuda.Event(enable_timing=True)
                        ev0.record()
                    rng = _Range(f"ebsd match queries [{q0 + s0}, {q0 + s1}) x dictionary [{d0}, {d1})")
                    rng.__enter__()
                    if self.manhattan:
                        splits = max(1, min(max_splits, split_cap, (nd + 63) // 64,
                                            2 * sms // max(1, ns_pad // 64) + 1))
                        kernels.manhattan_topk(q_rows.f32[s0:s1], ns, ns_pad, dict_rows.f32[:nd], self.n_pix,
                                               self.n_cand, splits, part_val, part_idx, splits, 0, d0)
                    else:
                        kernels.match_topk(q_rows.lp[s0:s0 + ns_pad], d_lp, nd, self.lp_dtype, col_scale,
                                           self.n_cand, splits, part_val, part_idx, splits, 0, d0, status,
                                           tile_n=cfg.tile_n, max_ctas=max_ctas, col_bias=col_bias,
                                           row_scale=row_scale[s0:] if row_scale is not None else None)
                    rng.__exit__()
                    if timers is not None:
                        ev1.record()
                        timers.append((ev0, ev1, 2.0 * ns * nd * self.n_pix))
                    run = ci > 0
                    g0, g1 = q0 + s0, q0 + s1
                    mtimers = MERGE_TIMERS
                    if mtimers is not None:
                        m0 = torch.cuda.Event(enable_timing=True)
                        m1 = torch.cuda.Event(enable_timing=True)
                        m0.record()
                    rng = _Range(f"ebsd merge queries [{g0}, {g1})")
                    rng.__enter__()
                    kernels.merge_rescore(
                        part_val, part_idx, ns, splits, self.n_cand,
                        q_rows.f32[s0:s1] if self.rescore else None,
                        dict_rows.f32[:nd] if self.rescore else None, d0,
                        self.n_pix, None if self.manhattan else q_rows.norm[s0:], dict_rows.norm,
                        q_rows.lp_scale[s0:] if (q_rows.lp_scale is not None and not self.manhattan) else None,
                        self.sim, min(max(self.n_rescore, self.n_cand if self.manhattan else 0),
                                      splits * self.n_cand, 128), k,
                        out_val[g0:g1] if run else None, out_idx[g0:g1] if run else None,
                        out_val[g0:g1], out_idx[g0:g1], gate_rel=gate, n_rescored=RESCORE_COUNTER)
                    rng.__exit__()
                    if mtimers is not None:
                        m1.record()
                        mtimers.append((m0, m1))
        if check:
            check_status(status)
        return out_idx, out_val


def check_status(status: torch.Tensor) -> None:
    """Raise if a match kernel reported an error in its device status word."""
    st = int(status.item())
    if st != 0:
        code = "device wait timed out" if st == DEVICE_TIMEOUT else f"status {st:#x}"
        raise RuntimeError(f"dictionary match kernel reported an error: {code}")
