"""Drop-in dictionary indexing (mirror of ebsdtorch/ebsd/indexing.py).

``dictionary_index_orientations`` (indexing.py:14-211) and
``pca_dictionary_index_orientations`` (indexing.py:214-476) keep the
reference's arguments, return None and write the same results into the
ExperimentPatterns object: ``raw_indexing_results[phase] = (quaternions
(N, k, 4), metrics (N, k))`` followed by ``combine_indexing_results``.

Behind them every step runs on this package's sm_100a kernels: FP64 grid
generation, the fused projector, pattern preparation, the tcgen05
contraction with streaming top-k and the FP32 re-score. The reference's
chunk-size arguments are accepted and ignored (chunking is planned from the
free device memory); ``quantized_if_x86`` / ``quantized_via_ao`` are CPU
options and ignored. Keyword-only extras: ``precision`` ("bf16" | "fp8"),
``rescore_k`` (FP32 re-score depth, 0 = off), ``similarity`` ("dot" = the
reference's raw dot of zero-mean patterns | "cosine"), ``device``,
``workspace_bytes``; PCA DI also takes ``component_slice``.

Both functions also store ``experiment_patterns.raw_indexing_indices[phase]``
(positions in that phase's permuted dictionary) and
``experiment_patterns.dictionaries[phase]`` (that dictionary).
"""

from __future__ import annotations

from typing import List, Optional, Union

import torch
from torch import Tensor

from .. import kernels
from ..engine import Searcher, SearchConfig, default_budget, wave_query_tiles
from ..kernels import RowBuffers, round_up
from ..s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle


def _device(mp, device) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("ebsdtorch_b200 dictionary indexing requires a CUDA (sm_100) device")
    if device is not None:
        return torch.device(device)
    d = mp.master_pattern.device
    return d if d.type == "cuda" else torch.device("cuda", torch.cuda.current_device())


def _check_common(distance_metric: str, average_pattern_center: bool):
    if distance_metric not in ("angular", "euclidean", "manhattan"):
        raise NotImplementedError(f"'{distance_metric}' not supported.")
    if not average_pattern_center:
        raise NotImplementedError(
            "average_pattern_center=False is not supported (the reference never initialises the per-scan-point "
            "coordinates it needs)")


def _similarity(distance_metric: str, similarity: str) -> str:
    """The engine's score for the reference's distance_metric: "angular" is
    the raw dot of zero-mean rows (or its cosine when asked), "euclidean" the
    squared euclidean distance, "manhattan" the L1 distance (knn.py:85-97)."""
    if distance_metric in ("euclidean", "manhattan"):
        if similarity != "dot":
            raise ValueError("similarity applies to distance_metric='angular' only")
        return distance_metric
    return similarity


def _unit_rays_soa(geometry, binning: int, signal_mask: Optional[Tensor], device) -> Tensor:
    """(3, P') float32 unit rays of the masked, binned detector pixels."""
    coords = geometry.get_coords_sample_frame(binning=(binning, binning))
    c = coords.detach().reshape(-1, 3).double().cpu()
    c = c / c.norm(dim=-1, keepdim=True)
    if signal_mask is not None:
        m = signal_mask.reshape(-1).cpu().bool()
        if m.numel() != c.shape[0]:
            raise ValueError(f"signal_mask has {m.numel()} pixels but the binned detector has {c.shape[0]}")
        c = c[m]
    return c.t().contiguous().float().to(device)


def _pix_index(signal_mask: Optional[Tensor], device) -> Optional[Tensor]:
    if signal_mask is None:
        return None
    return torch.nonzero(signal_mask.reshape(-1).cpu().bool()).reshape(-1).to(torch.int32).to(device)


def _master_pattern_tensor(mp, binning: int, device) -> Tensor:
    t = mp.master_pattern.detach().to(device=device, dtype=torch.float32).contiguous()
    if binning > 1:
        t = kernels.avg_pool(t, binning)
    return t


def _pattern_source(experiment_patterns, device):
    pats = experiment_patterns.patterns
    if pats.dtype not in kernels.PATTERN_DTYPES:
        pats = pats.float()
    if pats.device.type == "cuda" and pats.device != device:
        pats = pats.to(device)
    return pats


# match waves per query chunk when the patterns stream from pinned host memory
HOST_CHUNK_WAVES = 8


class _QueryFill:
    """Query rows of patterns [q0, q1) (K2). Device patterns go straight to
    the prep kernel. Host patterns are first copied into one of two device
    staging buffers. When they are pinned, `prefetch(q0, q1)` (called by the
    engine once the current chunk is filled) starts the next chunk's copy on
    a side stream, so the host-to-device transfer runs under the current
    chunk's match kernels."""

    def __init__(self, pats: Tensor, binning: int, pix_index, n_pix: int, subtract_mean: bool, device):
        self.pats, self.binning, self.pix_index, self.n_pix = pats, binning, pix_index, n_pix
        self.subtract_mean, self.device = subtract_mean, device
        self.host = pats.device.type != "cuda"
        self.copy_stream = torch.cuda.Stream(device) if self.host and pats.is_pinned() else None
        self.slots = [None, None]      # staging buffers
        self.slot_free = [None, None]  # event: the last prep reading the slot is done
        self.next_slot = 0
        self.pending = {}              # (q0, q1) -> (slot, copy-done event)

    def _stage(self, q0: int, q1: int, stream) -> tuple:
        slot = self.next_slot
        self.next_slot ^= 1
        n = q1 - q0
        buf = self.slots[slot]
        if buf is None or buf.shape[0] < n:
            buf = torch.empty((n,) + tuple(self.pats.shape[1:]), dtype=self.pats.dtype, device=self.device)
            self.slots[slot] = buf
        if self.slot_free[slot] is not None:
            stream.wait_event(self.slot_free[slot])
        with torch.cuda.stream(stream):
            buf[:n].copy_(self.pats[q0:q1], non_blocking=True)
        if stream is self.copy_stream:
            buf.record_stream(stream)
        done = torch.cuda.Event()
        done.record(stream)
        return slot, done

    def prefetch(self, q0: int, q1: int) -> None:
        if self.copy_stream is not None and (q0, q1) not in self.pending and len(self.pending) < 1:
            self.pending[(q0, q1)] = self._stage(q0, q1, self.copy_stream)

    def __call__(self, q0: int, q1: int, bufs: RowBuffers) -> None:
        if not self.host:
            kernels.prep_patterns(self.pats[q0:q1].contiguous(), bufs, self.binning, self.pix_index, self.n_pix,
                                  self.subtract_mean)
            return
        cur = torch.cuda.current_stream(self.device)
        if (q0, q1) in self.pending:
            slot, done = self.pending.pop((q0, q1))
            cur.wait_event(done)
        else:
            for key, (slot, done) in list(self.pending.items()):  # a prefetch that was not used
                cur.wait_event(done)
                self.slot_free[slot] = done
                del self.pending[key]
            slot, _ = self._stage(q0, q1, cur)
        kernels.prep_patterns(self.slots[slot][:q1 - q0], bufs, self.binning, self.pix_index, self.n_pix,
                              self.subtract_mean)
        free = torch.cuda.Event()
        free.record(cur)
        self.slot_free[slot] = free


def _query_fill(pats: Tensor, binning: int, pix_index, n_pix: int, subtract_mean: bool, device):
    return _QueryFill(pats, binning, pix_index, n_pix, subtract_mean, device)


def _store(experiment_patterns, phase: int, ori: Tensor, idx: Tensor, val: Tensor, out_dtype):
    Q, k = idx.shape
    quats = kernels.gather_rows(ori, idx.reshape(-1)).reshape(Q, k, 4)
    experiment_patterns.set_raw_indexing_results(quats, val.to(out_dtype), phase_id=phase)
    if not hasattr(experiment_patterns, "raw_indexing_indices"):
        experiment_patterns.raw_indexing_indices = {}
        experiment_patterns.dictionaries = {}
    experiment_patterns.raw_indexing_indices[phase] = idx
    experiment_patterns.dictionaries[phase] = ori


def _metric_dtype(match_dtype):
    return match_dtype if match_dtype in (torch.float16, torch.bfloat16, torch.float32, torch.float64) \
        else torch.float32


def dictionary_index_orientations(
    master_patterns,
    geometry,
    experiment_patterns,
    signal_mask: Optional[Tensor] = None,
    subtract_exp_pat_mean: bool = True,
    experiment_chunk_size: int = 256,
    dictionary_resolution_degrees: float = 0.5,
    dictionary_chunk_size: int = 256,
    virtual_binning: int = 1,
    top_k_matches: int = 1,
    distance_metric: str = "angular",
    match_dtype: torch.dtype = torch.float16,
    quantized_if_x86: bool = True,
    average_pattern_center: bool = True,
    *,
    precision: str = "bf16",
    rescore_k: int = 32,
    similarity: str = "dot",
    device=None,
    workspace_bytes: Optional[int] = None,
) -> None:
    """Plain dictionary indexing (indexing.py:14-211). See the module doc."""
    _check_common(distance_metric, average_pattern_center)
    if not isinstance(master_patterns, (list, tuple)):
        master_patterns = [master_patterns]
    n_q = experiment_patterns.n_patterns
    # the reference honours subtract_exp_pat_mean only on its all-at-once path
    subtract = bool(subtract_exp_pat_mean) if experiment_chunk_size > n_q else True
    cfg = SearchConfig(precision=precision, rescore_k=rescore_k, similarity=_similarity(distance_metric, similarity),
                       workspace_bytes=workspace_bytes)
    pats_host = experiment_patterns.patterns
    stream_host = pats_host.device.type != "cuda" and pats_host.is_pinned()
    for i, mp in enumerate(master_patterns):
        dev = _device(mp, device)
        with torch.cuda.device(dev):  # kernels launch on the device that holds the data
            if stream_host:
                # chunks of a few match waves, so each chunk's copy runs under the
                # previous chunk's match and only the first copy is exposed
                cfg.max_query_chunk = HOST_CHUNK_WAVES * wave_query_tiles(dev) * kernels.TILE_Q
            ori = sample_ori_fz_laue_angle(mp.laue_group, dictionary_resolution_degrees, dev, permute=True)
            rays = _unit_rays_soa(geometry, virtual_binning, signal_mask, dev)
            mp_t = _master_pattern_tensor(mp, virtual_binning, dev)
            pix_index = _pix_index(signal_mask, dev)
            n_pix = rays.shape[1]
            pats = _pattern_source(experiment_patterns, dev)

            def fill_dict(d0, d1, bufs, mp_t=mp_t, rays=rays, ori=ori):
                kernels.project(mp_t, rays, ori[d0:d1], bufs, subtract_mean=True)

            searcher = Searcher(ori.shape[0], n_q, n_pix, int(top_k_matches), cfg, dev)
            idx, val = searcher.run(fill_dict, _query_fill(pats, virtual_binning, pix_index, n_pix, subtract, dev))
            _store(experiment_patterns, i, ori, idx, val, _metric_dtype(match_dtype))
    experiment_patterns.combine_indexing_results(higher_is_better=(distance_metric == "angular"))


# --------------------------------------------------------------------- PCA


def fit_pca_components(mp_t: Tensor, rays: Tensor, ori_learn: Tensor, n_components: int,
                       component_slice: str = "top", timings: Optional[dict] = None) -> Tensor:
    """PCA basis of the zero-mean simulated patterns of `ori_learn`
    (indexing.py:290-355, pca_covmat.py:94-158). The covariance is an
    FP32-class product on the tensor cores (3-term bf16 split) of the
    column-centred rows, divided by N - 1; its eigenvectors come from
    torch.linalg.eigh. Returns (n_eff, P') float32 component rows.

    component_slice "top": the n leading eigenvectors. "reference": the
    reference's slice ``[:, -n : -n + 300]`` (indexing.py:355), which keeps at
    most 300 and, for P' >= 300 and n < 300, none. `timings`, when given,
    receives the seconds of the covariance and of the eigendecomposition."""
    import time

    dev = mp_t.device
    t0 = time.perf_counter()
    N, P = ori_learn.shape[0], rays.shape[1]
    if N < 2:
        raise ValueError("PCA needs at least two learning orientations")
    X = torch.empty((N, P), dtype=torch.float32, device=dev)
    kernels.project(mp_t, rays, ori_learn, RowBuffers(f32=X), subtract_mean=True)
    mu = kernels.col_mean(X)
    seg = round_up(N, 64)
    A3 = kernels.split3(X, 0, True, seg, round_up(P, kernels.TILE_Q), 3 * seg, shift=mu)
    B3 = kernels.split3(X, 1, True, seg, round_up(P, kernels.TILE_D), 3 * seg, shift=mu)
    del X
    cov = torch.empty((P, P), dtype=torch.float32, device=dev)
    status = kernels.gemm_nt(A3, B3, cov, alpha=1.0 / (N - 1), m_valid=P, n_valid=P)
    del A3, B3
    if int(status.item()) != 0:
        raise RuntimeError("covariance GEMM reported a device timeout")
    t1 = time.perf_counter()
    _, vecs = torch.linalg.eigh(cov)
    del cov
    if timings is not None:
        torch.cuda.synchronize(dev)
        timings["covariance_s"] = t1 - t0
        timings["eigh_s"] = time.perf_counter() - t1
    if component_slice == "reference":
        V = vecs[:, -n_components:(-n_components + 300)]
    elif component_slice == "top":
        V = vecs[:, -n_components:]
    else:
        raise ValueError("component_slice must be 'top' or 'reference'")
    if V.shape[1] == 0:
        raise ValueError(
            f"the reference component slice [-{n_components}:{300 - n_components}] selects no components "
            f"for {P} pixels; use component_slice='top'")
    return V.t().contiguous()


# When set to a list, _Projector appends (start, end, flops) CUDA-event
# triples around every projection (split + GEMM; measurement only).
PROJ_TIMERS: Optional[list] = None


class _Projector:
    """rows (n x P') fp32 -> rows @ comps.T (n x n_comp) fp32 on the tensor
    cores. TF32 (kind::tf32, ebsd_gemm_f32) straight from the FP32 rows when
    P' is a multiple of 4 (16-byte rows for the tensor-memory copies);
    otherwise the 3-term bf16 split of both operands. At 128 x 128 px and
    1,024 components both come within ~1e-4 of FP64 (relative to each row's
    largest component); TF32 needs no split pass and one third of the tensor
    work."""

    def __init__(self, comps: Tensor):
        self.n_comp, self.P = comps.shape
        self.status = torch.zeros(1, dtype=torch.int32, device=comps.device)
        self.tf32 = self.P % 4 == 0
        if self.tf32:
            self.comps = comps.contiguous()
        else:
            self.seg = round_up(self.P, 64)
            self.B3 = kernels.split3(comps, 1, False, self.seg, round_up(self.n_comp, kernels.TILE_D), 3 * self.seg)

    def __call__(self, X: Tensor, out: Tensor) -> None:
        n = X.shape[0]
        timers = PROJ_TIMERS
        if timers is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
        if self.tf32 and X.stride(0) % 4 == 0 and X.data_ptr() % 16 == 0:
            kernels.gemm_f32(X, self.comps, out, status=self.status)
        else:
            if not hasattr(self, "B3"):
                self.seg = round_up(self.P, 64)
                self.B3 = kernels.split3(self.comps, 1, False, self.seg, round_up(self.n_comp, kernels.TILE_D),
                                         3 * self.seg)
            A3 = kernels.split3(X, 0, False, self.seg, round_up(n, kernels.TILE_Q), 3 * self.seg)
            kernels.gemm_nt(A3, self.B3, out, m_valid=n, n_valid=self.n_comp, status=self.status)
        if timers is not None:
            ev[1].record()
            timers.append((ev[0], ev[1], 2.0 * n * self.P * self.n_comp))


def _finish_rows(Y: Tensor, bufs: RowBuffers):
    """lp copy + norms of already-final fp32 rows Y (n x n_comp)."""
    kernels.prep_patterns(Y.view(Y.shape[0], 1, Y.shape[1]),
                          RowBuffers(lp=bufs.lp, lp_dtype=bufs.lp_dtype, norm=bufs.norm, lp_scale=bufs.lp_scale),
                          subtract_mean=False)


def pca_dictionary_index_orientations(
    master_patterns,
    geometry,
    experiment_patterns,
    n_pca_components: int,
    signal_mask: Optional[Tensor] = None,
    subtract_exp_pat_mean: bool = True,
    experiment_chunk_size: int = 256,
    dictionary_resolution_learn_deg: float = 0.5,
    dictionary_resolution_index_deg: float = 0.5,
    dictionary_chunk_size: int = 256,
    virtual_binning: int = 1,
    top_k_matches: int = 1,
    distance_metric: str = "angular",
    match_dtype: torch.dtype = torch.float16,
    quantized_via_ao: bool = True,
    average_pattern_center: bool = True,
    *,
    component_slice: str = "top",
    precision: str = "bf16",
    rescore_k: int = 32,
    similarity: str = "dot",
    device=None,
    workspace_bytes: Optional[int] = None,
    sub_chunk: int = 16384,
    components=None,
) -> None:
    """PCA dictionary indexing (indexing.py:214-476). See the module doc and
    fit_pca_components for ``component_slice``. ``components``: optional
    basis from an earlier call (``experiment_patterns.pca_components`` -- one
    (n_comp, P') float32 tensor, or a list with one per master pattern) that
    is used instead of fitting one; the learning dictionary is then not
    built."""
    _check_common(distance_metric, average_pattern_center)
    if not isinstance(master_patterns, (list, tuple)):
        master_patterns = [master_patterns]
    n_q = experiment_patterns.n_patterns
    subtract = bool(subtract_exp_pat_mean) if experiment_chunk_size > n_q else True
    for i, mp in enumerate(master_patterns):
        dev = _device(mp, device)
        with torch.cuda.device(dev):  # kernels launch on the device that holds the data
            rays = _unit_rays_soa(geometry, virtual_binning, signal_mask, dev)
            mp_t = _master_pattern_tensor(mp, virtual_binning, dev)
            pix_index = _pix_index(signal_mask, dev)
            P = rays.shape[1]
            given = components[i] if isinstance(components, (list, tuple, dict)) else components
            if given is None:
                ori = sample_ori_fz_laue_angle(mp.laue_group, dictionary_resolution_learn_deg, dev)
                comps = fit_pca_components(mp_t, rays, ori, int(n_pca_components), component_slice)
                if dictionary_resolution_learn_deg != dictionary_resolution_index_deg:
                    ori = sample_ori_fz_laue_angle(mp.laue_group, dictionary_resolution_index_deg, dev)
            else:
                comps = given.to(device=dev, dtype=torch.float32).contiguous()
                if comps.dim() != 2 or comps.shape[1] != P:
                    raise ValueError(f"components must be (n_comp, {P}) for this detector, got {tuple(comps.shape)}")
                # the reference draws the learning dictionary's permutation
                # first: keep the global generator in step with it
                ori_learn = sample_ori_fz_laue_angle(mp.laue_group, dictionary_resolution_learn_deg, dev)
                ori = ori_learn if dictionary_resolution_learn_deg == dictionary_resolution_index_deg else \
                    sample_ori_fz_laue_angle(mp.laue_group, dictionary_resolution_index_deg, dev)
                del ori_learn
            proj = _Projector(comps)
            n_comp = comps.shape[0]
            pats = _pattern_source(experiment_patterns, dev)
            qfill_full = _query_fill(pats, virtual_binning, pix_index, P, subtract, dev)

            def fill_dict(d0, d1, bufs, mp_t=mp_t, rays=rays, ori=ori, proj=proj):
                for s0 in range(d0, d1, sub_chunk):
                    s1 = min(d1, s0 + sub_chunk)
                    X = torch.empty((s1 - s0, P), dtype=torch.float32, device=dev)
                    kernels.project(mp_t, rays, ori[s0:s1], RowBuffers(f32=X), subtract_mean=True)
                    Y = bufs.f32[s0 - d0:s1 - d0] if bufs.f32 is not None else torch.empty(
                        (s1 - s0, n_comp), dtype=torch.float32, device=dev)
                    proj(X, Y)
                    _finish_rows(Y, _slice(bufs, s0 - d0, s1 - d0))

            def fill_queries(q0, q1, bufs, proj=proj):
                for s0 in range(q0, q1, sub_chunk):
                    s1 = min(q1, s0 + sub_chunk)
                    X = torch.empty((s1 - s0, P), dtype=torch.float32, device=dev)
                    qfill_full(s0, s1, RowBuffers(f32=X))
                    Y = bufs.f32[s0 - q0:s1 - q0] if bufs.f32 is not None else torch.empty(
                        (s1 - s0, n_comp), dtype=torch.float32, device=dev)
                    proj(X, Y)
                    _finish_rows(Y, _slice(bufs, s0 - q0, s1 - q0))

            budget = workspace_bytes or int(default_budget(dev) * 0.7)
            cfg = SearchConfig(precision=precision, rescore_k=rescore_k,
                               similarity=_similarity(distance_metric, similarity), workspace_bytes=budget)
            searcher = Searcher(ori.shape[0], n_q, n_comp, int(top_k_matches), cfg, dev)
            idx, val = searcher.run(fill_dict, fill_queries)
            if int(proj.status.item()) != 0:
                raise RuntimeError("PCA projection GEMM reported a device timeout")
            _store(experiment_patterns, i, ori, idx, val, _metric_dtype(match_dtype))
            experiment_patterns.pca_components = getattr(experiment_patterns, "pca_components", {})
            experiment_patterns.pca_components[i] = comps
    experiment_patterns.combine_indexing_results(higher_is_better=(distance_metric == "angular"))


def _slice(bufs: RowBuffers, r0: int, r1: int) -> RowBuffers:
    return RowBuffers(
        f32=None,
        lp=bufs.lp[r0:r1] if bufs.lp is not None else None,
        lp_dtype=bufs.lp_dtype,
        norm=bufs.norm[r0:r1] if bufs.norm is not None else None,
        lp_scale=bufs.lp_scale[r0:r1] if bufs.lp_scale is not None else None,
    )
