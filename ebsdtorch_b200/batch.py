"""Batched dictionary indexing of many scan maps of uneven size, detector
shape and phase, replayed as one CUDA graph.

Plan. Maps are grouped by (phase = master-pattern object, detector geometry,
matching precision). Each group's dictionary is projected once into device
memory and serves all of its maps. Inside a group, the maps that share
(top_k, FP32 re-score depth) are searched together as one concatenated query
set, so a 1,000-pattern map fills the same match launches as a 200,000-pattern
one. The match launch shape (dictionary rows per CTA tile, dictionary ranges
per query tile, one-wave launches or one persistent launch per query chunk) is
chosen per group shape by `LaunchTuner`, which times the candidate shapes on
the group's own dictionary and a sample of its own queries. After one eager
run the whole sequence (per group: projection, query preparation including
the host-to-device copies of pinned host patterns, matches, merges,
orientation gathers) is captured into one CUDA graph; `run()` replays it.

The per-map results equal those of `dictionary_index_orientations` on the
same dictionary: the same kernels run on the same rows, only the launch
grouping differs. No counterpart in the reference (ebsdtorch indexes one scan
per call).
"""

from __future__ import annotations

import hashlib
import json
import os
from dataclasses import dataclass, field
from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple

import torch

from . import kernels
from .engine import RowSet, Searcher, SearchConfig, check_status
from .kernels import LP_DTYPES, TILE_D, TILE_Q, RowBuffers, round_up


@dataclass
class MapJob:
    """One scan map to index.

    master_pattern: a MasterPattern (`master_pattern` tensor, `laue_group`);
    maps sharing the object share its dictionary. geometry: an EBSDGeometry.
    experiment_patterns: ExperimentPatterns whose patterns (N, H, W) are
    float32, float16, uint16 or uint8, on the device or in pinned host
    memory. rescore_k > 0 re-scores the best candidates in FP32 (the reference
    metric, the FP32 path); 0 returns the low-precision scores (the bf16 path).
    """

    master_pattern: Any
    geometry: Any
    experiment_patterns: Any
    top_k: int = 1
    rescore_k: int = 32
    precision: str = "bf16"


# candidate match launch shapes (SearchConfig fields)
LAUNCH_SHAPES: Tuple[Dict[str, Any], ...] = (
    {},
    {"persistent": True, "splits": 4},
    {"persistent": True, "splits": 2},
    {"persistent": True, "splits": 8},
    {"tile_n": 128},
    {"persistent": True, "splits": 4, "tile_n": 128},
)

# the plan sets every chunk size itself, so the searches never ask the driver
# for free memory (which must not happen while a graph is being captured)
_NO_BUDGET_LIMIT = 1 << 62


class LaunchTuner:
    """Chooses the match launch shape per problem shape by timing.

    `pick(key, time_shape)` returns the cached choice for `key`, or times
    every shape in `shapes` with `time_shape(shape) -> milliseconds` (the
    fastest of `repeats` calls after one warm-up call), caches and returns the
    fastest. With `cache_file` the choices persist as JSON between processes.
    """

    def __init__(self, shapes: Sequence[Dict[str, Any]] = LAUNCH_SHAPES, repeats: int = 1,
                 cache_file: Optional[str] = None):
        self.shapes = [dict(s) for s in shapes]
        self.repeats = max(1, int(repeats))
        self.cache_file = cache_file
        self.cache: Dict[str, Dict[str, Any]] = {}
        if cache_file and os.path.exists(cache_file):
            with open(cache_file) as f:
                self.cache = json.load(f)

    @staticmethod
    def key(n_pix: int, n_dict: int, precision: str, n_cand: int, rescore: bool, sms: int) -> str:
        return f"p{n_pix}-d{round_up(n_dict, TILE_D)}-{precision}-c{n_cand}-r{int(rescore)}-sm{sms}"

    def pick(self, key: str, time_shape: Callable[[Dict[str, Any]], float]) -> Dict[str, Any]:
        if key in self.cache:
            return dict(self.cache[key]["shape"])
        timings = []
        for shape in self.shapes:
            time_shape(shape)  # warm-up (launch attributes, tensor maps, caches)
            ms = min(time_shape(shape) for _ in range(self.repeats))
            timings.append((ms, shape))
        best_ms, best = min(timings, key=lambda t: t[0])
        self.cache[key] = {"shape": best, "ms": best_ms,
                           "tried": [{"shape": s, "ms": round(t, 4)} for t, s in timings]}
        if self.cache_file:
            with open(self.cache_file, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
        return dict(best)


@dataclass
class _SubGroup:
    top_k: int
    rescore_k: int
    maps: List[int] = field(default_factory=list)
    offsets: List[int] = field(default_factory=list)  # start of each map in the concatenation
    n_queries: int = 0
    cfg: Optional[SearchConfig] = None


@dataclass
class _Group:
    phase: int  # index into BatchIndexer.phases
    precision: str
    rays: torch.Tensor
    shape: Tuple[int, int]
    subgroups: Dict[Tuple[int, int], _SubGroup] = field(default_factory=dict)

    @property
    def rescore(self) -> bool:
        return any(s.rescore_k > 0 for s in self.subgroups.values())


def _row_slice(bufs: RowBuffers, a: int, b: int) -> RowBuffers:
    def cut(t):
        return t[a:b] if t is not None else None

    return RowBuffers(f32=cut(bufs.f32), lp=cut(bufs.lp), lp_dtype=bufs.lp_dtype, norm=cut(bufs.norm),
                      lp_scale=cut(bufs.lp_scale))


class BatchIndexer:
    """Index many maps (MapJob) in one planned batch; see the module doc.

    dictionary_resolution_degrees: one value, or a dict keyed by Laue group.
    query_chunk: query rows prepared per chunk (device memory for
    chunk x pixels x (4 + 2) bytes). After `run()` every job's
    ExperimentPatterns holds its results as after
    `dictionary_index_orientations` (raw_indexing_results, orientations,
    best_metrics, raw_indexing_indices, dictionaries). A captured graph reads
    the patterns from the tensors it was captured with: refill them in place
    to index new data of the same sizes.
    """

    def __init__(self, jobs: Sequence[MapJob], dictionary_resolution_degrees=0.5, device=None,
                 tuner: Optional[LaunchTuner] = None, autotune: bool = True, query_chunk: int = 32768):
        from .ebsd.indexing import _master_pattern_tensor, _unit_rays_soa
        from .s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

        if not jobs:
            raise ValueError("no maps to index")
        if not torch.cuda.is_available():
            raise RuntimeError("ebsdtorch_b200 batched indexing requires a CUDA (sm_100) device")
        self.device = torch.device(device) if device is not None else torch.device("cuda",
                                                                                   torch.cuda.current_device())
        self.jobs = list(jobs)
        self.tuner = tuner if tuner is not None else LaunchTuner()
        self.autotune = autotune
        self.query_chunk = round_up(int(query_chunk), TILE_Q)
        dev = self.device
        # phases: one dictionary (orientations) and master pattern per MasterPattern object
        self.phases: List[Dict[str, Any]] = []
        phase_of: Dict[int, int] = {}
        groups: Dict[Tuple, _Group] = {}
        for i, job in enumerate(self.jobs):
            if job.precision not in LP_DTYPES:
                raise ValueError(f"precision must be one of {sorted(LP_DTYPES)}, got {job.precision!r}")
            if job.top_k < 1:
                raise ValueError("top_k must be >= 1")
            pats = job.experiment_patterns.patterns
            if pats.dtype not in kernels.PATTERN_DTYPES:
                raise TypeError(f"map {i}: patterns must be float32, float16, uint16 or uint8, got {pats.dtype}")
            if pats.device.type != "cuda" and not pats.is_pinned():
                raise ValueError(f"map {i}: host patterns must be in pinned memory (they are copied inside the "
                                 "CUDA graph)")
            mp = job.master_pattern
            if id(mp) not in phase_of:
                laue = int(mp.laue_group)
                res = dictionary_resolution_degrees
                res = float(res[laue]) if isinstance(res, dict) else float(res)
                phase_of[id(mp)] = len(self.phases)
                self.phases.append({"laue": laue, "resolution": res, "mp": _master_pattern_tensor(mp, 1, dev),
                                    "ori": sample_ori_fz_laue_angle(laue, res, dev, permute=True)})
            ph = phase_of[id(mp)]
            rays = _unit_rays_soa(job.geometry, 1, None, dev)
            shape = tuple(pats.shape[-2:])
            if rays.shape[1] != shape[0] * shape[1]:
                raise ValueError(f"map {i}: patterns {shape} do not match the detector of its geometry")
            digest = hashlib.sha1(rays.cpu().numpy().tobytes()).hexdigest()
            gkey = (ph, shape, digest, job.precision)
            if gkey not in groups:
                groups[gkey] = _Group(ph, job.precision, rays, shape)
            g = groups[gkey]
            sub = g.subgroups.setdefault((job.top_k, job.rescore_k), _SubGroup(job.top_k, job.rescore_k))
            sub.offsets.append(sub.n_queries)
            sub.maps.append(i)
            sub.n_queries += int(pats.shape[0])
        self.groups: List[_Group] = list(groups.values())
        for g in self.groups:
            n_dict = self.phases[g.phase]["ori"].shape[0]
            for sub in g.subgroups.values():
                if sub.top_k > n_dict:
                    raise ValueError(f"top_k ({sub.top_k}) exceeds the dictionary size ({n_dict})")
                sub.cfg = SearchConfig(precision=g.precision, rescore_k=sub.rescore_k,
                                       query_chunk=min(self.query_chunk, round_up(sub.n_queries, TILE_Q)),
                                       workspace_bytes=_NO_BUDGET_LIMIT)
        self._phase_of_map = {m: g.phase for g in self.groups for sub in g.subgroups.values() for m in sub.maps}
        # one arena for the dictionary rows of every group: groups run one
        # after the other, and a single block (rather than one allocation per
        # group shape) keeps the graph's memory at the largest group
        self._arena_bytes = max(RowSet.storage_bytes(self.phases[g.phase]["ori"].shape[0], g.rays.shape[1], TILE_D,
                                                     LP_DTYPES[g.precision], g.rescore) for g in self.groups)
        self._arena: Optional[torch.Tensor] = None
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self._outputs = None
        self._tuned = False

    # ------------------------------------------------------------------ plan
    @property
    def n_patterns(self) -> int:
        return sum(int(j.experiment_patterns.patterns.shape[0]) for j in self.jobs)

    def describe(self) -> List[Dict[str, Any]]:
        """One entry per (group, sub-group): sizes and the chosen launch shape."""
        out = []
        for g in self.groups:
            ph = self.phases[g.phase]
            for sub in g.subgroups.values():
                c = sub.cfg
                out.append({"laue": ph["laue"], "dictionary": int(ph["ori"].shape[0]), "detector": list(g.shape),
                            "precision": g.precision, "top_k": sub.top_k, "rescore_k": sub.rescore_k,
                            "maps": len(sub.maps), "patterns": sub.n_queries,
                            "launch": {"tile_n": c.tile_n or 256, "splits": c.splits, "persistent": c.persistent}})
        return out

    def _fill(self, sub: _SubGroup) -> Callable[[int, int, RowBuffers], None]:
        dev = self.device
        starts = sub.offsets + [sub.n_queries]
        sources = [self.jobs[m].experiment_patterns.patterns for m in sub.maps]

        def fill(q0: int, q1: int, bufs: RowBuffers) -> None:
            for j, pats in enumerate(sources):
                a, b = max(q0, starts[j]), min(q1, starts[j + 1])
                if a >= b:
                    continue
                chunk = pats[a - starts[j]:b - starts[j]]
                if chunk.device.type != "cuda":
                    chunk = chunk.to(dev, non_blocking=True)
                kernels.prep_patterns(chunk.contiguous(), _row_slice(bufs, a - q0, b - q0))

        return fill

    def _dictionary(self, g: _Group) -> RowSet:
        ph = self.phases[g.phase]
        ori = ph["ori"]
        if self._arena is None:
            self._arena = torch.empty(self._arena_bytes, dtype=torch.uint8, device=self.device)
        rows = RowSet(ori.shape[0], g.rays.shape[1], TILE_D, LP_DTYPES[g.precision], g.rescore, self.device,
                      storage=self._arena)
        kernels.project(ph["mp"], g.rays, ori, rows.buffers(0, ori.shape[0]))
        return rows

    def tune(self, sample_queries: int = 4 * 37 * TILE_Q) -> None:
        """Choose each sub-group's launch shape (eager; synchronises)."""
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        for g in self.groups:
            rows = self._dictionary(g)
            n_dict, n_pix = rows.n_rows, rows.n_pix
            for sub in g.subgroups.values():
                n_s = min(sub.n_queries, sample_queries)
                fill = self._fill(sub)
                base = sub.cfg

                def time_shape(shape, n_s=n_s, fill=fill, base=base, sub=sub):
                    cfg = SearchConfig(precision=base.precision, rescore_k=base.rescore_k,
                                       query_chunk=round_up(n_s, TILE_Q), workspace_bytes=_NO_BUDGET_LIMIT, **shape)
                    s = Searcher(n_dict, n_s, n_pix, sub.top_k, cfg, self.device)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    s.run(None, fill, resident=rows)
                    e1.record()
                    torch.cuda.synchronize(self.device)
                    return e0.elapsed_time(e1)

                probe = Searcher(n_dict, 1, n_pix, sub.top_k, base, self.device)
                key = LaunchTuner.key(n_pix, n_dict, g.precision, probe.n_cand, sub.rescore_k > 0, sms)
                shape = self.tuner.pick(key, time_shape)
                sub.cfg = SearchConfig(precision=base.precision, rescore_k=base.rescore_k,
                                       query_chunk=base.query_chunk, workspace_bytes=base.workspace_bytes, **shape)
            del rows
        torch.cuda.empty_cache()
        self._tuned = True

    # --------------------------------------------------------------- execute
    def _enqueue(self):
        """All work of the batch on the current stream, no host sync; returns
        per-map (indices, scores, quaternions) device tensors."""
        self.status.zero_()
        outs: List[Optional[Tuple[torch.Tensor, torch.Tensor, torch.Tensor]]] = [None] * len(self.jobs)
        for g in self.groups:
            ori = self.phases[g.phase]["ori"]
            rows = self._dictionary(g)
            for sub in g.subgroups.values():
                s = Searcher(rows.n_rows, sub.n_queries, rows.n_pix, sub.top_k, sub.cfg, self.device)
                idx, val = s.run(None, self._fill(sub), resident=rows, check=False, status=self.status)
                for j, m in enumerate(sub.maps):
                    a = sub.offsets[j]
                    b = sub.offsets[j + 1] if j + 1 < len(sub.maps) else sub.n_queries
                    quats = kernels.gather_rows(ori, idx[a:b].reshape(-1)).reshape(b - a, sub.top_k, 4)
                    outs[m] = (idx[a:b], val[a:b], quats)
            del rows
        return outs

    def run(self, use_graph: bool = True) -> None:
        """Index every map. The first graph run tunes (if enabled), runs the
        batch eagerly once, then captures it; later runs replay the graph
        (the patterns are read again from the same tensors)."""
        if self.autotune and not self._tuned:
            self.tune()
        if not use_graph:
            outs = self._enqueue()
        else:
            if self.graph is None:
                self._enqueue()
                torch.cuda.synchronize(self.device)
                check_status(self.status)
                # the graph gets its own memory pool: hand the eager run's
                # cached blocks back first so the two do not add up
                torch.cuda.empty_cache()
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph):
                    self._outputs = self._enqueue()
                self.graph = graph
            self.graph.replay()
            outs = self._outputs
        torch.cuda.synchronize(self.device)
        check_status(self.status)
        self._store(outs)

    def _store(self, outs) -> None:
        for m, job in enumerate(self.jobs):
            idx, val, quats = outs[m]
            exp = job.experiment_patterns
            exp.set_raw_indexing_results(quats.clone(), val.clone(), phase_id=0)
            exp.raw_indexing_indices = {0: idx.clone()}
            exp.dictionaries = {0: self.phases[self._phase_of_map[m]]["ori"]}
            exp.combine_indexing_results(higher_is_better=True)

    def release_graph(self) -> None:
        """Drop the captured graph, its memory pool and the dictionary arena."""
        self.graph = None
        self._outputs = None
        self._arena = None
