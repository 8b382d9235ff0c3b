"""Timed baselines that run the reference ebsdtorch itself.

TEST INFRASTRUCTURE ONLY: used by ``bench.py``'s baseline legs (the reference
arm, the ``cpu_baseline`` object and the plain-FP32-GPU-DI comparison). The
product path never imports it. The reference is loaded from ``oracle/_ref``
(staged by ``oracle/stage_ref.py``) through ``oracle/ref_loader.py``.

The indexing baselines call the reference's public
``dictionary_index_orientations`` (ebsdtorch/ebsd/indexing.py:14-211)
unmodified, with its own MasterPattern, EBSDGeometry and ExperimentPatterns
objects; the baselines of the steps either side of indexing (pattern-centre
fitting, preprocessing, grid refinement; end of this file) call the
reference's own functions for those steps the same way, on bounded samples.

The reference's cost of one call is affine in the query count at a fixed
dictionary: T(Q) = alpha + beta * Q, where alpha is the dictionary projection
(qu_apply + grid_sample, indexing.py:107-143) and beta the per-query
preparation + matching + top-k merge. Both scale linearly with the dictionary
size D. A bounded sample therefore times two calls (Q_a and Q_b queries
against the same dictionary), solves for alpha and beta, and rates the full
workload as Q / ((alpha + beta * Q) * D / D_sample).
"""

from __future__ import annotations

import os
import time
from typing import Dict, Optional, Sequence, Tuple

from . import ref_loader


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def _reference_objects(mp_tensor, det, pc=(0.5, 0.5, 0.6), tilts=(0.0, 70.0, 0.0), laue=11):
    from ebsdtorch.ebsd.geometry import EBSDGeometry
    from ebsdtorch.ebsd.master_pattern import MasterPattern

    mp = MasterPattern(mp_tensor, laue_group=laue)
    geom = EBSDGeometry(tuple(det), tilts_degrees=tilts, proj_center=pc).to(mp_tensor.device)
    return mp, geom


def reference_patterns(mp_tensor, det, n: int, mean_counts: float, seed: int):
    """(n, H, W) float32 patterns made by the reference's own projector
    (qu_apply + MasterPattern.interpolate) at seeded uniform orientations,
    scaled to a mean count and Poisson sampled; on mp_tensor's device."""
    import torch
    from ebsdtorch.s2_and_so3.quaternions import qu_apply
    from ebsdtorch.s2_and_so3.sampling import so3_uniform_quat

    mp, geom = _reference_objects(mp_tensor, det)
    dev = mp_tensor.device
    g = torch.Generator().manual_seed(seed)
    state = torch.random.get_rng_state()
    torch.manual_seed(seed)
    quats = so3_uniform_quat(n, torch.device("cpu")).to(dev)
    torch.random.set_rng_state(state)
    with torch.no_grad():
        dc = geom.get_coords_sample_frame(binning=(1, 1))
        dc = dc / dc.norm(dim=-1, keepdim=True)
        out = torch.empty((n, *det), dtype=torch.float32, device=dev)
        for s0 in range(0, n, 256):
            s1 = min(n, s0 + 256)
            x = mp.interpolate(qu_apply(quats[s0:s1, None, :], dc[None]), normalize_coords=False).reshape(
                s1 - s0, *det)
            x = x - x.amin(dim=(1, 2), keepdim=True)
            x = x * (mean_counts / x.mean(dim=(1, 2), keepdim=True).clamp_min(1e-12))
            out[s0:s1] = torch.poisson(x.cpu(), generator=g).to(dev)
    return out


def _call(ref, mp_tensor, det, pats, res, k, dc, ec, match_dtype, quantized, seed=0):
    """One reference dictionary_index_orientations call; returns (seconds,
    ExperimentPatterns)."""
    import torch
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns

    mp, geom = _reference_objects(mp_tensor, det)
    exp = ExperimentPatterns(pats)
    torch.manual_seed(seed)
    if pats.is_cuda:
        torch.cuda.synchronize()
    t0 = time.perf_counter()
    with ref_loader.quiet_stdout():
        ref.dictionary_index_orientations(
            mp, geom, exp, dictionary_resolution_degrees=res, top_k_matches=k, dictionary_chunk_size=dc,
            experiment_chunk_size=ec, match_dtype=match_dtype, quantized_if_x86=quantized)
    if pats.is_cuda:
        torch.cuda.synchronize()
    return time.perf_counter() - t0, exp


def dictionary_size(laue: int, res: float) -> int:
    import torch
    from ebsdtorch.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    return int(sample_ori_fz_laue_angle(laue, res, torch.device("cpu"), permute=False).shape[0])


class CpuSample:
    """The reference's own CPU dictionary indexing on a bounded sample of a
    workload (Q_full patterns of det pixels against D_full rows, top-k).

    Each step() is two reference calls against a `sample_res` dictionary
    (D_s rows): one with q_a patterns and one with q_b; the rate of the full
    workload follows from the affine model in the module docstring."""

    def __init__(self, mp_tensor_cpu, det, q_full: int, d_full: int, k: int, mean_counts: float,
                 sample_res: float = 2.5, q_a: int = 32768, q_b: int = 1024, dc: int = 4096, ec: int = 1024,
                 threads: Optional[int] = None):
        import torch

        self.ref = ref_loader.load_indexing()
        self.threads = threads or host_threads()
        torch.set_num_threads(self.threads)
        self.mp, self.det, self.k = mp_tensor_cpu, tuple(det), k
        self.q_full, self.d_full = q_full, d_full
        self.res, self.q_a, self.q_b, self.dc, self.ec = sample_res, q_a, q_b, dc, ec
        self.d_s = dictionary_size(11, sample_res)
        # 4,096 distinct projected patterns, repeated up to q_a (the cost of a
        # call does not depend on the pixel values)
        base = reference_patterns(mp_tensor_cpu, det, min(q_a, 4096), mean_counts, seed=4242)
        reps = -(-q_a // base.shape[0])
        self.pats = torch.cat([base] * reps)[:q_a].contiguous()

    def step(self, quantized: bool) -> Tuple[float, float]:
        """Seconds of the q_a-pattern call and of the q_b-pattern call."""
        import torch

        t_a, _ = _call(self.ref, self.mp, self.det, self.pats, self.res, self.k, self.dc, self.ec,
                       torch.float32, quantized)
        t_b, _ = _call(self.ref, self.mp, self.det, self.pats[:self.q_b], self.res, self.k, self.dc, self.ec,
                       torch.float32, quantized)
        return t_a, t_b

    def rate(self, t_a: float, t_b: float) -> Dict[str, float]:
        """Full-workload rate from the two call times (affine model)."""
        beta = max(1e-12, (t_a - t_b) / (self.q_a - self.q_b))
        alpha = max(0.0, t_a - beta * self.q_a)
        t_full = (alpha + beta * self.q_full) * self.d_full / self.d_s
        return {"rate": self.q_full / t_full, "t_a": t_a, "t_b": t_b, "projection_s": alpha,
                "per_pattern_s": beta, "t_full": t_full}

    def describe(self) -> str:
        return (f"reference dictionary_index_orientations on the host CPU ({cpu_model()}, {self.threads} threads): "
                f"per step two calls against its own m-3m {self.res} deg dictionary ({self.d_s:,} rows) with "
                f"{self.q_a:,} and {self.q_b:,} patterns of {self.det[0]}x{self.det[1]} px (dictionary chunk "
                f"{self.dc}, experiment chunk {self.ec}, top-{self.k}); projection and per-pattern costs solved "
                f"from the two times and scaled to {self.q_full:,} patterns x {self.d_full:,} rows")


def run_cpu_baseline(mp_tensor_cpu, det, q_full, d_full, k, mean_counts, steps: int, warmup: int,
                     variants: Sequence[bool] = (True, False)) -> Dict:
    """Rate per variant (quantized_if_x86 True = the reference's default
    int8 FBGEMM path, False = float32) over `steps` steps after `warmup`
    untimed ones; variants alternate step by step, and each variant's rate
    comes from the medians of its two call times. `value` is the faster
    variant's rate."""
    import statistics

    s = CpuSample(mp_tensor_cpu, det, q_full, d_full, k, mean_counts)
    times = {v: [] for v in variants}
    for i in range(warmup):
        s.step(variants[i % len(variants)])
    for i in range(max(steps, len(variants))):
        v = variants[i % len(variants)]
        times[v].append(s.step(v))
    fits = {v: s.rate(statistics.median(t[0] for t in ts), statistics.median(t[1] for t in ts))
            for v, ts in times.items() if ts}
    best = max(fits, key=lambda v: fits[v]["rate"])
    name = lambda v: "int8 (quantized_if_x86=True)" if v else "float32 (quantized_if_x86=False)"  # noqa: E731
    return {"value": fits[best]["rate"], "quantized_if_x86": best,
            "by_variant": {name(v): f for v, f in fits.items()},
            "cores": s.threads, "cpu_model": cpu_model(), "sample": s.describe(),
            "steps_per_variant": {name(v): len(ts) for v, ts in times.items()}}


def fp32_gpu_di(mp_tensor, det, pats, res: float, k: int, q_full: int,
                q_sub: Tuple[int, int] = (8192, 16384),
                sweep: Sequence[Tuple[int, int]] = ((1024, 1024), (1024, 4096), (1024, 8192), (4096, 1024),
                                                    (4096, 4096), (4096, 8192), (8192, 1024), (8192, 4096),
                                                    (8192, 8192))) -> Dict:
    """Plain FP32 dictionary indexing on the GPU: the reference's
    dictionary_index_orientations(match_dtype=torch.float32) with TF32 off
    (torch's default), for every (dictionary_chunk_size,
    experiment_chunk_size) of `sweep` on the first q_sub[0] patterns; the
    fastest pair is re-run on q_sub[1] patterns and the full-workload rate
    follows from the affine model. Returns the timings, the rate and the
    reference's top-1 orientations of the first q_sub[0] patterns (fastest
    pair)."""
    import torch

    torch.backends.cuda.matmul.allow_tf32 = False
    ref = ref_loader.load_indexing()
    qa, qb = q_sub
    rows, best, best_exp = [], None, None
    for dc, ec in sweep:
        t, exp = _call(ref, mp_tensor, det, pats[:qa], res, k, dc, ec, torch.float32, False)
        rows.append({"dictionary_chunk_size": dc, "experiment_chunk_size": ec, "seconds": t})
        if best is None or t < best[2]:
            best, best_exp = (dc, ec, t), exp
    top1 = best_exp.raw_indexing_results[0][0][:, 0].clone()
    del best_exp
    t_b, _ = _call(ref, mp_tensor, det, pats[:qb], res, k, best[0], best[1], torch.float32, False)
    beta = max(0.0, (t_b - best[2]) / (qb - qa))
    alpha = max(0.0, best[2] - beta * qa)
    rate = q_full / (alpha + beta * q_full)
    return {"rate": rate, "best_chunks": {"dictionary_chunk_size": best[0], "experiment_chunk_size": best[1]},
            "sweep_at": qa, "sweep": rows, "second_point": {"patterns": qb, "seconds": t_b},
            "projection_s": alpha, "per_pattern_s": beta, "top1_quats": top1}


# ---------------------------------------------------------------------------
# host-CPU baselines of the steps either side of indexing, each a bounded
# sample of the bench's workload run through the reference's own function
# ---------------------------------------------------------------------------

def _all_threads() -> int:
    import torch

    n = host_threads()
    torch.set_num_threads(n)
    return n


def fitting_module():
    """The reference's ebsd/fitting.py. It imports matplotlib (for a plotting
    helper) and, through io/read_master_pattern.py, h5py; the fitter uses
    neither, so empty stand-in modules are registered when they are absent."""
    import sys
    import types

    ref_loader.import_reference()
    for name in ("matplotlib", "matplotlib.pyplot", "h5py"):
        try:
            __import__(name)
        except ImportError:
            sys.modules[name] = types.ModuleType(name)
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    from ebsdtorch.ebsd import fitting

    return fitting


def pcfit_cpu(mp_tensor_cpu, pats_cpu, kw: Dict, z_steps: int) -> Dict:
    """The reference's spatial_fft_pc_fitter (fitting.py:359-540) on the
    host's threads for one pc_z step over the whole dictionary; a fit visits
    z_steps such steps, so the rate is 1 / (seconds * z_steps)."""
    import contextlib
    import io

    F = fitting_module()
    from ebsdtorch.ebsd.master_pattern import MasterPattern

    cores = _all_threads()
    kw1 = dict(kw, pc_z_steps=1, pc_z_max=kw["pc_z_min"])
    mp = MasterPattern(mp_tensor_cpu.clone(), laue_group=11)
    with ref_loader.quiet_stdout(), contextlib.redirect_stderr(io.StringIO()):
        t0 = time.perf_counter()
        F.spatial_fft_pc_fitter(mp, pats_cpu.clone(), **kw1)
        secs = time.perf_counter() - t0
    return {"value": 1.0 / (secs * z_steps), "unit": "fits/s", "cores": cores, "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": "the reference's spatial_fft_pc_fitter on the host CPU (%d threads), one pc_z step over the "
                      "whole dictionary (%.1f s), times %d steps" % (cores, secs, z_steps)}


def preprocess_cpu(counts_cpu, k_rad: int, coeff: float) -> Dict:
    """The reference's standard_clean (experiment_pats.py:285-295) and nlpar
    (nlpar.py:21-192) on the host's threads, on a (scan_h, scan_w, h, w)
    crop of detector counts; rate in patterns/s."""
    ref_loader.import_reference()
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.preprocessing.nlpar import nlpar

    cores = _all_threads()
    sh, sw, h, w = counts_cpu.shape
    t0 = time.perf_counter()
    e = ExperimentPatterns(counts_cpu.reshape(sh * sw, h, w).float().clone())
    e.standard_clean()
    nlpar(e.patterns.view(sh, sw, h, w), k_rad=k_rad, coeff=coeff)
    secs = time.perf_counter() - t0
    return {"value": sh * sw / secs, "unit": "patterns/s", "cores": cores, "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": "the reference's standard_clean + nlpar (k_rad %d) on the host CPU (%d threads), a %d x %d "
                      "crop of the scan (%.1f s)" % (k_rad, cores, sh, sw, secs)}


def refine_cpu(mp_tensor_cpu, det, pats_cpu, start_cpu, semi_edge_deg: float, n_iter: int = 3,
               radius: int = 1) -> Dict:
    """The reference's orientation_grid_refinement (refining.py:71-244) on
    the host's threads, FP32 matching, on the given patterns; patterns/s."""
    import contextlib
    import io

    import torch

    ref_loader.import_reference()
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.ebsd.refining import orientation_grid_refinement

    cores = _all_threads()
    mp, geom = _reference_objects(mp_tensor_cpu, det)
    n = pats_cpu.shape[0]
    exp = ExperimentPatterns(pats_cpu.clone())
    exp.set_orientations(start_cpu.clone())
    exp.phases = torch.zeros(n, dtype=torch.int64)
    with ref_loader.quiet_stdout(), contextlib.redirect_stderr(io.StringIO()):
        t0 = time.perf_counter()
        orientation_grid_refinement(mp, geom, exp, grid_semi_edge_in_degrees=semi_edge_deg, batch_size=n,
                                    n_iter=n_iter, kernel_radius_in_steps=radius, match_dtype=torch.float32)
        secs = time.perf_counter() - t0
    return {"value": n / secs, "unit": "patterns/s", "cores": cores, "kind": "reference", "cpu_model": cpu_model(),
            "sample": "the reference's orientation_grid_refinement on the host CPU (%d threads, FP32), %d patterns "
                      "(%.1f s)" % (cores, n, secs)}
