"""Benchmark: patterns indexed per second, plain dictionary indexing.

Workload (default): 128 x 128 detector (16,384 px), PC (0.5, 0.5, 0.6), 70 deg
tilt; synthetic 2 x 1001 x 1001 modified-Lambert master pattern; m-3m
dictionary at 0.5 deg = 328,720 orientations projected on the fly; 262,144
query patterns (a 512 x 512 map) at mean 100 counts; top-8 per pattern.
A step is one full dictionary_index_orientations call (grid generation,
projection, pattern preparation, tensor-core match with streaming top-k,
FP32 re-score of the best 32 candidates, result write-back). Inputs are far
larger than L2 (17 GB of patterns, 10.8 GB of bf16 dictionary), so no flush
is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload full|small] [--precision bf16|fp8]

Multi-GPU (torchrun, one rank per GPU): every rank indexes its own full map
(replicas, weak scaling, no collective on the data path); the timed region
is bracketed by barriers and the slowest rank's time is reported.

Baselines run the reference itself (staged in oracle/_ref by oracle/stage_ref.py;
the NumPy port in oracle/ only when it is not staged):
  --impl reference   the reference's own CPU dictionary_index_orientations on
                     all host threads, int8 (its default) and float32, on a
                     bounded sample, rated for the full workload
  plain_fp32_di      the reference's own dictionary_index_orientations with
                     match_dtype=float32 on this GPU (chunk-size sweep)
  cpu_baseline       the reference's default CPU path, as --impl reference

Companion objects of the default line: the e4m3 path (with its roofline
against a measured e4m3 GEMM peak), the learned-proposal path (network
trained outside the timed region), the margin-gated FP32 re-score, and, on a
single GPU, PCA DI, grid refinement, preprocessing and pattern-centre
fitting. Each also has a mode of its own (--pca, --refine, --preprocess,
--pcfit, --learned, --batched) printing its line alone.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "patterns indexed/s (128^2, 333k dict) vs plain FP32 DI; % within 0.5deg misori"
UNIT = "patterns/s"

WORKLOADS = {
    "full": dict(name="plain DI 128x128 px, m-3m 0.5deg dictionary (328,720), 262,144 patterns, top-8",
                 mp=1001, det=(128, 128), res=0.5, Q=262144, k=8, counts=100.0),
    "small": dict(name="plain DI 60x60 px, m-3m 1.0deg dictionary (36,829), 4,096 patterns, top-1",
                  mp=257, det=(60, 60), res=1.0, Q=4096, k=1, counts=200.0),
    # profiling case: the full-size kernels' shapes at a few GB of device memory
    "profile": dict(name="plain DI 128x128 px, m-3m 1.0deg dictionary (36,829), 8,192 patterns, top-8",
                    mp=1001, det=(128, 128), res=1.0, Q=8192, k=8, counts=100.0),
    # second profiling case: a larger dictionary, to see how the match kernel's
    # DRAM traffic per launch grows with the dictionary rows
    "profile075": dict(name="plain DI 128x128 px, m-3m 0.75deg dictionary, 8,192 patterns, top-8",
                       mp=1001, det=(128, 128), res=0.75, Q=8192, k=8, counts=100.0),
}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        mhz, maxmhz, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1].split()[0]))
                maxmhz = float(parts[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not mhz:
            return None
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": maxmhz, "reasons": sorted(reasons),
                "samples": len(mhz)}


def _dist():
    import torch.distributed as dist

    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and not dist.is_initialized():
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return dist if dist.is_initialized() else None


def _max_over_ranks(x: float, dist, device) -> float:
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------- CPU port


def cpu_rate(wl, sample_dict=1024, sample_q=256, threads=None):
    """Reference algorithm on the host cores (oracle NumPy port, float32, all
    BLAS threads): times projection of `sample_dict` dictionary rows, query
    preparation of `sample_q` patterns and their dot-product top-k, then
    extrapolates to the full workload (Q patterns against D rows)."""
    import numpy as np

    from ebsdtorch_b200.synthetic import random_quaternions, synthetic_master_pattern
    from oracle import di_oracle as O

    rng = np.random.default_rng(0)
    mp = synthetic_master_pattern(wl["mp"], seed=0).numpy().astype(np.float32)
    h, w = wl["det"]
    rays = O.unit_rays(O.detector_coords_sample_frame((h, w), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0))).astype(np.float32)
    quats = random_quaternions(sample_dict, 7).numpy()
    pats = rng.standard_normal((sample_q, h, w)).astype(np.float32)
    t0 = time.perf_counter()
    d = O.dictionary_rows(mp, rays, quats, dtype=np.float32, chunk=256)
    t1 = time.perf_counter()
    q = O.prep_patterns(pats, dtype=np.float32)
    t2 = time.perf_counter()
    O.topk_dot(q, d, wl["k"], chunk=sample_dict)
    t3 = time.perf_counter()
    D = {0.5: 328720, 1.0: 36829}[wl["res"]]
    t_row = (t1 - t0) / sample_dict
    t_q = (t2 - t1) / sample_q
    t_pair = (t3 - t2) / (sample_q * sample_dict)
    total = D * t_row + wl["Q"] * t_q + wl["Q"] * D * t_pair
    return wl["Q"] / total, (t3 - t0), os.cpu_count() if threads is None else threads


def _reference_staged() -> bool:
    from oracle import ref_loader

    return ref_loader.reference_root() is not None


def _d_full(wl) -> int:
    return {0.5: 328720, 1.0: 36829}[wl["res"]]


def reference_cpu_baseline(wl, steps, warmup, variants=(True, False)):
    """The reference's own CPU dictionary_index_orientations (staged in
    oracle/_ref) on a bounded sample, or the NumPy port when the reference is
    not staged. Returns the cpu_baseline object."""
    if _reference_staged():
        from ebsdtorch_b200.synthetic import synthetic_master_pattern
        from oracle import ref_baselines as RB

        mp = synthetic_master_pattern(wl["mp"], seed=0)
        r = RB.run_cpu_baseline(mp, wl["det"], wl["Q"], _d_full(wl), wl["k"], wl["counts"], steps, warmup,
                                variants=variants)
        return {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                "sample": r["sample"], "cpu_model": r["cpu_model"], "quantized_if_x86": r["quantized_if_x86"],
                "by_variant": {k: {"rate": v["rate"], "t_a_s": v["t_a"], "t_b_s": v["t_b"],
                                   "projection_s": v["projection_s"], "per_pattern_s": v["per_pattern_s"]}
                               for k, v in r["by_variant"].items()},
                "steps_per_variant": r["steps_per_variant"]}
    rates = []
    for i in range(warmup + steps):
        rr, secs, cores = cpu_rate(wl)
        if i >= warmup:
            rates.append(rr)
    return {"value": statistics.median(rates), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"{wl['name']}: per step 1,024 dictionary rows projected and 256 patterns matched against "
                       "them (oracle NumPy float32 port; the reference is not staged), rate extrapolated to the "
                       "full workload")}


def run_reference(args, wl):
    dist = _dist()
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = reference_cpu_baseline(wl, args.steps, args.warmup)
    v = cb["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": wl["Q"] / v * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("int8 (FBGEMM dynamic quantization)" if cb.get("quantized_if_x86") else "f32"),
        "data": "synthetic",
        "config": {"workload": wl["name"], "l2": "inputs larger than L2"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm


def _reference_rows_torch(mp, rays, quats):
    """Dictionary rows exactly as the reference builds them, in torch eager
    ops: qu_apply (quaternions.py:186-213), rosca_lambert_side_by_side
    (sphere.py:145-185), grid_sample bilinear / border / align_corners=False
    (master_pattern.py:197-206), row mean subtraction (indexing.py:139-143)."""
    import math

    import torch

    w, x, y, z = (quats[:, None, i] for i in range(4))
    vx, vy, vz = rays[0][None], rays[1][None], rays[2][None]
    iw = w - x * vx - y * vy - z * vz
    ix = w * vx + x + y * vz - z * vy
    iy = w * vy - x * vz + y + z * vx
    iz = w * vz + x * vy - y * vx + z
    ox = -iw * x + ix * w - iy * z + iz * y
    oy = -iw * y + ix * z + iy * w - iz * x
    oz = -iw * z - ix * y + iy * x + iz * w
    fac = torch.sqrt(torch.clamp(2.0 * (1.0 - oz.abs()), min=0.0))
    cond = oy.abs() <= ox.abs()
    big, sml = torch.where(cond, ox, oy), torch.where(cond, oy, ox)
    sgn = torch.where(big < 0, -1.0, 1.0)
    simple = sgn * fac * (2.0 / 8.0 ** 0.5)
    arct = sgn * fac * torch.atan2(sml * sgn, big.abs()) * (2.0 * 2.0 ** 0.5 / math.pi)
    u = torch.where(cond, simple, arct) / 2.0 - 0.5 + torch.where(oz < 0, 1.0, 0.0)
    v = torch.where(cond, arct, simple)
    grid = torch.stack((u, v), dim=-1)[None]
    out = torch.nn.functional.grid_sample(mp[None, None], grid, mode="bilinear", padding_mode="border",
                                          align_corners=False)[0, 0]
    return out - out.mean(dim=-1, keepdim=True)


def plain_fp32_gpu_di(wl, mp, rays, dictionary, queries_f32, k, chunk=8192, return_values=False):
    """The reference's plain FP32 DI loop on the GPU (torch eager, TF32 off):
    per dictionary chunk, project it, then query @ chunk.T in FP32, chunk
    top-k and a running top-k merge (knn.py:80-103, 219-266). Returns
    (indices (Q, k), seconds spent projecting, seconds spent matching), and
    the sorted FP32 values as a fourth item with return_values."""
    import torch

    torch.backends.cuda.matmul.allow_tf32 = False
    Q = queries_f32.shape[0]
    best_v = torch.full((Q, k), -float("inf"), device=queries_f32.device)
    best_i = torch.zeros((Q, k), dtype=torch.int64, device=queries_f32.device)
    t_proj = t_match = 0.0
    for d0 in range(0, dictionary.shape[0], chunk):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rows = _reference_rows_torch(mp, rays, dictionary[d0:d0 + chunk])
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        sim = queries_f32 @ rows.t()
        v, i = torch.topk(sim, min(k, rows.shape[0]), dim=1, largest=True, sorted=False)
        allv, alli = torch.cat((best_v, v), 1), torch.cat((best_i, i + d0), 1)
        sel = torch.topk(allv, k, dim=1, largest=True, sorted=False)[1]
        best_v, best_i = torch.gather(allv, 1, sel), torch.gather(alli, 1, sel)
        torch.cuda.synchronize()
        t_proj += t1 - t0
        t_match += time.perf_counter() - t1
    order = torch.topk(best_v, k, dim=1, largest=True, sorted=True)[1]
    if return_values:
        return torch.gather(best_i, 1, order), t_proj, t_match, torch.gather(best_v, 1, order)
    return torch.gather(best_i, 1, order), t_proj, t_match


# DRAM bytes (read + write) of one one-wave match launch (18 query tiles,
# 2,304 queries, against the whole dictionary, bf16 rows of 128^2 px),
# captured with ncu (dram__bytes_read.sum + dram__bytes_write.sum) at two
# dictionary sizes. The traffic is affine in the dictionary rows; the full
# launch's figure is its extrapolation.
MATCH_DRAM_BYTES = ((36829, 2549037056 + 3763456), (89312, 6199060224 + 5258240))
MATCH_WAVE_QUERIES = 2304


def match_traffic_estimate(d_rows: int) -> float:
    (d1, b1), (d2, b2) = MATCH_DRAM_BYTES
    return b1 + (b2 - b1) * (d_rows - d1) / (d2 - d1)


def gemm_peak_tflops(kind: str, dev, seconds: float = 3.0, n: int = 8192) -> dict:
    """Library GEMM throughput on this GPU, the denominator for a kernel of
    the same element type: cuBLASLt e4m3 x e4m3 -> bf16 (torch._scaled_mm,
    per-tensor scales) or bf16 x bf16 (torch.matmul), n^3. `burst`: 50
    calls after warm-up; `sustained`: calls repeated for `seconds` (the power
    cap settles), rate of the last two thirds. CUDA events throughout."""
    import torch

    g = torch.Generator(device=dev).manual_seed(0)
    a = torch.randn((n, n), device=dev, generator=g)
    b = torch.randn((n, n), device=dev, generator=g)
    if kind == "e4m3":
        a8, b8 = a.to(torch.float8_e4m3fn), b.to(torch.float8_e4m3fn).t()
        one = torch.ones((), device=dev)

        def f():
            return torch._scaled_mm(a8, b8, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
    else:
        a16, b16 = a.bfloat16(), b.bfloat16()

        def f():
            return a16 @ b16
    del a, b
    flop = 2.0 * n ** 3
    for _ in range(10):
        f()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(50):
        f()
    e1.record()
    torch.cuda.synchronize()
    burst = 50 * flop / (e0.elapsed_time(e1) / 1e3) / 1e12
    marks = []
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        marks.append(ev)
        for _ in range(100):
            f()
        torch.cuda.synchronize()
    ev = torch.cuda.Event(enable_timing=True)
    ev.record()
    marks.append(ev)
    torch.cuda.synchronize()
    first = len(marks) // 3
    sustained = (len(marks) - 1 - first) * 100 * flop / (marks[first].elapsed_time(marks[-1]) / 1e3) / 1e12
    return {"burst": burst, "sustained": sustained, "how": f"{kind} {n}^3 cuBLASLt GEMM via torch, CUDA events, "
                                                          f"{seconds:.0f} s loop for the sustained rate"}


def learned_block(args, wl, mp, geom, pats, exp_plain, ref_top1, n_sub, dist, dev):
    """Companion measurement of the learned path on the headline run's own
    patterns: the proposal network is trained first (outside the timed
    region), then learned proposal + coarse-to-fine local DI + plain-DI
    fallback is timed over `args.steps` calls, patterns resident in HBM, and
    once more end to end from pinned host memory. Agreement is measured
    against this run's plain DI (whose top-1 is the FP32 top-1) and, on the
    first n_sub patterns, against the reference's FP32 GPU DI."""
    import torch

    from ebsdtorch_b200.ebsd import ExperimentPatterns
    from ebsdtorch_b200.learned import train_proposal_cnn
    from ebsdtorch_b200.local_search import learned_dictionary_index
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    t0 = time.perf_counter()
    model, losses = train_proposal_cnn(mp.master_pattern, geom, 11, steps=args.train_steps, batch=256, lr=1e-3,
                                       mean_counts=wl["counts"], seed=0)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    pyramid = tuple(float(v) for v in args.pyramid.split(",") if v)
    kw = dict(dictionary_resolution_degrees=wl["res"], max_angle_deg=args.max_angle,
              pyramid_resolutions_deg=pyramid, fallback_ratio=args.fallback_ratio, stage_margin=args.stage_margin)
    exp = ExperimentPatterns(pats)

    def step():
        torch.manual_seed(0)
        return learned_dictionary_index(mp, geom, exp, model, **kw)

    for _ in range(max(1, min(args.warmup, 3))):
        step()
    torch.cuda.synchronize()
    _barrier(dist)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        st = step()
    e1.record()
    torch.cuda.synchronize()
    _barrier(dist)
    t = _max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, dev)
    n = args.gpus
    ours_q = exp.orientations.float().contiguous()
    ang = disori_angle_laue(ours_q, exp_plain.orientations.float().contiguous(), 11, 11)
    out = {"value": n * wl["Q"] * args.steps / t, "unit": UNIT, "ms_per_step": t / args.steps * 1e3,
           "within_0.5deg_of_plain_di": float((ang < math.radians(0.5)).float().mean()),
           "same_top1_index_as_plain_di": float((exp.raw_indexing_indices[0][:, 0] ==
                                                 exp_plain.raw_indexing_indices[0][:, 0]).float().mean()),
           "fallback_fraction": st.n_fallback / st.n_patterns, "stage_radii_deg": st.stage_radii_deg,
           "stage_mean_candidates": st.stage_mean_candidates, "stage_seconds": st.seconds,
           "train_seconds_untimed": t_train, "train_patterns": 256 * args.train_steps,
           "final_train_loss": float(losses[-100:].mean()),
           "how": "CNN proposal (bf16, own kernels) + local DI within %.1f deg on the %s deg dictionaries, then the "
                  "full one, + plain-DI fallback below %.2f x the map median" % (args.max_angle, args.pyramid,
                                                                                args.fallback_ratio)}
    if ref_top1 is not None:
        a = disori_angle_laue(ours_q[:n_sub].contiguous(), ref_top1, 11, 11)
        out["within_0.5deg_of_reference_fp32_di"] = float((a < math.radians(0.5)).float().mean())
        out["reference_subset"] = n_sub
    if not args.no_e2e:
        try:
            host = torch.empty(pats.shape, dtype=pats.dtype, pin_memory=True)
            host.copy_(pats)
        except RuntimeError:
            host = pats.cpu()
        exp_h = ExperimentPatterns(host)
        ori_host = torch.empty((wl["Q"], 4), dtype=torch.float32, pin_memory=True)
        torch.manual_seed(0)
        learned_dictionary_index(mp, geom, exp_h, model, **kw)
        torch.cuda.synchronize()
        _barrier(dist)
        h0 = time.perf_counter()
        e2e_steps = max(1, args.steps // 2)
        for _ in range(e2e_steps):
            torch.manual_seed(0)
            learned_dictionary_index(mp, geom, exp_h, model, **kw)
            ori_host.copy_(exp_h.orientations.float(), non_blocking=True)
        torch.cuda.synchronize()
        _barrier(dist)
        th = _max_over_ranks(time.perf_counter() - h0, dist, dev)
        out["e2e"] = {"value": n * wl["Q"] * e2e_steps / th, "unit": UNIT,
                      "h2d_bytes_per_step": int(host.numel() * host.element_size()),
                      "d2h_bytes_per_step": int(ori_host.numel() * 4), "host_memory": "pinned"}
        del exp_h, host
    del exp, model
    return out


def run_ours(args, wl):
    import torch

    from ebsdtorch_b200 import _capi, engine, synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations

    dist = _dist()
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    _capi.load()

    mp = MasterPattern(synthetic.synthetic_master_pattern(wl["mp"], seed=0, device=dev), laue_group=11)
    geom = EBSDGeometry(wl["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    truth = synthetic.random_quaternions(wl["Q"], 1000 + rank).to(dev)
    pats = synthetic.synthetic_patterns(mp.master_pattern, geom, truth, mean_counts=wl["counts"], seed=2000 + rank)
    exp = ExperimentPatterns(pats)
    kw = dict(dictionary_resolution_degrees=wl["res"], top_k_matches=wl["k"], match_dtype=torch.float32,
              precision=args.precision, rescore_k=32)

    def step():
        torch.manual_seed(0)
        dictionary_index_orientations(mp, geom, exp, **kw)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region: patterns resident in HBM ----
    engine.MATCH_TIMERS, engine.MERGE_TIMERS = [], []
    launches0 = _capi.launch_count
    with ClockSampler(local) as clocks:
        _barrier(dist)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        _barrier(dist)
    launches = (_capi.launch_count - launches0) // args.steps
    elapsed = e0.elapsed_time(e1) / 1e3
    t_max = _max_over_ranks(elapsed, dist, dev)
    n = args.gpus
    value = n * wl["Q"] * args.steps / t_max
    timers = engine.MATCH_TIMERS
    merge_ms = sum(a.elapsed_time(b) for a, b in engine.MERGE_TIMERS)
    engine.MATCH_TIMERS = engine.MERGE_TIMERS = None
    # rows the margin-gated FP32 re-score reads (one untimed call with the counter)
    counter = torch.zeros(1, dtype=torch.int64, device=dev)
    engine.RESCORE_COUNTER = counter
    step()
    torch.cuda.synchronize()
    engine.RESCORE_COUNTER = None
    rows_per_query = int(counter.item()) / wl["Q"]
    n_pix = int(wl["det"][0] * wl["det"][1])
    rescore = {"share_of_step": merge_ms / 1e3 / elapsed, "rows_rescored_per_query": rows_per_query,
               "rows_cap": 32, "bytes_per_query": (rows_per_query + 1) * n_pix * 4,
               "achieved_gbs": wl["Q"] * args.steps * (rows_per_query + 1) * n_pix * 4 / (merge_ms / 1e3) / 1e9,
               "how": "merge + margin-gated FP32 re-score (k_merge_rescore); bytes = FP32 rows re-scored + the "
                      "query row, per query"}
    match_ms = [a.elapsed_time(b) for a, b, _ in timers]
    match_flops = [f for _, _, f in timers]
    avg_launch_s = sum(match_ms) / len(match_ms) / 1e3
    achieved_tflops = (sum(match_flops) / len(match_flops)) / avg_launch_s / 1e12
    match_share = sum(match_ms) / 1e3 / elapsed
    n_dict_rows = int(exp.dictionaries[0].shape[0])
    # the captures were of 128^2 bf16 rows: no figure for other row lengths
    traffic = match_traffic_estimate(n_dict_rows) if (args.precision == "bf16" and
                                                      tuple(wl["det"]) == (128, 128)) else None

    # accuracy vs the true orientations (reported, cheap)
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    ang = disori_angle_laue(exp.orientations.float().contiguous(), truth, 11, 11)
    within_half = float((ang < torch.deg2rad(torch.tensor(0.5))).float().mean())
    median_deg = float(torch.rad2deg(torch.median(ang)))

    # plain FP32 GPU DI (the reference algorithm in torch eager) on a query
    # subset: agreement of our top-1 with it, and its extrapolated rate
    fp32_cmp = None
    ref_top1 = None  # the FP32 comparison's top-1 orientations of the first n_sub patterns
    if not args.no_fp32_compare:
        n_sub = min(wl["Q"], args.fp32_subset)
        ori = exp.dictionaries[0]
        ours_q = exp.raw_indexing_results[0][0][:n_sub, 0].float().contiguous()
        if _reference_staged():
            # the reference's own dictionary_index_orientations(match_dtype=float32)
            # on this GPU, chunk sweep + two-point fit (oracle/ref_baselines.py)
            from oracle import ref_baselines as RB

            torch.cuda.empty_cache()

            r = RB.fp32_gpu_di(mp.master_pattern, tuple(wl["det"]), pats, wl["res"], wl["k"], wl["Q"],
                               q_sub=(n_sub, 2 * n_sub))
            ref_top1 = r.pop("top1_quats").float().contiguous()
            fp32_rate = r["rate"]
            a = disori_angle_laue(ours_q, ref_top1, 11, 11)
            same_idx = float(((ours_q - ref_top1).abs().amax(dim=1) < 1e-5).float().mean())
            how = ("the reference's own dictionary_index_orientations(match_dtype=torch.float32, TF32 off) on the "
                   f"same GPU: chunk sweep on {n_sub} patterns, fastest pair re-run on {2 * n_sub}, full-workload "
                   "rate from the affine fit (projection + per-pattern cost)")
            extra = {k: r[k] for k in ("best_chunks", "sweep", "second_point", "projection_s", "per_pattern_s")}
        else:
            from ebsdtorch_b200 import kernels
            from ebsdtorch_b200.ebsd.indexing import _unit_rays_soa
            from ebsdtorch_b200.kernels import RowBuffers

            rays = _unit_rays_soa(geom, 1, None, dev)
            q_sub = torch.empty((n_sub, rays.shape[1]), dtype=torch.float32, device=dev)
            kernels.prep_patterns(pats[:n_sub], RowBuffers(f32=q_sub))
            ref_idx, t_proj, t_match = plain_fp32_gpu_di(wl, mp.master_pattern, rays, ori, q_sub, 1)
            ref_top1 = ori[ref_idx[:, 0]].contiguous()
            a = disori_angle_laue(ours_q, ref_top1, 11, 11)
            same_idx = float((exp.raw_indexing_indices[0][:n_sub, 0] == ref_idx[:, 0]).float().mean())
            fp32_rate = wl["Q"] / (t_proj + t_match * wl["Q"] / n_sub)
            how = ("reference algorithm restated in torch eager ops (FP32, TF32 off; the reference is not staged), "
                   "dictionary chunks of 8192, timed on the same GPU for a query subset and extrapolated")
            extra = {}
            del q_sub
        agree = float((a < torch.deg2rad(torch.tensor(0.5))).float().mean())
        fp32_cmp = {"within_0.5deg_of_plain_fp32_di": agree, "same_top1_orientation": same_idx, "subset": n_sub,
                    "plain_fp32_gpu_di_rate": fp32_rate, "speedup_vs_plain_fp32_gpu_di": value / n / fp32_rate,
                    "how": how, **extra}

    # ---- the e4m3 path on the same patterns (device-resident, same timing) ----
    fp8 = None
    if args.precision == "bf16" and not args.no_fp8:
        exp8 = ExperimentPatterns(pats)
        kw8 = dict(kw, precision="fp8")

        def step8():
            torch.manual_seed(0)
            dictionary_index_orientations(mp, geom, exp8, **kw8)

        step8()
        torch.cuda.synchronize()
        _barrier(dist)
        engine.MATCH_TIMERS = []
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(args.steps):
            step8()
        f1.record()
        torch.cuda.synchronize()
        _barrier(dist)
        t8 = _max_over_ranks(f0.elapsed_time(f1) / 1e3, dist, dev)
        timers8, engine.MATCH_TIMERS = engine.MATCH_TIMERS, None
        ms8 = [a.elapsed_time(b) for a, b, _ in timers8]
        fl8 = [f for _, _, f in timers8]
        ach8 = (sum(fl8) / len(fl8)) / (sum(ms8) / len(ms8) / 1e3) / 1e12
        try:
            pk8 = gemm_peak_tflops("e4m3", dev)
        except Exception as exc:  # torch._scaled_mm unavailable: no measured e4m3 denominator
            pk8 = {"sustained": None, "burst": None, "how": f"not measured ({exc})"}
        i8 = exp8.raw_indexing_indices[0][:, 0]
        fp8 = {"value": n * wl["Q"] * args.steps / t8, "unit": UNIT, "ms_per_step": t8 / args.steps * 1e3,
               "same_top1_index_as_bf16": float((i8 == exp.raw_indexing_indices[0][:, 0]).float().mean()),
               "precision": "e4m3 match (per-row absmax scale) + FP32 re-score of top-32",
               "roofline": {"bound": "tensor", "achieved": ach8, "peak": pk8["sustained"], "unit": "TFLOP/s",
                            "frac": ach8 / pk8["sustained"] if pk8["sustained"] else None,
                            "kernel": "k_tc_gemm kind::f8f6f4 (match + top-k)",
                            "peak_source": "measured here: " + pk8["how"], "peak_burst": pk8["burst"],
                            "share_of_step": sum(ms8) / 1e3 / t8}}
        if fp32_cmp is not None:
            q8 = exp8.raw_indexing_results[0][0][:n_sub, 0].float().contiguous()
            fp8["same_top1_orientation_as_plain_fp32_di"] = float(
                ((q8 - ref_top1).abs().amax(dim=1) < 1e-5).float().mean())
            fp8["within_0.5deg_of_plain_fp32_di"] = float(
                (disori_angle_laue(q8, ref_top1, 11, 11) < torch.deg2rad(torch.tensor(0.5))).float().mean())
            fp8["speedup_vs_plain_fp32_gpu_di"] = fp8["value"] / n / fp32_cmp["plain_fp32_gpu_di_rate"]
        del exp8

    # ---- the learned path on the same patterns (training untimed) ----
    learned = None
    if not args.no_learned and tuple(wl["det"]) == (128, 128):
        learned = learned_block(args, wl, mp, geom, pats, exp, ref_top1, n_sub if fp32_cmp else 0, dist, dev)

    # ---- companion measurements of the other rows (single GPU): PCA DI and
    # grid refinement on this run's own patterns, preprocessing and pattern-
    # centre fitting on their own small workloads ----
    companions = None
    if not args.no_companions and n == 1 and tuple(wl["det"]) == (128, 128):
        di_ori = exp.orientations.clone()
        companions = {"pca": pca_block(args, wl, mp, geom, truth, pats, dev),
                      "refine": refine_block(args, wl, mp, geom, truth, pats, di_ori, dev, min(args.steps, 3))}
        del di_ori
        # the companions' CPU baselines only where the reference itself runs
        # (bounded samples of a few seconds each)
        short = argparse.Namespace(**{**vars(args), "no_cpu_baseline": args.no_cpu_baseline or
                                      not _reference_staged()})
        companions["preprocess"] = run_preprocess(short)
        companions["pcfit"] = run_pcfit(short)

    # ---- end to end: host (pinned) patterns, H2D + D2H inside the timed region ----
    e2e = None
    if not args.no_e2e:
        try:
            host = torch.empty(pats.shape, dtype=torch.float32, pin_memory=True)
            host.copy_(pats)
            pinned = True
        except RuntimeError:
            host = pats.cpu()
            pinned = False
        del exp
        exp_h = ExperimentPatterns(host)
        # one untimed call through the host path (side stream, staging buffers)
        torch.manual_seed(0)
        dictionary_index_orientations(mp, geom, exp_h, **kw)
        torch.cuda.synchronize()
        _barrier(dist)
        t0 = time.perf_counter()
        e2e_steps = max(1, args.steps // 2)
        for _ in range(e2e_steps):
            torch.manual_seed(0)
            dictionary_index_orientations(mp, geom, exp_h, **kw)
            q_out = exp_h.raw_indexing_results[0][0].cpu()
            m_out = exp_h.raw_indexing_results[0][1].cpu()
        torch.cuda.synchronize()
        _barrier(dist)
        t_e2e = _max_over_ranks(time.perf_counter() - t0, dist, dev)
        e2e = {"value": n * wl["Q"] * e2e_steps / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": int(host.numel() * 4),
               "d2h_bytes_per_step": int(q_out.numel() * 4 + m_out.numel() * 4),
               "host_memory": "pinned" if pinned else "pageable"}
        del host, exp_h

    peaks, peak_kind = _peaks()
    peak = peaks.get("bf16_tflops_sustained", 1400.0)
    if args.precision == "fp8":
        peak = 2.0 * peak  # no measured fp8 denominator: twice the measured bf16
    # the same kind of cuBLAS GEMM timed on this GPU in this run, under the
    # same power cap: a second denominator beside the contract's peak
    here = None
    if n == 1 and args.precision == "bf16" and not args.no_companions:
        try:
            pk16 = gemm_peak_tflops("bf16", dev)
            here = {"sustained": pk16["sustained"], "burst": pk16["burst"], "how": pk16["how"],
                    "frac_of_sustained": achieved_tflops / pk16["sustained"]}
        except Exception as exc:
            here = {"sustained": None, "how": f"not measured ({exc})"}
    clk = clocks.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": {"workload": wl["name"], "precision": f"{args.precision} match + FP32 re-score of top-32",
                   "parallelism": f"replicas x{n} (query maps independent)", "l2": "inputs larger than L2"},
        "e2e": e2e,
        "gpu_launches": int(launches * args.steps),
        "roofline": {"bound": "tensor", "achieved": achieved_tflops, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved_tflops / peak, "traffic": traffic,
                     "traffic_source": ("ncu DRAM bytes of one-wave launches at 36,829 and 89,312 dictionary rows, "
                                        "extrapolated (affine in the rows) to %d rows; per one-wave launch of %d "
                                        "queries" % (n_dict_rows, MATCH_WAVE_QUERIES)) if traffic is not None else None,
                     "algorithmic_bytes": ((n_dict_rows + MATCH_WAVE_QUERIES) * 128 * 128 * 2
                                           if traffic is not None else None),
                     "kernel": "k_tc_gemm (match + streaming top-k)",
                     "peak_source": f"{peak_kind} bf16_tflops_sustained" + (" x2 for fp8" if args.precision == "fp8"
                                                                             else ""),
                     "peak_measured_here": here,
                     "share_of_step": match_share},
        "rescore": rescore,
        "accuracy": {"within_0.5deg_of_truth": within_half, "median_misori_deg": median_deg},
        "plain_fp32_di": fp32_cmp,
        "fp8": fp8,
        "learned": learned,
        "companions": companions,
        "clocks": clk,
    }
    if rank == 0 and n == 1 and not args.no_cpu_baseline:
        # the reference's default CPU path (int8 quantized matching), the same
        # routine as --impl reference with one warm-up and two timed steps
        line["cpu_baseline"] = reference_cpu_baseline(wl, steps=2, warmup=1, variants=(True,))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_learned(args, wl):
    """Learned proposal + local search + plain-DI fallback on the full
    workload (the CNN is trained first on freshly projected patterns)."""
    import torch

    from ebsdtorch_b200 import _capi, synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations
    from ebsdtorch_b200.learned import train_proposal_cnn
    from ebsdtorch_b200.local_search import learned_dictionary_index

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    _capi.load()
    mp_t = synthetic.synthetic_master_pattern(wl["mp"], seed=0, device=dev)
    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry(wl["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    t0 = time.perf_counter()
    model, losses = train_proposal_cnn(mp_t, geom, 11, steps=args.train_steps, batch=256, lr=1e-3,
                                       mean_counts=wl["counts"], seed=0)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    truth = synthetic.random_quaternions(wl["Q"], 5000).to(dev)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=wl["counts"], seed=5001)
    exp = ExperimentPatterns(pats)
    pyramid = tuple(float(v) for v in args.pyramid.split(",") if v)
    for _ in range(args.warmup):
        torch.manual_seed(0)
        learned_dictionary_index(mp, geom, exp, model, dictionary_resolution_degrees=wl["res"],
                                 max_angle_deg=args.max_angle, pyramid_resolutions_deg=pyramid,
                                 fallback_ratio=args.fallback_ratio, stage_margin=args.stage_margin)
    torch.cuda.synchronize()
    with ClockSampler(int(dev.index or 0)) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            torch.manual_seed(0)
            st = learned_dictionary_index(mp, geom, exp, model, dictionary_resolution_degrees=wl["res"],
                                          max_angle_deg=args.max_angle, pyramid_resolutions_deg=pyramid,
                                          fallback_ratio=args.fallback_ratio, stage_margin=args.stage_margin)
        e1.record()
        torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3 / args.steps
    learned_idx = exp.raw_indexing_indices[0][:, 0].clone()
    # end to end: patterns in pinned host memory, orientations read back
    e2e = None
    if not args.no_e2e:
        exp_h = ExperimentPatterns(pats.cpu().pin_memory())
        ori_host = torch.empty((wl["Q"], 4), dtype=torch.float32).pin_memory()
        torch.manual_seed(0)
        learned_dictionary_index(mp, geom, exp_h, model, dictionary_resolution_degrees=wl["res"],
                                 max_angle_deg=args.max_angle, pyramid_resolutions_deg=pyramid,
                                 fallback_ratio=args.fallback_ratio, stage_margin=args.stage_margin)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            torch.manual_seed(0)
            learned_dictionary_index(mp, geom, exp_h, model, dictionary_resolution_degrees=wl["res"],
                                     max_angle_deg=args.max_angle, pyramid_resolutions_deg=pyramid,
                                     fallback_ratio=args.fallback_ratio, stage_margin=args.stage_margin)
            ori_host.copy_(exp_h.orientations.float(), non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e = {"value": wl["Q"] / (e0.elapsed_time(e1) / 1e3 / args.steps), "unit": UNIT,
               "h2d_bytes_per_step": int(pats.numel() * pats.element_size()),
               "d2h_bytes_per_step": int(ori_host.numel() * 4), "host_memory": "pinned"}
        del exp_h
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    perr = torch.rad2deg(disori_angle_laue(exp.proposals.contiguous(), truth.float().contiguous(), 11, 11))
    prop_err = {f"p{q}": float(torch.quantile(perr, q / 100.0)) for q in (50, 90, 99)}
    prop_err["frac_within_max_angle"] = float((perr <= args.max_angle).float().mean())
    # plain DI on the same patterns (bf16 + FP32 re-score == FP32 DI top-1)
    exp_f = ExperimentPatterns(pats)
    torch.manual_seed(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dictionary_index_orientations(mp, geom, exp_f, dictionary_resolution_degrees=wl["res"], top_k_matches=1,
                                  match_dtype=torch.float32)
    torch.cuda.synchronize()
    t_full = time.perf_counter() - t0
    ang = disori_angle_laue(exp.orientations.float().contiguous(), exp_f.orientations.float().contiguous(), 11, 11)
    # local cosine / map median before the fallback, for patterns that agree
    # with plain DI and for those that do not (how the threshold separates them)
    ratio = exp.local_cosine_ratio
    miss = ang >= math.radians(0.5)
    qs = torch.tensor([0.01, 0.05, 0.5, 0.95, 0.99], device=ratio.device)
    ratio_q = {"agree": [round(float(v), 4) for v in torch.quantile(ratio[~miss], qs)] if bool((~miss).any()) else [],
               "miss": [round(float(v), 4) for v in torch.quantile(ratio[miss], qs)] if bool(miss.any()) else []}
    line = {
        "metric": METRIC, "value": wl["Q"] / secs, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
        "config": {"workload": "learned proposal + coarse-to-fine local DI (<= %.1f deg of the proposal on the %s deg "
                               "dictionaries, then the full one) + plain-DI fallback; " % (args.max_angle, args.pyramid)
                               + wl["name"], "train_steps": args.train_steps, "train_batch": 256,
                   "train_patterns": 256 * args.train_steps},
        "learned": {"within_0.5deg_of_plain_di": float((ang < math.radians(0.5)).float().mean()),
                    "same_top1_index_as_plain_di": float((learned_idx == exp_f.raw_indexing_indices[0][:, 0])
                                                         .float().mean()),
                    "fallback_fraction": st.n_fallback / st.n_patterns, "mean_candidates": st.mean_candidates,
                    "stage_radii_deg": st.stage_radii_deg, "stage_mean_candidates": st.stage_mean_candidates,
                    "proposal_error_deg": prop_err, "fallback_ratio": args.fallback_ratio,
                    "stage_margin_cells": args.stage_margin,
                    "cosine_over_median_q01_05_50_95_99": ratio_q,
                    "stage_seconds": st.seconds, "train_seconds": t_train,
                    "final_train_loss": float(losses[-100:].mean()),
                    "plain_di_seconds_same_gpu": t_full, "speedup_vs_plain_di_bf16": t_full / secs},
        "e2e": e2e,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def run_refine(args, wl):
    import torch

    from ebsdtorch_b200 import _capi
    from ebsdtorch_b200.ebsd import ExperimentPatterns, dictionary_index_orientations

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    _capi.load()
    mp, geom, truth, pats = _full_workload_inputs(wl, dev)
    exp = ExperimentPatterns(pats)
    torch.manual_seed(0)
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=wl["res"], top_k_matches=1,
                                  match_dtype=torch.float32)
    print(json.dumps(refine_block(args, wl, mp, geom, truth, pats, exp.orientations.clone(), dev, args.steps)),
          flush=True)


def refine_block(args, wl, mp, geom, truth, pats, di_ori, dev, steps) -> dict:
    """Orientation grid refinement after DI on the full workload: the timed
    refinement of every pattern from its DI orientation
    (orientation_grid_refinement, radius 1 (27 candidates), 3 iterations,
    semi-edge = the dictionary resolution, left FZ reduction)."""
    import torch

    from ebsdtorch_b200.ebsd import ExperimentPatterns, orientation_grid_refinement
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    exp = ExperimentPatterns(pats)
    exp.phases = torch.zeros(pats.shape[0], dtype=torch.uint8, device=pats.device)  # one phase, as after DI
    before = torch.rad2deg(disori_angle_laue(di_ori.float().contiguous(), truth, 11, 11))
    kw = dict(grid_semi_edge_in_degrees=wl["res"], batch_size=wl["Q"], n_iter=3, kernel_radius_in_steps=1,
              fz_reduction="left")
    for _ in range(max(1, min(args.warmup, 3))):
        exp.set_orientations(di_ori.clone())
        orientation_grid_refinement(mp, geom, exp, **kw)
    torch.cuda.synchronize()
    with ClockSampler(int(dev.index or 0)) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total = 0.0
        for _ in range(steps):
            exp.set_orientations(di_ori.clone())
            torch.cuda.synchronize()
            e0.record()
            orientation_grid_refinement(mp, geom, exp, **kw)
            e1.record()
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1) / 1e3
    secs = total / steps
    after = torch.rad2deg(disori_angle_laue(exp.orientations.float().contiguous(), truth, 11, 11))
    n_pix = wl["det"][0] * wl["det"][1]
    samples = wl["Q"] * 27 * 3 * n_pix
    line = {
        "metric": "patterns refined/s (orientation grid refinement after DI)", "value": wl["Q"] / secs,
        "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": secs * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "grid refinement (radius 1 = 27 candidates, 3 iterations, semi-edge %.2f deg, "
                               "left FZ reduction) of plain-DI results; " % wl["res"] + wl["name"]},
        "simulated_samples_per_s": samples / secs,
        "misorientation_to_truth_deg": {"di_median": float(before.median()), "refined_median": float(after.median()),
                                        "di_within_0.5": float((before < 0.5).float().mean()),
                                        "refined_within_0.5": float((after < 0.5).float().mean())},
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline and _reference_staged():
        from oracle import ref_baselines as RB

        m = 256  # a bounded sample of the same patterns and starting orientations
        line["cpu_baseline"] = RB.refine_cpu(mp.master_pattern.cpu(), wl["det"], pats[:m].float().cpu(),
                                             di_ori[:m].float().cpu(), wl["res"])
    del exp
    return line


def _short_step_counts(args, step):
    """Warm-up and timed step counts for modes whose step lasts milliseconds:
    at least `args.warmup` untimed steps and one second of them (the SM clock
    ramps up under load), then at least `args.steps` timed steps and half a
    second of them (so that the clock sampler sees the timed region)."""
    import torch

    n, t0 = 0, time.perf_counter()
    while n < args.warmup or time.perf_counter() - t0 < 1.0:
        step()
        torch.cuda.synchronize()
        n += 1
    per_step = (time.perf_counter() - t0) / n
    return max(args.steps, int(math.ceil(0.5 / max(per_step, 1e-6))))


PREPROCESS = dict(scan=(256, 256), det=(60, 60), k_rad=3, grains=64, mp=257, counts=100.0,
                  name="256 x 256 scan of 60 x 60 uint16 detector-count patterns (65,536), 64 grains")


def _grain_scan(cfg, mp, dev):
    """uint16 counts of a scan of Voronoi grains (one random orientation per
    grain, Poisson noise)."""
    import torch

    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry

    hs, ws = cfg["scan"]
    gen = torch.Generator().manual_seed(11)
    seeds = torch.rand((cfg["grains"], 2), generator=gen) * torch.tensor([hs, ws])
    yy, xx = torch.meshgrid(torch.arange(hs), torch.arange(ws), indexing="ij")
    pts = torch.stack((yy.reshape(-1), xx.reshape(-1)), dim=1).float()
    grain = torch.cdist(pts, seeds).argmin(dim=1)
    truth = synthetic.random_quaternions(cfg["grains"], 12)[grain].to(dev)
    geom = EBSDGeometry(cfg["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    return synthetic.synthetic_patterns(mp, geom, truth, mean_counts=cfg["counts"], seed=13, counts=True)


def preprocess_cpu_rate(cfg, scan=(24, 24)):
    """The oracle (NumPy float64) of standard_clean + nlpar on a `scan` crop."""
    import numpy as np

    from oracle import di_oracle as O

    rng = np.random.default_rng(0)
    h, w = cfg["det"]
    data = rng.poisson(cfg["counts"], size=scan + (h, w)).astype(np.float64)
    t0 = time.perf_counter()
    clean = O.standard_clean(data.reshape(-1, h, w))
    O.nlpar(clean.reshape(scan + (h, w)), cfg["k_rad"], 0.375)
    secs = time.perf_counter() - t0
    return scan[0] * scan[1] / secs, secs


def run_preprocess(args):
    """Experimental-pattern preprocessing, the reference's cleaning sequence
    (experiment_pats.py:287-316): standard_clean (overall background,
    min-max, CLAHE, min-max: one mean pass and one fused CLAHE pass) then
    do_nlpar(k_rad=3). `value`: counts resident in HBM; `e2e`: pinned host
    uint16 counts in, cleaned FP32 patterns back to pinned host memory."""
    import torch

    from ebsdtorch_b200 import _capi, synthetic
    from ebsdtorch_b200.ebsd import ExperimentPatterns
    from ebsdtorch_b200.preprocessing import nlpar_offsets, pattern_mean

    cfg = PREPROCESS
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    _capi.load()
    hs, ws = cfg["scan"]
    h, w = cfg["det"]
    n, n_pix = hs * ws, h * w
    mp = synthetic.synthetic_master_pattern(cfg["mp"], seed=0, device=dev)
    counts = _grain_scan(cfg, mp, dev).view(hs, ws, h, w).contiguous()

    def step(src):
        e = ExperimentPatterns(src)
        e.standard_clean()
        e.do_nlpar(k_rad=cfg["k_rad"])
        return e.patterns

    steps = _short_step_counts(args, lambda: step(counts))
    l0 = _capi.launch_count
    with ClockSampler(int(dev.index or 0)) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            out = step(counts)
        e1.record()
        torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3 / steps
    launches = (_capi.launch_count - l0) // steps

    # end to end: pinned host counts in, pinned host FP32 patterns out
    host_in = counts.cpu().pin_memory()
    host_out = torch.empty((n, h, w), dtype=torch.float32).pin_memory()
    for _ in range(2):
        host_out.copy_(step(host_in.to(dev, non_blocking=True)), non_blocking=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        host_out.copy_(step(host_in.to(dev, non_blocking=True)), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_secs = e0.elapsed_time(e1) / 1e3 / args.steps

    # the passes one by one on the same data (CUDA events around each)
    from ebsdtorch_b200._capi import call, load, ptr

    x = counts.view(n, n_pix).float()
    stream = torch.cuda.current_stream(dev).cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev)

    def timed(fn, reps=5):
        fn()
        ts = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    mean = pattern_mean(x)
    y = torch.empty_like(x)
    kern = {"pattern_mean": timed(lambda: pattern_mean(x))}
    kern["clahe_fused"] = timed(lambda: call("ebsd_clahe", ptr(x), n, h, w, n_pix, ptr(mean), 1, 40.0, 64, 4, 4, 1,
                                             ptr(y), n_pix, stream))
    off = nlpar_offsets(cfg["k_rad"]).to(dev, torch.int32).contiguous()
    K = off.shape[0]
    d = torch.empty((n, K), device=dev)
    wsb = int(load().ebsd_nlpar_workspace_bytes(hs, ws))
    wsp = torch.empty(wsb, dtype=torch.uint8, device=dev)
    kern["nlpar_dists"] = timed(lambda: call("ebsd_nlpar_dists", ptr(y), hs, ws, n_pix, n_pix, cfg["k_rad"], ptr(off),
                                             0, K, K, ptr(d), stream))
    kern["nlpar_weights"] = timed(lambda: call("ebsd_nlpar_weights", ptr(d), hs, ws, n_pix, ptr(off), K, 0.375,
                                               1e-6, 0.0, ptr(wsp), wsb, stream))
    out2 = torch.empty_like(y)
    kern["nlpar_average"] = timed(lambda: call("ebsd_nlpar_average", ptr(y), hs, ws, n_pix, n_pix, cfg["k_rad"],
                                               ptr(off), 0, K, K, ptr(d), 0, ptr(out2), n_pix, stream))
    peaks, src = _peaks()
    props = torch.cuda.get_device_properties(dev)
    pairs = n * K * n_pix
    top = max(kern, key=kern.get)
    alg_bytes = {"pattern_mean": n * n_pix * 4, "clahe_fused": 2 * n * n_pix * 4, "nlpar_dists": n * n_pix * 4,
                 "nlpar_weights": 2 * n * K * 4, "nlpar_average": 2 * n * n_pix * 4}
    ach = alg_bytes[top] / (kern[top] / 1e3) / 1e9
    # one 4-byte shared-memory load per (point, offset, pixel) and lane
    smem_pairs_peak = props.multi_processor_count * 32 * 1.965e9
    line = {
        "metric": "patterns preprocessed/s (standard_clean + do_nlpar k_rad 3)", "value": n / secs, "unit": UNIT,
        "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": secs * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["name"] + "; standard_clean (clip 40, 64 bins, 4 x 4 tiles) then NLPAR "
                   "(k_rad 3 = 49 offsets, coeff 0.375)", "l2": "inputs larger than L2 (943 MB FP32)"},
        "gpu_launches": launches,
        "e2e": {"value": n / e2e_secs, "unit": UNIT, "h2d_bytes_per_step": n * n_pix * 2,
                "d2h_bytes_per_step": n * n_pix * 4},
        "kernels_ms": kern,
        "roofline": {"bound": "hbm", "kernel": top, "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": ach / peaks["hbm_gbs"], "traffic": None, "peak_source": src},
        "clahe_fused_hbm": {"achieved": alg_bytes["clahe_fused"] / (kern["clahe_fused"] / 1e3) / 1e9,
                            "frac": alg_bytes["clahe_fused"] / (kern["clahe_fused"] / 1e3) / 1e9 / peaks["hbm_gbs"]},
        "nlpar_pairs_per_s": {"dists": pairs / (kern["nlpar_dists"] / 1e3),
                              "average": pairs / (kern["nlpar_average"] / 1e3),
                              "smem_load_bound": smem_pairs_peak,
                              "dists_frac": pairs / (kern["nlpar_dists"] / 1e3) / smem_pairs_peak,
                              "average_frac": pairs / (kern["nlpar_average"] / 1e3) / smem_pairs_peak},
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline and _reference_staged():
        from oracle import ref_baselines as RB

        # a 64 x 64 crop of the same scan (4,096 patterns)
        line["cpu_baseline"] = RB.preprocess_cpu(host_in[:64, :64].float(), cfg["k_rad"], 0.375)
    elif not args.no_cpu_baseline:
        r, csecs = preprocess_cpu_rate(cfg)
        line["cpu_baseline"] = {"value": r, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": "oracle (NumPy float64) standard_clean + nlpar k_rad 3 on a 24 x 24 crop "
                                          "of 60 x 60 patterns (%.1f s)" % csecs}
    del out
    return line


PCFIT = dict(det=(60, 60), n=16, x=(0.35, 0.65), y=(0.35, 0.65), z=(0.4, 0.7, 8), res=2.0, bs=1024, mp=257,
             pc=(0.5, 0.5, 0.55),
             name="16 patterns of 60 x 60, pc_x / pc_y in [0.35, 0.65] (enlarged detector 78 x 78), 8 pc_z steps, "
                  "m-3m 2.0 deg dictionary")


def run_pcfit(args):
    """Pattern-centre fitting (spatial_fft_pc_fitter, fitting.py:359-540):
    whole fits on the device (the tensor-core correlation path), the stages
    of one dictionary batch timed apart (projection on the enlarged detector,
    spectra, fused inverse transforms + max over the batch, fold), and the
    same fits through the cuFFT path for comparison."""
    import torch

    from ebsdtorch_b200 import _capi, kernels, synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, MasterPattern, spatial_fft_pc_fitter
    from ebsdtorch_b200.ebsd import fitting as F
    from ebsdtorch_b200.ebsd.indexing import _master_pattern_tensor
    from ebsdtorch_b200.kernels import RowBuffers
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    cfg = PCFIT
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    _capi.load()
    mp_t = synthetic.synthetic_master_pattern(cfg["mp"], seed=0, device=dev)
    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry(cfg["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=cfg["pc"])
    truth = synthetic.random_quaternions(cfg["n"], 21).to(dev)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=200.0, seed=22).float()
    pats = pats.view(cfg["n"], 1, *cfg["det"])
    kw = dict(pc_x_min=cfg["x"][0], pc_x_max=cfg["x"][1], pc_y_min=cfg["y"][0], pc_y_max=cfg["y"][1],
              pc_z_min=cfg["z"][0], pc_z_max=cfg["z"][1], pc_z_steps=cfg["z"][2], dictionary_resolution_deg=cfg["res"],
              dictionary_indexing_batch_size=cfg["bs"], orientation_index="global")
    H, W = cfg["det"]
    pix, pad, (hp, wp) = F.get_3D_pixel_coords_with_periphery((H, W), torch.device("cpu"), *cfg["x"], *cfg["y"], 1)
    if not F.xcorr_supported(hp, wp):
        raise RuntimeError(f"the {hp} x {wp} enlarged detector is outside the correlation kernels' range")

    def timed_fits(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            res = spatial_fft_pc_fitter(mp, pats, **kw)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / steps, res

    steps = _short_step_counts(args, lambda: spatial_fft_pc_fitter(mp, pats, **kw))
    l0 = _capi.launch_count
    with ClockSampler(int(dev.index or 0)) as clocks:
        secs, (pc, q) = timed_fits(steps)
    launches = (_capi.launch_count - l0) // steps
    n_dict = sample_ori_fz_laue_angle(11, cfg["res"], dev).shape[0]
    z_steps = cfg["z"][2]
    evals = n_dict * z_steps * cfg["n"] * hp * wp  # (orientation, pc_z, pattern, pc_x / pc_y shift) scores

    # the same fits through cuFFT (torch.fft) + ebsd_pcfit_reduce
    supported = F.xcorr_supported
    F.xcorr_supported = lambda h, w: False
    try:
        spatial_fft_pc_fitter(mp, pats, **kw)
        fft_secs, (pc_fft, q_fft) = timed_fits(max(1, min(steps, 5)))
    finally:
        F.xcorr_supported = supported

    # stages of one batch of cfg["bs"] orientations
    rays = F._rays_soa(pix.double().numpy(), 0.55, 70.0, 0.0, (H, W), dev)
    quats = sample_ori_fz_laue_angle(11, cfg["res"], dev)[:cfg["bs"]].float().contiguous()
    n, B = quats.shape[0], cfg["n"]
    spec_len = 4 * (hp // 2 + 1) * (wp // 2 + 1)
    sims = torch.empty((n, hp * wp), device=dev)
    spec = torch.empty((n, spec_len), device=dev)
    tables = torch.empty((int(_capi.load().ebsd_pcfit_xcorr_table_bytes(hp, wp)),), dtype=torch.uint8, device=dev)
    _capi.call("ebsd_pcfit_xcorr_tables", hp, wp, tables.data_ptr(), tables.numel(), None)
    terms = torch.randn((B, spec_len), device=dev)
    keys = torch.zeros((B * hp * wp,), dtype=torch.int64, device=dev)
    best = torch.zeros((B, hp, wp), device=dev)
    best_i = torch.zeros((B, hp, wp), dtype=torch.int64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    mp_b = _master_pattern_tensor(mp, 1, dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def st_project():
        kernels.project(mp_b, rays, quats, RowBuffers(f32=sims), subtract_mean=False)

    def st_spectra():
        _capi.call("ebsd_pcfit_spectra", sims.data_ptr(), hp * wp, n, hp, wp, tables.data_ptr(), spec.data_ptr(),
                   status.data_ptr(), stream)

    def st_xcorr():
        _capi.call("ebsd_pcfit_xcorr_max", spec.data_ptr(), n, terms.data_ptr(), B, hp, wp, tables.data_ptr(),
                   keys.data_ptr(), 0, status.data_ptr(), stream)

    def st_fold():
        _capi.call("ebsd_pcfit_fold", keys.data_ptr(), keys.numel(), best.data_ptr(), best_i.data_ptr(), stream)

    stages = {}
    for name, fn in (("project", st_project), ("spectra", st_spectra), ("xcorr_max", st_xcorr), ("fold", st_fold)):
        fn()
        ts = []
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        stages[name] = statistics.median(ts)
    if int(status.item()) != 0:
        raise RuntimeError("pattern-centre correlation kernels reported a device timeout")
    peaks, src = _peaks()
    # bf16 tensor FLOPs of the 3-term split per (pattern, simulated pattern)
    # pair: stage A (2 WF rows x H x 2 H2) + stage B (H x W x 2 WF)
    h2, wf = hp // 2 + 1, wp // 2 + 1
    pair_flops = 2 * 3 * (2 * wf * hp * 2 * h2 + hp * wp * 2 * wf)
    xc_tflops = pair_flops * n * B / (stages["xcorr_max"] / 1e3) / 1e12
    line = {
        "metric": "pattern-centre fits/s (spatial FFT search)", "value": 1.0 / secs, "unit": "fits/s", "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": secs * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3 (FP32-class split)", "data": "synthetic",
        "config": {"workload": cfg["name"] + " (%d orientations)" % n_dict,
                   "l2": "spectra and maps stay on chip; the projected batch (25 MB) is L2-resident"},
        "gpu_launches": launches,
        "scores_per_s": evals / secs,
        "fit": {"pc": [float(v) for v in pc.cpu()], "simulated_pc": list(cfg["pc"])},
        "fft_path": {"fits_per_s": 1.0 / fft_secs, "same_pc": bool(torch.equal(pc, pc_fft)),
                     "same_orientations": bool(torch.equal(q, q_fft)),
                     "how": "the same fits with cuFFT rfft2 / spectrum product / irfft2 + ebsd_pcfit_reduce"},
        "batch_stages_ms": stages,
        "roofline": {"bound": "tensor", "kernel": "k_xc_max (inverse DFTs + max over the batch)",
                     "achieved": xc_tflops, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                     "frac": xc_tflops / peaks["bf16_tflops"], "traffic": None,
                     "peak_source": src + " bf16_tflops (burst; the kernel is timed alone)",
                     "flops": "bf16 tensor FLOPs of the 3-term split, unpadded: 6 (4 WF H H2 + 2 H W WF) per pair"},
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline and _reference_staged():
        from oracle import ref_baselines as RB

        kw_ref = dict(pc_x_min=cfg["x"][0], pc_x_max=cfg["x"][1], pc_y_min=cfg["y"][0], pc_y_max=cfg["y"][1],
                      pc_z_min=cfg["z"][0], pc_z_max=cfg["z"][1], pc_z_steps=cfg["z"][2], primary_tilt_deg=70.0,
                      secondary_tilt_deg=0.0, dictionary_resolution_deg=cfg["res"],
                      dictionary_indexing_batch_size=cfg["bs"])
        torch.manual_seed(0)
        line["cpu_baseline"] = RB.pcfit_cpu(mp_t.cpu(), pats.cpu(), kw_ref, z_steps)
    elif not args.no_cpu_baseline:
        from oracle import di_oracle as O

        q64 = quats[:64].double().cpu().numpy()
        t0 = time.perf_counter()
        O.spatial_fft_pc_fit(mp_t.double().cpu().numpy(), pats[:, :, :, :].cpu().numpy(), q64, pc_x_min=cfg["x"][0],
                             pc_x_max=cfg["x"][1], pc_y_min=cfg["y"][0], pc_y_max=cfg["y"][1], pc_z_min=0.55,
                             pc_z_max=0.55, pc_z_steps=1, batch_size=64)
        t_cpu = (time.perf_counter() - t0) * (n_dict / 64) * z_steps
        line["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "fits/s", "cores": 1, "kind": "port",
                                "sample": "oracle (NumPy float64) on 64 orientations x 1 pc_z step, extrapolated to "
                                          "%d orientations x %d steps" % (n_dict, z_steps)}
    return line


BATCHED = dict(maps=48, q_min=1000, q_max=200000, detectors=((60, 60), (80, 80), (128, 128), (160, 160)),
               phases=((11, 0.5), (9, 0.615), (5, 0.88)), mp=1001, counts=100.0, seed=3)


def _full_workload_inputs(wl, dev, rank=0):
    """Master pattern, geometry, true orientations and patterns of a workload
    (seeded; rank 0 gets the same map in every mode)."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, MasterPattern

    mp = MasterPattern(synthetic.synthetic_master_pattern(wl["mp"], seed=0, device=dev), laue_group=11)
    geom = EBSDGeometry(wl["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    truth = synthetic.random_quaternions(wl["Q"], 1000 + rank).to(dev)
    pats = synthetic.synthetic_patterns(mp.master_pattern, geom, truth, mean_counts=wl["counts"], seed=2000 + rank)
    return mp, geom, truth, pats


def run_pca(args):
    import torch

    from ebsdtorch_b200 import _capi

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    _capi.load()
    # the profiling workload keeps the projection and match launches' shapes
    # (16,384-row sub-chunks, 1,024 components) at a few GB: 8,192 patterns,
    # the 1.0 deg dictionary, and a basis fitted on the 2.0 deg dictionary
    wl = WORKLOADS["profile" if args.workload == "profile" else "full"]
    learn_res = 2.0 if args.workload == "profile" else 0.9
    mp, geom, truth, pats = _full_workload_inputs(wl, dev)
    print(json.dumps(pca_block(args, wl, mp, geom, truth, pats, dev, learn_res=learn_res)), flush=True)


def pca_block(args, wl, mp, geom, truth, pats, dev, learn_res: float = 0.9) -> dict:
    """PCA dictionary indexing at the full size: 128 x 128 px, a basis of
    1,024 components fitted on the m-3m 0.9 deg dictionary (51,312 rows),
    indexing against the 0.5 deg dictionary (328,720 rows), 262,144 patterns,
    top-8. The fit (covariance + eigendecomposition) is a one-time cost,
    timed and reported on its own; a step is one
    pca_dictionary_index_orientations call given that basis (dictionary
    projection + PCA projection, query preparation + projection, match,
    FP32 re-score in PCA space)."""
    import torch

    from ebsdtorch_b200 import _capi, engine
    from ebsdtorch_b200.ebsd import ExperimentPatterns, dictionary_index_orientations, pca_dictionary_index_orientations
    from ebsdtorch_b200.ebsd import indexing as I
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    n_comp = 1024
    exp = ExperimentPatterns(pats)

    # ---- one-time fit ----
    rays = I._unit_rays_soa(geom, 1, None, dev)
    torch.manual_seed(0)
    ori_learn = sample_ori_fz_laue_angle(11, learn_res, dev)
    fit = {"learn_rows": int(ori_learn.shape[0])}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    comps = I.fit_pca_components(mp.master_pattern, rays, ori_learn, n_comp, "top", timings=fit)
    torch.cuda.synchronize()
    fit["total_s"] = time.perf_counter() - t0
    del ori_learn
    kw = dict(n_pca_components=n_comp, dictionary_resolution_learn_deg=learn_res,
              dictionary_resolution_index_deg=wl["res"], top_k_matches=wl["k"], match_dtype=torch.float32,
              components=comps)

    def step():
        torch.manual_seed(0)
        pca_dictionary_index_orientations(mp, geom, exp, **kw)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    engine.MATCH_TIMERS, I.PROJ_TIMERS = [], []
    launches0 = _capi.launch_count
    with ClockSampler(int(dev.index or 0)) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    launches = (_capi.launch_count - launches0) // args.steps
    t = e0.elapsed_time(e1) / 1e3
    mt, pt = engine.MATCH_TIMERS, I.PROJ_TIMERS
    engine.MATCH_TIMERS = I.PROJ_TIMERS = None
    match_ms = [a.elapsed_time(b) for a, b, _ in mt]
    match_fl = [f for _, _, f in mt]
    proj_ms = [a.elapsed_time(b) for a, b, _ in pt]
    proj_fl = [f for _, _, f in pt]
    achieved = (sum(match_fl) / len(match_fl)) / (sum(match_ms) / len(match_ms) / 1e3) / 1e12
    peaks, peak_kind = _peaks()
    peak = peaks.get("bf16_tflops_sustained", 1400.0)
    D = int(exp.dictionaries[0].shape[0])
    P = rays.shape[1]
    value = wl["Q"] * args.steps / t
    # FP32-class accuracy of the split GEMM: a few dictionary-like rows against FP64
    X = pats[:64].reshape(64, -1).double()
    X = X - X.mean(dim=1, keepdim=True)
    Y = torch.empty((64, n_comp), dtype=torch.float32, device=dev)
    I._Projector(comps)(X.float().contiguous(), Y)
    Y64 = X @ comps.double().t()
    proj_err = float(((Y.double() - Y64).abs().max(dim=1).values / Y64.abs().max(dim=1).values).max())
    # agreement with plain DI (bf16 match + FP32 re-score == FP32 top-1) on a subset
    n_sub = min(wl["Q"], args.fp32_subset)
    exp_p = ExperimentPatterns(pats[:n_sub])
    torch.manual_seed(0)
    dictionary_index_orientations(mp, geom, exp_p, dictionary_resolution_degrees=wl["res"], top_k_matches=1,
                                  match_dtype=torch.float32)
    a = disori_angle_laue(exp.orientations[:n_sub].float().contiguous(), exp_p.orientations.float().contiguous(),
                          11, 11)
    b = disori_angle_laue(exp.orientations.float().contiguous(), truth, 11, 11)
    # end to end from pinned host patterns
    e2e = None
    if not args.no_e2e:
        host = torch.empty(pats.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(pats)
        exp_h = ExperimentPatterns(host)
        torch.manual_seed(0)
        pca_dictionary_index_orientations(mp, geom, exp_h, **kw)
        torch.cuda.synchronize()
        h0 = time.perf_counter()
        e2e_steps = max(1, args.steps // 2)
        for _ in range(e2e_steps):
            torch.manual_seed(0)
            pca_dictionary_index_orientations(mp, geom, exp_h, **kw)
            q_out = exp_h.raw_indexing_results[0][0].cpu()
            m_out = exp_h.raw_indexing_results[0][1].cpu()
        torch.cuda.synchronize()
        e2e = {"value": wl["Q"] * e2e_steps / (time.perf_counter() - h0), "unit": UNIT,
               "h2d_bytes_per_step": int(host.numel() * 4), "d2h_bytes_per_step": int(q_out.numel() * 4 +
                                                                                   m_out.numel() * 4),
               "host_memory": "pinned"}
        del exp_h, host
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16", "data": "synthetic",
        "config": {"workload": f"PCA DI 128x128 px, {n_comp} components fitted on the m-3m {learn_res} deg dictionary "
                               f"({fit['learn_rows']:,}), indexing {D:,} rows, {wl['Q']:,} patterns, top-{wl['k']}",
                   "precision": "PCA projections TF32 on tcgen05 (kind::tf32, FP32 accumulation); bf16 match + "
                                "FP32 re-score of top-32 in PCA space",
                   "l2": "inputs larger than L2"},
        "e2e": e2e,
        "gpu_launches": int(launches * args.steps),
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None, "kernel": "k_tc_gemm (match + streaming top-k, K=1024)",
                     "peak_source": f"{peak_kind} bf16_tflops_sustained",
                     "share_of_step": sum(match_ms) / 1e3 / t},
        "projection": {"share_of_step": sum(proj_ms) / 1e3 / t,
                       "tflops": sum(proj_fl) / (sum(proj_ms) / 1e3) / 1e12,
                       "max_rel_error_vs_fp64": proj_err,
                       "how": "TF32 tcgen05 GEMM (kind::tf32, ebsd_gemm_f32) straight from the FP32 rows"},
        "algorithmic_flops_per_pattern": {"match_2DK": 2.0 * D * n_comp, "query_projection_2PK": 2.0 * P * n_comp,
                                          "dictionary_projection_amortised": 2.0 * D * P * n_comp / wl["Q"]},
        "fit_one_time": fit,
        "accuracy": {"within_0.5deg_of_plain_di": float((a < math.radians(0.5)).float().mean()),
                     "same_top1_orientation_as_plain_di": float(
                         ((exp.orientations[:n_sub].float() - exp_p.orientations.float()).abs().amax(1) < 1e-5)
                         .float().mean()),
                     "subset": n_sub, "within_0.5deg_of_truth": float((b < math.radians(0.5)).float().mean())},
        "clocks": clocks.summary(),
    }
    del exp, exp_p, comps
    return line


def run_batched(args):
    """Many scan maps of uneven size, detector shape and phase in
    one planned batch (BatchIndexer), replayed as one CUDA graph. Patterns
    are uint16 detector counts; `value` has them resident in HBM, `e2e` in
    pinned host memory (copied inside the graph every step)."""
    import numpy as np
    import torch

    from ebsdtorch_b200 import _capi, synthetic
    from ebsdtorch_b200.batch import BatchIndexer, LaunchTuner, MapJob
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern

    cfg = BATCHED
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    _capi.load()
    rng = np.random.default_rng(cfg["seed"])
    phases = [MasterPattern(synthetic.synthetic_master_pattern(cfg["mp"], seed=10 + i, device=dev, laue_group=laue),
                            laue_group=laue) for i, (laue, _) in enumerate(cfg["phases"])]
    geoms = [EBSDGeometry(d, tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6)) for d in cfg["detectors"]]
    specs = []
    for i in range(cfg["maps"]):
        q = int(round(math.exp(rng.uniform(math.log(cfg["q_min"]), math.log(cfg["q_max"])))))
        specs.append((q, int(rng.integers(len(geoms))), int(rng.integers(len(phases))), bool(rng.integers(2))))
    t0 = time.perf_counter()
    jobs = []
    for i, (q, gi, pi, fp32) in enumerate(specs):
        truth = synthetic.random_quaternions(q, 7000 + i).to(dev)
        pats = synthetic.synthetic_patterns(phases[pi].master_pattern, geoms[gi], truth, mean_counts=cfg["counts"],
                                            seed=8000 + i, counts=True)
        jobs.append(MapJob(phases[pi], geoms[gi], ExperimentPatterns(pats), top_k=8 if fp32 else 1,
                           rescore_k=32 if fp32 else 0))
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    res = {laue: r for laue, r in cfg["phases"]}
    tuner = LaunchTuner()
    torch.manual_seed(0)
    b = BatchIndexer(jobs, dictionary_resolution_degrees=res, device=dev, tuner=tuner)
    n_pat = b.n_patterns
    flops = 0.0
    for g in b.groups:
        d = b.phases[g.phase]["ori"].shape[0]
        flops += sum(2.0 * sub.n_queries * d * g.rays.shape[1] for sub in g.subgroups.values())
    t0 = time.perf_counter()
    b.run(use_graph=True)  # tune, eager run, capture, first replay
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    for _ in range(max(0, args.warmup - 1)):
        b.run(use_graph=True)

    def timed(bi, host_out):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            bi.graph.replay()
            if host_out:  # results back to the host, every map
                for o in bi._outputs:
                    o[0].to("cpu", non_blocking=True)
                    o[1].to("cpu", non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / args.steps

    with ClockSampler(int(dev.index or 0)) as clocks:
        secs = timed(b, False)
    # agreement with the reference algorithm in FP32 on 512 patterns of the
    # largest map of each phase
    agree = {}
    for pi in range(len(phases)):
        cand = [i for i, s in enumerate(specs) if s[2] == pi]
        if not cand:
            continue
        m = max(cand, key=lambda i: specs[i][0])
        job = jobs[m]
        from ebsdtorch_b200.ebsd.indexing import _unit_rays_soa

        rays = _unit_rays_soa(job.geometry, 1, None, dev)
        pats = job.experiment_patterns.patterns[:512].float()
        qf = pats.reshape(pats.shape[0], -1)
        qf = qf - qf.mean(dim=1, keepdim=True)
        ref_i, _, _ = plain_fp32_gpu_di(None, job.master_pattern.master_pattern, rays,
                                        job.experiment_patterns.dictionaries[0], qf, 1)
        got = job.experiment_patterns.raw_indexing_indices[0][:512, 0]
        agree[f"laue{cfg['phases'][pi][0]}_map{m}"] = float((got == ref_i[:, 0]).float().mean())
    plan = b.describe()
    b.release_graph()
    del b
    torch.cuda.empty_cache()
    # e2e: the same batch with the patterns in pinned host memory
    h2d = 0
    d2h = 0
    for job in jobs:
        p = job.experiment_patterns.patterns
        host = torch.empty(p.shape, dtype=p.dtype, pin_memory=True)
        host.copy_(p)
        job.experiment_patterns.patterns = host
        h2d += host.numel() * host.element_size()
        d2h += host.shape[0] * job.top_k * 12
        del p
    torch.cuda.empty_cache()
    torch.manual_seed(0)
    b2 = BatchIndexer(jobs, dictionary_resolution_degrees=res, device=dev, tuner=tuner)
    b2.run(use_graph=True)
    e2e_secs = timed(b2, True)
    b2.release_graph()
    line = {
        "metric": "patterns indexed/s, batched uneven maps (48 maps of 1k-200k patterns, mixed detectors and phases)", "value": n_pat / secs, "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
        "config": {"workload": "%d maps, patterns log-uniform in [%d, %d] (%d in total), detectors %s, phases "
                               "m-3m / 6/mmm / 4/mmm, bf16 match with FP32 re-score (top-8) or bf16 scores "
                               "(top-1) per map, uint16 detector counts, one CUDA graph per batch"
                               % (cfg["maps"], cfg["q_min"], cfg["q_max"], n_pat,
                                  "/".join(f"{h}x{w}" for h, w in cfg["detectors"])),
                   "dictionaries": {str(b2.phases[i]["laue"]): int(b2.phases[i]["ori"].shape[0])
                                    for i in range(len(b2.phases))},
                   "l2": "inputs larger than L2"},
        "e2e": {"value": n_pat / e2e_secs, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "host_memory": "pinned"},
        "step_flops": flops, "step_tflops": flops / secs / 1e12,
        "setup_seconds": {"data_generation": t_gen, "tune_eager_capture": t_setup},
        "plan": plan, "top1_vs_plain_fp32_di_512": agree,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="full")
    ap.add_argument("--precision", choices=["bf16", "fp8"], default="bf16")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32-compare", action="store_true")
    ap.add_argument("--no-fp8", action="store_true", help="skip the companion e4m3 measurement")
    ap.add_argument("--no-learned", action="store_true", help="skip the companion learned-path measurement")
    ap.add_argument("--no-companions", action="store_true",
                    help="skip the companion PCA / refinement / preprocessing / pattern-centre-fit measurements")
    ap.add_argument("--fp32-subset", type=int, default=8192)
    ap.add_argument("--learned", action="store_true", help="time the learned-proposal path instead")
    ap.add_argument("--batched", action="store_true", help="time batched uneven maps (48 maps, mixed sizes, detectors, phases) instead")
    ap.add_argument("--refine", action="store_true", help="time orientation grid refinement after DI instead")
    ap.add_argument("--preprocess", action="store_true", help="time pattern preprocessing (clean + NLPAR) instead")
    ap.add_argument("--pcfit", action="store_true", help="time pattern-centre fitting instead")
    ap.add_argument("--pca", action="store_true", help="time PCA dictionary indexing (1,024 components) instead")
    ap.add_argument("--train-steps", type=int, default=8000)
    ap.add_argument("--max-angle", type=float, default=16.0)
    ap.add_argument("--fallback-ratio", type=float, default=0.95)
    ap.add_argument("--stage-margin", type=float, default=1.6)
    ap.add_argument("--pyramid", default="3.0,1.5,0.75", help="intermediate dictionary resolutions (deg), coarse first")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, wl)
    elif args.learned:
        run_learned(args, wl)
    elif args.batched:
        run_batched(args)
    elif args.refine:
        run_refine(args, wl)
    elif args.preprocess:
        print(json.dumps(run_preprocess(args)), flush=True)
    elif args.pcfit:
        print(json.dumps(run_pcfit(args)), flush=True)
    elif args.pca:
        run_pca(args)
    else:
        run_ours(args, wl)


if __name__ == "__main__":
    main()
