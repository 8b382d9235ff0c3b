"""Precision report of the full-size plain-DI path against an FP64 CPU oracle.

Workload: 128 x 128 patterns, the m-3m 0.5 deg dictionary (328,720 rows),
master pattern 2 x 1001 x 1001, mean 100 counts; a 4,096-pattern subset of
the scan is checked. For every pattern the FP64 oracle rebuilds, in float64
on the CPU, the query row and the dictionary rows of the plain FP32 DI's top 8
(plus each tested path's top 1), and takes the FP64 best among them. That is
the FP64 global best whenever the FP32 top-1 / top-8 score gap exceeds twice
the FP32 row error (the guard below); patterns without that gap are counted
and left out. Reported per path (bf16 match + FP32 re-score, e4m3 match + FP32
re-score, and the reference's FP32 algorithm in torch): maximum similarity
error, top-1 agreement, and the median / 99th-percentile misorientation
between the path's top 1 and the FP64 top 1.
"""

import json
import multiprocessing as mp_ctx
import os

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"
N_SUBSET = 4096


def _fp64_scores(mp64, rays64, qrows64, cand_quats):
    """FP64 scores (n, c) of n query rows against their c candidate
    orientations each (oracle rows built in float64)."""
    n, c = cand_quats.shape[:2]
    rows = O.dictionary_rows(mp64, rays64, cand_quats.reshape(n * c, 4), dtype=np.float64, chunk=128)
    return np.einsum("qp,qjp->qj", qrows64, rows.reshape(n, c, -1))


def test_precision_report_against_fp64_oracle():
    import bench
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations
    from ebsdtorch_b200.ebsd.indexing import _unit_rays_soa

    det, res, pc = (128, 128), 0.5, (0.5, 0.5, 0.6)
    mp_t = synthetic.synthetic_master_pattern(1001, seed=0, device=DEV)
    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry(det, tilts_degrees=(0.0, 70.0, 0.0), proj_center=pc)
    truth = synthetic.random_quaternions(N_SUBSET, 4242).to(DEV)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=100.0, seed=4243)

    results = {}
    for prec in ("bf16", "fp8"):
        exp = ExperimentPatterns(pats.clone())
        torch.manual_seed(0)
        dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=res, top_k_matches=8,
                                      match_dtype=torch.float32, precision=prec)
        results[prec] = (exp.raw_indexing_indices[0][:, 0].cpu().numpy(),
                         exp.raw_indexing_results[0][1][:, 0].double().cpu().numpy())
        dictionary = exp.dictionaries[0]
    # the reference's algorithm in FP32 (torch eager): candidates and guard
    rays = _unit_rays_soa(geom, 1, None, DEV)
    q32 = pats.reshape(N_SUBSET, -1).float()
    q32 = q32 - q32.mean(dim=1, keepdim=True)
    idx32, _, _, val32 = bench.plain_fp32_gpu_di(None, mp_t, rays, dictionary, q32, 8, return_values=True)
    idx32, val32 = idx32.cpu().numpy(), val32.double().cpu().numpy()

    # FP64 oracle inputs: grid, permutation, rays, master pattern, queries
    n = dictionary.shape[0]
    torch.manual_seed(0)
    perm = torch.randperm(n).numpy()
    grid64 = O.sample_ori_fz_laue_angle(11, res, permutation=perm)
    assert np.abs(grid64.astype(np.float32) - dictionary.cpu().numpy()).max() <= 1e-7
    rays64 = O.unit_rays(O.detector_coords_sample_frame(det, pc, (0.0, 70.0, 0.0)))
    mp64 = mp_t.double().cpu().numpy()
    qrows64 = O.prep_patterns(pats.double().cpu().numpy())

    # candidates: FP32 top 8, then each tested path's top 1
    cand = np.concatenate([idx32] + [r[0][:, None] for r in results.values()], axis=1)
    parts = np.array_split(np.arange(N_SUBSET), 64)
    workers = max(1, min(16, os.cpu_count() or 1))
    with mp_ctx.get_context("spawn").Pool(workers) as pool:
        got = pool.starmap(_fp64_scores, [(mp64, rays64, qrows64[p], grid64[cand[p]]) for p in parts])
    s64 = np.concatenate(got, axis=0)
    # FP32 error of the reference algorithm's scores, and the guard: with a
    # top-1 / top-8 gap above twice that error the FP64 best is a candidate
    err32 = np.abs(val32 - s64[:, :8]).max()
    gap = val32[:, 0] - val32[:, 7]
    ok = gap > 4.0 * err32
    best64 = cand[np.arange(N_SUBSET), np.argmax(s64, axis=1)]

    def report(top1, sims=None):
        j = np.argmax(cand == top1[:, None], axis=1)
        agree = top1[ok] == best64[ok]
        mis = np.degrees(O.disori_angle(grid64[top1[ok]], grid64[best64[ok]], 11))
        out = {"top1_agreement": float(agree.mean()), "misori_median_deg": float(np.median(mis)),
               "misori_p99_deg": float(np.percentile(mis, 99)), "misori_max_deg": float(mis.max())}
        if sims is not None:
            ref = s64[np.arange(N_SUBSET), j]
            out["max_similarity_error"] = float(np.abs(sims - ref)[ok].max())
            out["max_similarity_error_rel"] = float((np.abs(sims - ref) / np.abs(ref))[ok].max())
        return out

    rep = {"subset": N_SUBSET, "guarded": int(ok.sum()), "fp32_reference_score_error": float(err32),
           "bf16_rescore32": report(*results["bf16"]), "e4m3_rescore32": report(*results["fp8"]),
           "fp32_reference_algorithm": report(idx32[:, 0])}
    print("PRECISION_REPORT " + json.dumps(rep))
    assert ok.mean() >= 0.98
    assert rep["bf16_rescore32"]["top1_agreement"] >= 0.995
    assert rep["e4m3_rescore32"]["top1_agreement"] >= 0.99
    assert rep["bf16_rescore32"]["max_similarity_error_rel"] <= 1e-4
    assert rep["bf16_rescore32"]["misori_median_deg"] <= 1e-4
