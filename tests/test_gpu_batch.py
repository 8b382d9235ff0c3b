"""Batched indexing of uneven maps (several phases, detector shapes, pattern
storage types, FP32 and bf16 paths) in one autotuned, graph-captured batch."""

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

N_ORACLE = 64  # patterns per map checked against the FP64 oracle

DEV = "cuda"


def _jobs():
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.batch import MapJob
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern

    cubic = MasterPattern(synthetic.synthetic_master_pattern(129, seed=1, device=DEV), laue_group=11)
    tetra = MasterPattern(synthetic.synthetic_master_pattern(129, seed=2, device=DEV, laue_group=5), laue_group=5)
    g24 = EBSDGeometry((24, 24), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    g32 = EBSDGeometry((32, 32), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    # (phase, geometry, patterns, top_k, rescore_k, uint16 counts in pinned host memory)
    spec = [(cubic, g24, 300, 3, 32, False), (cubic, g24, 1000, 1, 32, True), (cubic, g32, 700, 1, 0, False),
            (tetra, g32, 129, 2, 32, True), (tetra, g32, 2000, 2, 32, False), (tetra, g24, 450, 1, 0, True)]
    jobs = []
    for i, (mp, geom, n, k, r, host) in enumerate(spec):
        q = synthetic.random_quaternions(n, 100 + i).to(DEV)
        pats = synthetic.synthetic_patterns(mp.master_pattern, geom, q, mean_counts=150.0, seed=200 + i, counts=host)
        if host:
            pats = pats.cpu().pin_memory()
        jobs.append(MapJob(mp, geom, ExperimentPatterns(pats), top_k=k, rescore_k=r))
    return jobs


def _oracle_topk(job, ori, k, n):
    """FP64 oracle top-k (the reference algorithm, indexing.py:96-146 and
    knn.py:96-103) of the map's first n patterns over the batch's dictionary."""
    det = tuple(job.geometry.detector_shape)
    rays = O.unit_rays(O.detector_coords_sample_frame(det, (0.5, 0.5, 0.6), (0.0, 70.0, 0.0)))
    rows = O.dictionary_rows(job.master_pattern.master_pattern.cpu().numpy(), rays,
                             ori.cpu().numpy().astype(np.float64))
    q = O.prep_patterns(job.experiment_patterns.patterns[:n].cpu().numpy().astype(np.float64))
    return O.topk_dot(q, rows, k)


def test_batch_matches_the_oracle_per_map_and_graph_replays():
    from ebsdtorch_b200.batch import LAUNCH_SHAPES, BatchIndexer

    jobs = _jobs()
    torch.manual_seed(0)
    b = BatchIndexer(jobs, dictionary_resolution_degrees={11: 4.0, 5: 5.0})
    b.run(use_graph=False)
    plan = b.describe()
    # (phase, detector, top_k, rescore) sub-groups: the two 32x32 4/mmm maps
    # with top-2 and FP32 re-score are searched together
    assert len(plan) == 5 and sum(e["maps"] for e in plan) == 6
    for entry in plan:
        la = entry["launch"]
        assert any(la["tile_n"] == (s.get("tile_n") or 256) and la["persistent"] == s.get("persistent", False)
                   for s in LAUNCH_SHAPES), la
    eager = [(j.experiment_patterns.raw_indexing_indices[0].clone(),
              j.experiment_patterns.raw_indexing_results[0][1].clone()) for j in jobs]
    for job in jobs:
        exp = job.experiment_patterns
        idx = exp.raw_indexing_indices[0][:N_ORACLE].cpu().numpy()
        ref_i, ref_v = _oracle_topk(job, exp.dictionaries[0], job.top_k, N_ORACLE)
        if job.rescore_k > 0:
            # FP32 re-scored maps: the exact top-k and the reference's metric
            assert (idx == ref_i).mean() >= 0.99
            v = exp.raw_indexing_results[0][1][:N_ORACLE].double().cpu().numpy()
            same = idx == ref_i
            assert np.abs(v - ref_v)[same].max() <= 1e-4 * np.abs(ref_v).max()
        else:
            # bf16-only maps: the top-1 of the low-precision scores
            assert (idx[:, 0] == ref_i[:, 0]).mean() >= 0.95
        assert torch.equal(exp.orientations, exp.raw_indexing_results[0][0][:, 0])
    for _ in range(2):
        b.run(use_graph=True)
        for job, (i0, v0) in zip(jobs, eager):
            assert torch.equal(job.experiment_patterns.raw_indexing_indices[0], i0)
            assert torch.equal(job.experiment_patterns.raw_indexing_results[0][1], v0)
    # new data written into the same buffers is picked up by the replay
    p0 = jobs[0].experiment_patterns.patterns
    p0.copy_(p0.flip(0))
    b.run(use_graph=True)
    assert torch.equal(jobs[0].experiment_patterns.raw_indexing_indices[0], eager[0][0].flip(0))
    b.release_graph()


def test_batch_rejects_bad_jobs():
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.batch import BatchIndexer, MapJob
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern

    mp = MasterPattern(synthetic.synthetic_master_pattern(33, seed=1, device=DEV), laue_group=11)
    geom = EBSDGeometry((16, 16), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    with pytest.raises(ValueError):
        BatchIndexer([])
    with pytest.raises(ValueError):  # pageable host memory cannot be captured
        BatchIndexer([MapJob(mp, geom, ExperimentPatterns(torch.zeros(4, 16, 16)))], 10.0)
    with pytest.raises(ValueError):  # detector mismatch
        BatchIndexer([MapJob(mp, geom, ExperimentPatterns(torch.zeros(4, 12, 16, device=DEV)))], 10.0)
    with pytest.raises(TypeError):
        BatchIndexer([MapJob(mp, geom, ExperimentPatterns(torch.zeros(4, 16, 16, dtype=torch.int64, device=DEV)))],
                     10.0)
