"""Batched indexing of uneven maps (several phases, detector shapes, pattern
storage types, FP32 and bf16 paths) in one autotuned, graph-captured batch."""

import pytest
import torch

pytestmark = pytest.mark.gpu

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


def _fp32_topk(job, ori, k):
    """Exact FP32 top-k of the reference algorithm over the batch's dictionary."""
    import bench
    from ebsdtorch_b200.ebsd.indexing import _unit_rays_soa

    rays = _unit_rays_soa(job.geometry, 1, None, DEV)
    pats = job.experiment_patterns.patterns.to(DEV).float()
    q = pats.reshape(pats.shape[0], -1)
    q = q - q.mean(dim=1, keepdim=True)
    idx, _, _, val = bench.plain_fp32_gpu_di(None, job.master_pattern.master_pattern, rays, ori, q, k,
                                             return_values=True)
    return idx, val


def test_batch_matches_per_map_fp32_search_and_graph_replays():
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
        idx = exp.raw_indexing_indices[0]
        ref_i, ref_v = _fp32_topk(job, exp.dictionaries[0], job.top_k)
        if job.rescore_k > 0:
            assert (idx == ref_i).float().mean() >= 0.999
            v = exp.raw_indexing_results[0][1]
            assert float((v - ref_v).abs().max()) <= 1e-4 * float(ref_v.abs().max())
        else:
            assert (idx[:, 0] == ref_i[:, 0]).float().mean() >= 0.99
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
