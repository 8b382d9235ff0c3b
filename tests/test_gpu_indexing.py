"""End-to-end parity of the drop-in dictionary-indexing functions against the
reference's own outputs (golden vectors) and the CPU oracle."""

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _setup(d, binning_mask=True):
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern

    m = d["meta"]
    det, pc = (int(m[0]), int(m[1])), tuple(float(v) for v in m[2:5])
    mp = MasterPattern(torch.from_numpy(d["master_pattern"]), laue_group=11).to(DEV)
    geom = EBSDGeometry(det, tilts_degrees=(0.0, 70.0, 0.0), proj_center=pc).to(DEV)
    exp = ExperimentPatterns(torch.from_numpy(d["patterns"]).to(DEV))
    mask = torch.from_numpy(d["mask"]) if d["mask"].size else None
    return mp, geom, exp, mask


@pytest.mark.parametrize("case", ["di_a", "di_b", "di_c"])
@pytest.mark.parametrize("precision", ["bf16", "fp8"])
def test_dictionary_index_matches_reference(golden, case, precision):
    from ebsdtorch_b200.ebsd import dictionary_index_orientations

    d = golden(case)
    m = d["meta"]
    res, k, b, ec, dcs, seed = m[5], int(m[7]), int(m[8]), int(m[9]), int(m[10]), int(m[11])
    mp, geom, exp, mask = _setup(d)
    torch.manual_seed(seed)
    dictionary_index_orientations(mp, geom, exp, signal_mask=mask, experiment_chunk_size=ec,
                                  dictionary_resolution_degrees=res, dictionary_chunk_size=dcs,
                                  virtual_binning=b, top_k_matches=k, match_dtype=torch.float32,
                                  precision=precision)
    quats, metrics = exp.raw_indexing_results[0]
    assert quats.shape == d["quats"].shape and metrics.dtype == torch.float32
    assert np.abs(exp.dictionaries[0].cpu().numpy() - d["dictionary"]).max() < 2e-6
    same = np.abs(quats.cpu().numpy() - d["quats"]).max(-1) < 1e-5
    assert same.mean() == 1.0
    ref = d["metrics"]
    assert np.abs(metrics.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    assert np.abs(exp.orientations.cpu().numpy() - d["orientations"]).max() < 1e-5
    assert exp.phases.dtype == torch.uint8


def test_reference_test_case(golden):
    """tests/test_di.py:9-48 of the reference, with its fp16 default match dtype."""
    from ebsdtorch_b200.ebsd import (EBSDGeometry, ExperimentPatterns, MasterPattern,
                                     dictionary_index_orientations)

    d = golden("di_reftest")
    geom = EBSDGeometry(detector_shape=(5, 5), proj_center=(0.4221, 0.2179, 0.4954)).to(DEV)
    mp = MasterPattern(torch.from_numpy(d["master_pattern"]), laue_group=11).to(DEV)
    exp = ExperimentPatterns(torch.from_numpy(d["patterns"]).to(DEV))
    torch.manual_seed(int(d["seed"][0]))
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=10.0, dictionary_chunk_size=4096,
                                  signal_mask=None, virtual_binning=1, experiment_chunk_size=4096,
                                  match_dtype=torch.float16)
    assert exp.get_orientations().cpu().numpy().shape == (2, 4)
    assert exp.raw_indexing_results[0][1].dtype == torch.float16
    assert np.abs(exp.raw_indexing_results[0][0].cpu().numpy() - d["quats"]).max() < 1e-5
    assert np.allclose(exp.raw_indexing_results[0][1].float().cpu().numpy(), d["metrics"], rtol=2e-3)


def test_host_resident_patterns_stream(golden):
    """Patterns in pinned host memory are streamed to the GPU chunk by chunk."""
    from ebsdtorch_b200.ebsd import ExperimentPatterns, dictionary_index_orientations

    d = golden("di_a")
    m = d["meta"]
    mp, geom, _, _ = _setup(d)
    exp = ExperimentPatterns(torch.from_numpy(d["patterns"]).pin_memory())
    torch.manual_seed(int(m[11]))
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=m[5], top_k_matches=int(m[7]),
                                  match_dtype=torch.float32)
    assert np.abs(exp.raw_indexing_results[0][0].cpu().numpy() - d["quats"]).max() < 1e-5


def test_cosine_similarity_mode(golden):
    from ebsdtorch_b200.ebsd import dictionary_index_orientations

    d = golden("di_a")
    m = d["meta"]
    mp, geom, exp, _ = _setup(d)
    torch.manual_seed(int(m[11]))
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=m[5], top_k_matches=3,
                                  match_dtype=torch.float32, similarity="cosine")
    # oracle: cosine ranking over the same dictionary
    dic = exp.dictionaries[0].cpu().numpy().astype(np.float64)
    rays = O.unit_rays(O.detector_coords_sample_frame((16, 16), m[2:5], (0, 70, 0)))
    drows = O.dictionary_rows(d["master_pattern"], rays, dic)
    q = O.prep_patterns(d["patterns"])
    dn = drows / np.linalg.norm(drows, axis=1, keepdims=True)
    qn = q / np.linalg.norm(q, axis=1, keepdims=True)
    ri, rv = O.topk_dot(qn, dn, 3)
    assert (exp.raw_indexing_indices[0].cpu().numpy() == ri).mean() == 1.0
    assert np.abs(exp.raw_indexing_results[0][1].cpu().numpy() - rv).max() < 1e-5


@pytest.mark.parametrize("tag,slice_mode", [("top", "top"), ("shipped", "reference"),
                                            ("shipped_n100", "reference")])
def test_pca_dictionary_index_matches_reference(golden, tag, slice_mode):
    """PCA DI (learn on 5 deg, index on 8 deg) against the reference's output:
    same dictionary, same top-1 orientations, metric within FP32-class
    tolerance of the reference's eigenvector basis."""
    from ebsdtorch_b200.ebsd import (EBSDGeometry, ExperimentPatterns, MasterPattern,
                                     pca_dictionary_index_orientations)

    d = golden("pca_di")
    geom = EBSDGeometry((16, 16), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6)).to(DEV)
    mp = MasterPattern(torch.from_numpy(d["master_pattern"]), laue_group=11).to(DEV)
    exp = ExperimentPatterns(torch.from_numpy(d["patterns"]).to(DEV))
    torch.manual_seed(777)
    pca_dictionary_index_orientations(mp, geom, exp, n_pca_components=int(d[f"ncomp_{tag}"][0]),
                                      dictionary_resolution_learn_deg=5.0, dictionary_resolution_index_deg=8.0,
                                      top_k_matches=2, match_dtype=torch.float32, component_slice=slice_mode)
    q = exp.raw_indexing_results[0][0].cpu().numpy()
    assert np.abs(exp.dictionaries[0].cpu().numpy() - d["dictionary"]).max() < 2e-6
    top1 = np.abs(q[:, 0] - d[f"quats_{tag}"][:, 0]).max(-1) < 1e-5
    assert top1.mean() == 1.0
    ref = d[f"metrics_{tag}"]
    got = exp.raw_indexing_results[0][1].cpu().numpy()
    assert np.abs(got[:, 0] - ref[:, 0]).max() <= 1e-3 * np.abs(ref).max()


def test_pca_shipped_slice_empty_raises(golden):
    from ebsdtorch_b200.ebsd import (EBSDGeometry, ExperimentPatterns, MasterPattern,
                                     pca_dictionary_index_orientations)

    d = golden("pca_di")
    geom = EBSDGeometry((20, 20), proj_center=(0.5, 0.5, 0.6))
    mp = MasterPattern(torch.from_numpy(d["master_pattern"]), laue_group=11).to(DEV)
    exp = ExperimentPatterns(torch.randn(3, 20, 20, device=DEV))
    with pytest.raises(ValueError, match="selects no components"):
        pca_dictionary_index_orientations(mp, geom, exp, n_pca_components=100,
                                          dictionary_resolution_learn_deg=12.0,
                                          dictionary_resolution_index_deg=12.0, component_slice="reference")


def test_argument_errors_are_loud():
    from ebsdtorch_b200.ebsd import (EBSDGeometry, ExperimentPatterns, MasterPattern,
                                     dictionary_index_orientations)

    geom = EBSDGeometry((8, 8))
    mp = MasterPattern(torch.rand(9, 18), laue_group=11).to(DEV)
    exp = ExperimentPatterns(torch.randn(2, 8, 8, device=DEV))
    with pytest.raises(NotImplementedError, match="'chebyshev' not supported"):  # knn.py:98-99's message
        dictionary_index_orientations(mp, geom, exp, distance_metric="chebyshev", dictionary_resolution_degrees=15)
    with pytest.raises(NotImplementedError):
        dictionary_index_orientations(mp, geom, exp, average_pattern_center=False, dictionary_resolution_degrees=15)
    with pytest.raises(ValueError):
        dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=15, top_k_matches=1000)
    with pytest.raises(ValueError):
        dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=15, virtual_binning=3)


def test_synthetic_small_config_parity_and_accuracy():
    """Config-0 style synthetic case at reduced size: the GPU result equals the
    exact FP64 oracle DI on the same dictionary and patterns, and the indexed
    orientations are near the true ones."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import dictionary_index_orientations
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    mp, geom, exp, truth = synthetic.make_case(129, (40, 40), 256, seed=4)
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=2.0, top_k_matches=2,
                                  match_dtype=torch.float32)
    dic = exp.dictionaries[0].cpu().numpy().astype(np.float64)
    rays = O.unit_rays(O.detector_coords_sample_frame((40, 40), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0)))
    d = O.dictionary_rows(mp.master_pattern.cpu().numpy(), rays, dic)
    ri, rv = O.topk_dot(O.prep_patterns(exp.patterns.cpu().numpy()), d, 2)
    assert (exp.raw_indexing_indices[0].cpu().numpy()[:, 0] == ri[:, 0]).mean() >= 0.99
    got = exp.raw_indexing_results[0][1].cpu().numpy()
    assert np.abs(got - rv).max() <= 1e-4 * np.abs(rv).max()
    ang = disori_angle_laue(exp.orientations.float().contiguous(), truth, 11, 11)
    # 2 deg grid on a coarse 40 x 40 detector: nearest grid point ~1-2 deg away
    assert torch.median(ang).item() < np.deg2rad(4.0)


@pytest.mark.parametrize("case", [0, 1, 2, 3])
@pytest.mark.parametrize("precision", ["bf16", "fp8"])
def test_distance_metric_matches_reference(golden, case, precision):
    """distance_metric="euclidean" (cases 0, 1: the reference's squared
    distances, knn.py:85-91) and "manhattan" (cases 2, 3: L1 distances,
    :92-93), smallest first, combined with higher_is_better=False."""
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations

    d = golden("di_euclid")
    m = d[f"case{case}_meta"]
    det, res, k, b, ec, dcs, seed = (int(m[0]), int(m[1])), m[2], int(m[4]), int(m[5]), int(m[6]), int(m[7]), \
        int(m[8])
    mp = MasterPattern(torch.from_numpy(d[f"case{case}_master_pattern"]), laue_group=11).to(DEV)
    geom = EBSDGeometry(det, tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6)).to(DEV)
    exp = ExperimentPatterns(torch.from_numpy(d[f"case{case}_patterns"]).to(DEV))
    mask = torch.from_numpy(d[f"case{case}_mask"]) if d[f"case{case}_mask"].size else None
    torch.manual_seed(seed)
    dictionary_index_orientations(mp, geom, exp, signal_mask=mask, experiment_chunk_size=ec,
                                  dictionary_resolution_degrees=res, dictionary_chunk_size=dcs, virtual_binning=b,
                                  top_k_matches=k, distance_metric=str(d[f"case{case}_metric"]),
                                  match_dtype=torch.float32, precision=precision)
    quats, dists = exp.raw_indexing_results[0]
    ref = d[f"case{case}_dists"]
    assert np.abs(quats.cpu().numpy() - d[f"case{case}_quats"]).max() < 1e-5
    assert np.abs(dists.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    assert np.abs(exp.best_metrics.cpu().numpy() - d[f"case{case}_best"]).max() <= 1e-4 * np.abs(ref).max()


def test_euclidean_matches_oracle_with_dictionary_chunks():
    """The euclidean running merge across dictionary chunks (distances, not
    scores, carried between chunks) against the FP64 oracle."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import dictionary_index_orientations

    mp, geom, exp, _ = synthetic.make_case(129, (32, 32), 600, seed=5, mean_counts=80.0)
    torch.manual_seed(2)
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=4.0, top_k_matches=4,
                                  distance_metric="euclidean", match_dtype=torch.float32,
                                  workspace_bytes=6 << 20)
    dic = exp.dictionaries[0].cpu().numpy().astype(np.float64)
    rays = O.unit_rays(O.detector_coords_sample_frame((32, 32), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0)))
    rows = O.dictionary_rows(mp.master_pattern.cpu().numpy(), rays, dic)
    q = O.prep_patterns(exp.patterns.cpu().numpy())
    oi, ov = O.topk_euclidean(q, rows, 4)
    gi = exp.raw_indexing_indices[0].cpu().numpy()
    gv = exp.raw_indexing_results[0][1].cpu().numpy()
    assert (gi[:, 0] == oi[:, 0]).mean() >= 0.99
    same = gi == oi
    assert np.abs(gv - ov)[same].max() <= 1e-4 * np.abs(ov).max()


def test_manhattan_matches_oracle_with_dictionary_chunks():
    """The manhattan candidates (exact FP32 L1 distances on the CUDA cores)
    merged across dictionary chunks and ranges, against the FP64 oracle."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import dictionary_index_orientations

    mp, geom, exp, _ = synthetic.make_case(129, (32, 32), 300, seed=6, mean_counts=80.0)
    torch.manual_seed(4)
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=4.0, top_k_matches=5,
                                  distance_metric="manhattan", match_dtype=torch.float32, workspace_bytes=6 << 20)
    dic = exp.dictionaries[0].cpu().numpy().astype(np.float64)
    rays = O.unit_rays(O.detector_coords_sample_frame((32, 32), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0)))
    rows = O.dictionary_rows(mp.master_pattern.cpu().numpy(), rays, dic)
    q = O.prep_patterns(exp.patterns.cpu().numpy())
    oi, ov = O.topk_manhattan(q, rows, 5)
    gi = exp.raw_indexing_indices[0].cpu().numpy()
    gv = exp.raw_indexing_results[0][1].cpu().numpy()
    assert (gi[:, 0] == oi[:, 0]).mean() >= 0.99
    same = gi == oi
    assert np.abs(gv - ov)[same].max() <= 1e-4 * np.abs(ov).max()
    assert (np.diff(gv, axis=1) >= 0).all()
