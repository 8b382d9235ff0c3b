"""Orientation grid refinement on the GPU: the reference's own refinement
results (goldens), the FP64 oracle, and the accuracy it adds after DI."""

import math

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _golden_exp(g, ci):
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern

    det0, det1, b, edge, radius, axial, n_iter, shrink, avg = g[f"case{ci}_meta"]
    mp = MasterPattern(torch.from_numpy(g[f"case{ci}_master_pattern"]).to(DEV), laue_group=11)
    geom = EBSDGeometry((int(det0), int(det1)), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    exp = ExperimentPatterns(torch.from_numpy(g[f"case{ci}_patterns"]).to(DEV))
    exp.set_orientations(torch.from_numpy(g[f"case{ci}_start"]).to(DEV))
    exp.phases = torch.zeros(exp.n_patterns, dtype=torch.int64, device=DEV)
    if not avg:
        exp.set_spatial_coords(torch.from_numpy(g[f"case{ci}_spatial"]).to(DEV))
    kw = dict(grid_semi_edge_in_degrees=float(edge), batch_size=5, virtual_binning=int(b), n_iter=int(n_iter),
              axial_grid_dimension=int(axial), kernel_radius_in_steps=int(radius), shrink_factor=float(shrink),
              average_pattern_center=bool(avg), match_dtype=torch.float32)
    return mp, geom, exp, kw


@pytest.mark.parametrize("ci", [0, 1, 2])
def test_refinement_matches_reference_golden(golden, ci):
    from ebsdtorch_b200.ebsd import orientation_grid_refinement

    g = golden("refine")
    mp, geom, exp, kw = _golden_exp(g, ci)
    dots = orientation_grid_refinement(mp, geom, exp, **kw)
    q = exp.orientations.double().cpu().numpy()
    ref = g[f"case{ci}_refined"].astype(np.float64)
    err = np.minimum(np.abs(q - ref).max(1), np.abs(q + ref).max(1))
    assert err.max() < 1e-4, err
    ref_d = g[f"case{ci}_dots"]
    assert np.abs(dots[0].cpu().numpy() - ref_d).max() <= 1e-3 * np.abs(ref_d).max()


def test_refinement_matches_oracle_left_reduction():
    """fz_reduction='left' against the FP64 oracle (radius 2, 4 iterations)."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern, orientation_grid_refinement

    mp_t = synthetic.synthetic_master_pattern(129, seed=5, noise=0.0, device=DEV)
    geom = EBSDGeometry((24, 24), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    truth = synthetic.random_quaternions(40, 6).to(DEV)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=300.0, seed=7)
    rng = np.random.default_rng(8)
    ax = rng.standard_normal((40, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    h = np.radians(1.5) / 2
    dq = np.concatenate((np.full((40, 1), math.cos(h)), math.sin(h) * ax), axis=1)
    start = O.qu_std(O._qmul(dq, truth.double().cpu().numpy()))
    exp = ExperimentPatterns(pats.clone())
    exp.set_orientations(torch.from_numpy(start).float().to(DEV))
    exp.phases = torch.zeros(40, dtype=torch.int64, device=DEV)
    mp = MasterPattern(mp_t, laue_group=11)
    dots = orientation_grid_refinement(mp, geom, exp, 2.0, 64, n_iter=4, kernel_radius_in_steps=2,
                                       fz_reduction="left")
    rays = O.unit_rays(O.detector_coords_sample_frame((24, 24), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0)))
    rows = O.prep_patterns(pats.double().cpu().numpy())
    q_ref, d_ref = O.orientation_grid_refinement(mp_t.double().cpu().numpy(), rays, rows, start, 11, 2.0, n_iter=4,
                                                 radius=2, fz="left")
    q = exp.orientations.double().cpu().numpy()
    err = np.minimum(np.abs(q - q_ref).max(1), np.abs(q + q_ref).max(1))
    assert (err < 1e-4).mean() >= 0.95, err
    assert np.abs(dots[0].cpu().numpy() - d_ref).max() <= 1e-3 * np.abs(d_ref).max()


def test_refinement_improves_dictionary_indexing():
    """After DI on a 2 deg dictionary, refinement brings the orientations
    closer to the truth (the reason the step exists)."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import (EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations,
                                     orientation_grid_refinement)
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    mp_t = synthetic.synthetic_master_pattern(257, seed=1, device=DEV)
    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry((60, 60), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    truth = synthetic.random_quaternions(512, 31).to(DEV)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=300.0, seed=32)
    exp = ExperimentPatterns(pats)
    torch.manual_seed(0)
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=2.0, match_dtype=torch.float32)
    before = torch.rad2deg(disori_angle_laue(exp.orientations.float().contiguous(), truth, 11, 11))
    orientation_grid_refinement(mp, geom, exp, 2.0, 512, n_iter=6, fz_reduction="left")
    after = torch.rad2deg(disori_angle_laue(exp.orientations.float().contiguous(), truth, 11, 11))
    print({"median_before": float(before.median()), "median_after": float(after.median())})
    assert float(after.median()) < 0.6 * float(before.median())
