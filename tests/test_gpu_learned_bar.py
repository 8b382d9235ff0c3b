"""The learned path at full size meets its accuracy bar.

128 x 128 patterns, the m-3m 0.5 deg dictionary (328,720 orientations): the
proposal network is trained on 768k freshly projected patterns (3,000 steps
of 256), then learned proposal + coarse-to-fine local search + plain-DI
fallback indexes 8,192 held-out patterns. At least 99.5 % of them must lie
within 0.5 deg (disorientation, Laue m-3m) of plain FP32 dictionary indexing:
the reference algorithm (indexing.py:14-211) with FP32 rows and an FP32
matrix product (TF32 off) over the whole dictionary.
"""

import math

import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _plain_fp32_top1(mp_t, rays, ori, pats, chunk=32768):
    """Brute-force FP32 dictionary indexing, top-1 index per pattern."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.kernels import RowBuffers

    torch.backends.cuda.matmul.allow_tf32 = False
    P = rays.shape[1]
    q = torch.empty((pats.shape[0], P), dtype=torch.float32, device=DEV)
    kernels.prep_patterns(pats, RowBuffers(f32=q))
    best_v = torch.full((pats.shape[0],), -math.inf, device=DEV)
    best_i = torch.zeros(pats.shape[0], dtype=torch.int64, device=DEV)
    rows = torch.empty((chunk, P), dtype=torch.float32, device=DEV)
    for d0 in range(0, ori.shape[0], chunk):
        d1 = min(ori.shape[0], d0 + chunk)
        kernels.project(mp_t, rays, ori[d0:d1].contiguous(), RowBuffers(f32=rows[:d1 - d0]), subtract_mean=True)
        v, i = (q @ rows[:d1 - d0].t()).max(dim=1)
        better = v > best_v
        best_v = torch.where(better, v, best_v)
        best_i = torch.where(better, i + d0, best_i)
    return best_i


def test_learned_path_within_half_degree_of_plain_fp32_di():
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern
    from ebsdtorch_b200.ebsd.indexing import _unit_rays_soa
    from ebsdtorch_b200.learned import train_proposal_cnn
    from ebsdtorch_b200.local_search import learned_dictionary_index
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    mp_t = synthetic.synthetic_master_pattern(1001, seed=0, device=DEV)
    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry((128, 128), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    model, losses = train_proposal_cnn(mp_t, geom, 11, steps=3000, batch=256, lr=1e-3, mean_counts=100.0, seed=0)
    # held-out patterns: orientations and noise seeds the training never drew
    truth = synthetic.random_quaternions(8192, 5000).to(DEV)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=100.0, seed=5001)
    exp = ExperimentPatterns(pats)
    torch.manual_seed(0)
    st = learned_dictionary_index(mp, geom, exp, model, dictionary_resolution_degrees=0.5)
    ori = exp.dictionaries[0]
    assert ori.shape[0] == 328720
    ref = _plain_fp32_top1(mp_t, _unit_rays_soa(geom, 1, None, DEV), ori, pats)
    ang = disori_angle_laue(exp.orientations.float().contiguous(), ori[ref].contiguous(), 11, 11)
    within = float((ang < math.radians(0.5)).float().mean())
    same = float((exp.raw_indexing_indices[0][:, 0] == ref).float().mean())
    print({"within_0.5deg": within, "same_index": same, "fallback": st.n_fallback / st.n_patterns,
           "final_loss": float(losses[-100:].mean())})
    assert within >= 0.995
