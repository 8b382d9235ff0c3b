"""PCA dictionary indexing at full size against an FP64 reference.

128 x 128 patterns; a basis of 1,024 components fitted on the m-3m 0.9 deg
dictionary (51,312 rows); indexing against the 0.5 deg dictionary (328,720
rows); a 4,096-pattern subset. The FP64 reference recomputes, in float64
torch on the GPU, the same algorithm (pca_covmat.py:94-158 covariance of the
zero-mean rows, eigendecomposition, indexing.py:401-452 projections, dot
product top-1) from the same simulated rows (the projector's parity with the
reference is pinned elsewhere). Checked: the 3-term-split projection against
FP64 (relative to each row's largest component), the fitted subspace against
the FP64 one, top-1 agreement with FP64 PCA DI, and the fraction within
0.5 deg of plain DI.
"""

import math

import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda"
N_SUB = 4096
N_COMP = 1024


def test_pca_config1_against_fp64():
    from ebsdtorch_b200 import kernels, synthetic
    from ebsdtorch_b200.ebsd import (EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations,
                                     pca_dictionary_index_orientations)
    from ebsdtorch_b200.ebsd import indexing as I
    from ebsdtorch_b200.kernels import RowBuffers
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    mp_t = synthetic.synthetic_master_pattern(1001, seed=0, device=DEV)
    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry((128, 128), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    truth = synthetic.random_quaternions(N_SUB, 777).to(DEV)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=100.0, seed=778)
    rays = I._unit_rays_soa(geom, 1, None, DEV)
    P = rays.shape[1]

    exp = ExperimentPatterns(pats)
    torch.manual_seed(0)
    pca_dictionary_index_orientations(mp, geom, exp, n_pca_components=N_COMP, dictionary_resolution_learn_deg=0.9,
                                      dictionary_resolution_index_deg=0.5, top_k_matches=1,
                                      match_dtype=torch.float32)
    comps = exp.pca_components[0]
    ori = exp.dictionaries[0]
    assert comps.shape == (N_COMP, P) and ori.shape[0] == 328720

    # FP64 reference fit on the same learning rows (same permutation draw)
    torch.manual_seed(0)
    learn = sample_ori_fz_laue_angle(11, 0.9, DEV)
    assert learn.shape[0] == 51312
    X = torch.empty((learn.shape[0], P), dtype=torch.float32, device=DEV)
    kernels.project(mp_t, rays, learn, RowBuffers(f32=X), subtract_mean=True)
    X64 = X.double()
    del X
    X64 -= X64.mean(dim=0, keepdim=True)
    cov = (X64.t() @ X64) / (X64.shape[0] - 1)
    del X64
    _, vecs = torch.linalg.eigh(cov)
    del cov
    V64 = vecs[:, -N_COMP:].contiguous()  # (P, K)
    del vecs
    # subspace: ||V64^T C^T||_F^2 / K = mean squared cosine of the principal angles
    overlap = float(((V64.t() @ comps.double().t()) ** 2).sum() / N_COMP)

    # projection accuracy of the split GEMM on these patterns
    q = torch.empty((N_SUB, P), dtype=torch.float32, device=DEV)
    kernels.prep_patterns(pats, RowBuffers(f32=q))
    Y = torch.empty((N_SUB, N_COMP), dtype=torch.float32, device=DEV)
    I._Projector(comps)(q, Y)
    Y64 = q.double() @ comps.double().t()
    proj_err = float(((Y.double() - Y64).abs().amax(dim=1) / Y64.abs().amax(dim=1)).max())

    # FP64 PCA DI with the FP64 basis, top-1 over the whole dictionary
    qp = q.double() @ V64
    best_v = torch.full((N_SUB,), -math.inf, dtype=torch.float64, device=DEV)
    best_i = torch.zeros(N_SUB, dtype=torch.int64, device=DEV)
    rows = torch.empty((16384, P), dtype=torch.float32, device=DEV)
    for d0 in range(0, ori.shape[0], 16384):
        d1 = min(ori.shape[0], d0 + 16384)
        kernels.project(mp_t, rays, ori[d0:d1].contiguous(), RowBuffers(f32=rows[:d1 - d0]), subtract_mean=True)
        v, i = (qp @ (rows[:d1 - d0].double() @ V64).t()).max(dim=1)
        better = v > best_v
        best_v = torch.where(better, v, best_v)
        best_i = torch.where(better, i + d0, best_i)
    ours = exp.raw_indexing_indices[0][:, 0]
    agree64 = float((ours == best_i).float().mean())
    mis64 = disori_angle_laue(ori[ours].contiguous(), ori[best_i].contiguous(), 11, 11)

    # plain DI on the same patterns (bf16 + FP32 re-score == FP32 top-1)
    exp_p = ExperimentPatterns(pats)
    torch.manual_seed(0)
    dictionary_index_orientations(mp, geom, exp_p, dictionary_resolution_degrees=0.5, match_dtype=torch.float32)
    mis_plain = disori_angle_laue(exp.orientations.float().contiguous(), exp_p.orientations.float().contiguous(),
                                  11, 11)
    within_plain = float((mis_plain < math.radians(0.5)).float().mean())
    print({"subspace_overlap": overlap, "projection_rel_err": proj_err, "top1_agree_fp64_pca": agree64,
           "within_0.5deg_of_fp64_pca": float((mis64 < math.radians(0.5)).float().mean()),
           "within_0.5deg_of_plain_di": within_plain})
    assert proj_err < 1e-3
    assert overlap > 0.99
    assert float((mis64 < math.radians(0.5)).float().mean()) >= 0.99
    assert within_plain >= 0.95
