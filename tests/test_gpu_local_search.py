"""Local dictionary search around orientation proposals and the
learned-proposal indexing path."""

import math

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _case(det=(24, 24), res=3.0, n=200, seed=2):
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry
    from ebsdtorch_b200.ebsd.indexing import _unit_rays_soa
    from ebsdtorch_b200.local_search import PhaseDictionary

    mp = synthetic.synthetic_master_pattern(129, seed=seed, device=DEV)
    geom = EBSDGeometry(det, tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    rays = _unit_rays_soa(geom, 1, None, DEV)
    torch.manual_seed(seed)
    pd = PhaseDictionary(mp, rays, 11, res)
    truth = synthetic.random_quaternions(n, seed + 10).to(DEV)
    pats = synthetic.synthetic_patterns(mp, geom, truth, mean_counts=200.0, seed=seed + 20)
    return mp, geom, rays, pd, truth, pats


def test_local_search_matches_bruteforce_oracle():
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.kernels import RowBuffers
    from ebsdtorch_b200.local_search import local_search

    mp, geom, rays, pd, truth, pats = _case()
    Q, P = pats.shape[0], rays.shape[1]
    q_f32 = torch.empty((Q, P), device=DEV)
    kernels.prep_patterns(pats, RowBuffers(f32=q_f32))
    # proposals: the truth rotated by ~2 degrees about random axes
    rng = np.random.default_rng(0)
    ax = rng.standard_normal((Q, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    h = np.radians(2.0) / 2
    dq = np.concatenate((np.full((Q, 1), math.cos(h)), math.sin(h) * ax), axis=1)
    prop = O._qmul(truth.cpu().double().numpy(), dq)
    prop = np.where(prop[:, :1] < 0, -prop, prop)
    prop_t = torch.from_numpy(prop).float().to(DEV)
    for max_deg in (4.0, 8.0):
        idx, score, ncand = local_search(pd, q_f32, prop_t, max_angle_deg=max_deg)
        ri, rv = O.local_search_bruteforce(q_f32.double().cpu().numpy(), prop, pd.quats.double().cpu().numpy(),
                                           pd.rows.f32.double().cpu().numpy(), 11, math.radians(max_deg))
        got_i = idx.cpu().numpy()
        assert (got_i == ri).mean() >= 0.99, (max_deg, (got_i == ri).mean())
        ok = ri >= 0
        assert np.abs(score.cpu().numpy()[ok] - rv[ok]).max() <= 1e-5 * np.abs(rv[ok]).max()
        assert int(ncand.min()) >= 0
        # candidates ranked by the bf16 rows, best 8 re-scored in FP32
        li, ls, lc = local_search(pd, q_f32, prop_t, max_angle_deg=max_deg, n_rescore=8)
        assert torch.equal(lc, ncand)
        li_n = li.cpu().numpy()
        assert (li_n == ri).mean() >= 0.99, (max_deg, (li_n == ri).mean())
        same = (li_n == ri) & ok
        assert np.abs(ls.cpu().numpy()[same] - rv[same]).max() <= 1e-5 * np.abs(rv[ok]).max()
        # no re-score: the bf16 estimate of the bf16-best candidate
        ei, es, _ = local_search(pd, q_f32, prop_t, max_angle_deg=max_deg, n_rescore=0)
        assert (ei.cpu().numpy() == ri).mean() >= 0.9
        assert np.abs(es.cpu().numpy()[ok] - rv[ok]).max() <= 1e-2 * np.abs(rv[ok]).max()


def test_local_search_near_plain_di_answer_reproduces_it():
    """Proposals within the search radius of plain DI's answer (its own
    orientation rotated by 1.5 deg) give exactly plain DI's top-1."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.engine import Searcher, SearchConfig
    from ebsdtorch_b200.kernels import RowBuffers
    from ebsdtorch_b200.local_search import local_search

    mp, geom, rays, pd, truth, pats = _case(det=(32, 32), res=2.0, n=512)
    Q, P = pats.shape[0], rays.shape[1]
    q_f32 = torch.empty((Q, P), device=DEV)
    kernels.prep_patterns(pats, RowBuffers(f32=q_f32))

    def fill_q(a, b, bufs):
        kernels.prep_patterns(q_f32[a:b].reshape(b - a, 1, P), bufs, subtract_mean=False)

    full_i, full_v = Searcher(pd.n, Q, P, 1, SearchConfig(), DEV).run(None, fill_q, resident=pd.rows)
    best = pd.quats[full_i[:, 0]].double().cpu().numpy()
    rng = np.random.default_rng(1)
    ax = rng.standard_normal((Q, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    h = np.radians(1.5) / 2
    dq = np.concatenate((np.full((Q, 1), math.cos(h)), math.sin(h) * ax), axis=1)
    prop = torch.from_numpy(O._qmul(best, dq)).float().to(DEV)
    idx, score, _ = local_search(pd, q_f32, prop, max_angle_deg=5.0)
    assert torch.equal(idx, full_i[:, 0])
    assert torch.allclose(score, full_v[:, 0], rtol=1e-5)


def test_trained_network_gain():
    """What the trained network gains: with the same search radius and
    fallback rule, its proposals reproduce plain DI; an untrained network's
    proposals do not (the fallback threshold is relative to the map's median
    local score, so bad proposals also lower the bar)."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, dictionary_index_orientations
    from ebsdtorch_b200.learned import OrientationCNN, train_proposal_cnn
    from ebsdtorch_b200.local_search import learned_dictionary_index

    mp_t = synthetic.synthetic_master_pattern(257, seed=1, device=DEV)
    from ebsdtorch_b200.ebsd import MasterPattern

    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry((64, 64), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    model, losses = train_proposal_cnn(mp_t, geom, 11, steps=1500, batch=256, lr=1e-3, mean_counts=200.0, seed=0)
    truth = synthetic.random_quaternions(1024, 777).to(DEV)
    pats = synthetic.synthetic_patterns(mp_t, geom, truth, mean_counts=200.0, seed=778)
    exp_l = ExperimentPatterns(pats.clone())
    torch.manual_seed(5)
    st = learned_dictionary_index(mp, geom, exp_l, model, dictionary_resolution_degrees=1.0)
    exp_u = ExperimentPatterns(pats.clone())
    torch.manual_seed(5)
    st_u = learned_dictionary_index(mp, geom, exp_u, OrientationCNN((64, 64), 11, seed=9, device=DEV),
                                    dictionary_resolution_degrees=1.0)
    exp_f = ExperimentPatterns(pats.clone())
    torch.manual_seed(5)
    dictionary_index_orientations(mp, geom, exp_f, dictionary_resolution_degrees=1.0, match_dtype=torch.float32)
    full = exp_f.raw_indexing_indices[0][:, 0]
    agree = (exp_l.raw_indexing_indices[0][:, 0] == full).float().mean().item()
    agree_u = (exp_u.raw_indexing_indices[0][:, 0] == full).float().mean().item()
    print({"trained_fallback": st.n_fallback, "untrained_fallback": st_u.n_fallback, "agree": agree,
           "agree_untrained": agree_u, "final_loss": float(losses[-50:].mean()), "radii": st.stage_radii_deg,
           "stage_candidates": st.stage_mean_candidates})
    assert agree >= 0.97
    assert agree - agree_u >= 0.2
