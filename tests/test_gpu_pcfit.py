"""Pattern-centre fitting on the GPU against the reference's own results
(goldens) and the oracle."""

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _case(g, ci):
    from ebsdtorch_b200.ebsd import MasterPattern

    H, W, b, x0, x1, y0, y1, z0, z1, zs, tilt, sec, res, bs, seed = g[f"case{ci}_meta"]
    kw = dict(pc_x_min=x0, pc_x_max=x1, pc_y_min=y0, pc_y_max=y1, pc_z_min=z0, pc_z_max=z1, pc_z_steps=int(zs),
              primary_tilt_deg=tilt, secondary_tilt_deg=sec, dictionary_resolution_deg=res,
              dictionary_indexing_batch_size=int(bs), virtual_binning=int(b))
    mp = MasterPattern(torch.from_numpy(g[f"case{ci}_master_pattern"]).to(DEV), laue_group=11)
    return mp, torch.from_numpy(g[f"case{ci}_patterns"]).to(DEV), kw, int(seed)


@pytest.mark.parametrize("ci", [0, 1, 2])
def test_pc_fit_matches_reference(golden, ci):
    from ebsdtorch_b200.ebsd import spatial_fft_pc_fitter

    g = golden("pcfit")
    mp, pats, kw, seed = _case(g, ci)
    before = pats.clone()
    torch.manual_seed(seed)  # the dictionary permutation the reference drew
    pc, q = spatial_fft_pc_fitter(mp, pats, **kw)
    assert pc.device.type == "cuda" and q.shape == (pats.shape[0], 4)
    assert np.abs(pc.cpu().numpy() - g[f"case{ci}_best_pc"]).max() < 1e-6
    # same dictionary entries; the FZ grid is built in FP64 here and in FP32
    # by the reference, so the values agree to float32 rounding
    assert np.abs(q.cpu().numpy() - g[f"case{ci}_best_quats"]).max() < 2e-6
    assert torch.equal(pats, before)  # the caller's patterns are left alone


def test_enlarged_detector_projection_matches_reference(golden):
    """The projector on the fitter's enlarged-detector rays reproduces the
    reference's simulated dictionary patterns (pc_z = pc_z_min)."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.ebsd import fitting as F
    from ebsdtorch_b200.ebsd.indexing import _master_pattern_tensor
    from ebsdtorch_b200.kernels import RowBuffers

    g = golden("pcfit")
    for ci in range(3):
        mp, pats, kw, seed = _case(g, ci)
        H, W = pats.shape[-2:]
        pix, pad, (hp, wp) = F.get_3D_pixel_coords_with_periphery(
            (H, W), torch.device("cpu"), kw["pc_x_min"], kw["pc_x_max"], kw["pc_y_min"], kw["pc_y_max"],
            kw["virtual_binning"])
        z0 = float(torch.linspace(kw["pc_z_min"], kw["pc_z_max"], kw["pc_z_steps"])[0])
        rays = F._rays_soa(pix.double().numpy(), z0, kw["primary_tilt_deg"], kw["secondary_tilt_deg"], (H, W), DEV)
        q = torch.from_numpy(g[f"case{ci}_dictionary"][:4]).to(DEV).contiguous()
        out = torch.empty((4, hp * wp), device=DEV)
        kernels.project(_master_pattern_tensor(mp, kw["virtual_binning"], DEV), rays, q, RowBuffers(f32=out),
                        subtract_mean=False)
        assert float((out.view(4, hp, wp).cpu() - torch.from_numpy(g[f"case{ci}_sims"])).abs().max()) < 2e-4


def test_pc_fit_global_index_and_odd_width_match_oracle():
    """orientation_index='global' over several dictionary batches, an odd
    enlarged width (the reference cannot run it) and binning 2, against the
    oracle; and the reference index mode on the same case."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import MasterPattern, spatial_fft_pc_fitter
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    mp_t = synthetic.synthetic_master_pattern(129, seed=4, device=DEV)
    mp64 = mp_t.double().cpu().numpy()
    torch.manual_seed(77)
    dict_q = sample_ori_fz_laue_angle(11, 9.0, torch.device(DEV)).cpu().numpy()
    # three patterns simulated at dictionary orientations, PC (0.45, 0.55, 0.55)
    pix, _, _ = O.pixel_coords_with_periphery((32, 28), 0.5, 0.5, 0.5, 0.5, 1)
    rot, t = O.bruker_se3((0.45, 0.55, 0.55), -70.0, 0.0, (32, 28))
    pats = O.project_patterns(mp64, O.unit_rays(pix @ rot.T + t), dict_q[[5, 40, 60]].astype(np.float64))
    pats = pats.reshape(3, 1, 32, 28) + 0.05 * np.random.default_rng(6).standard_normal((3, 1, 32, 28))
    kw = dict(pc_x_min=0.3, pc_x_max=0.62, pc_y_min=0.4, pc_y_max=0.6, pc_z_min=0.45, pc_z_max=0.65, pc_z_steps=3,
              primary_tilt_deg=70.0, secondary_tilt_deg=0.0, virtual_binning=2)
    mp = MasterPattern(mp_t, laue_group=11)
    for mode in ("global", "reference"):
        torch.manual_seed(77)
        pc, q = spatial_fft_pc_fitter(mp, torch.from_numpy(pats).float().to(DEV), dictionary_resolution_deg=9.0,
                                      dictionary_indexing_batch_size=24, orientation_index=mode, **kw)
        ref_pc, idx, _ = O.spatial_fft_pc_fit(mp64, pats.astype(np.float32), dict_q, batch_size=24,
                                              batch_local_index=(mode == "reference"), **kw)
        assert np.abs(pc.cpu().numpy() - ref_pc).max() < 1e-6, mode
        assert np.array_equal(q.cpu().numpy(), dict_q[idx]), mode
    assert list(idx) == [5 % 24, 40 % 24, 60 % 24]  # reference mode: positions inside the winning batch
