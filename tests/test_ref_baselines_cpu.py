"""The host-CPU baselines that run the reference's own fitter, preprocessing
and refinement (oracle/ref_baselines.py) work on small inputs. Skipped when
the reference is not staged in oracle/_ref."""

import pytest
import torch

from oracle import ref_loader

pytestmark = pytest.mark.skipif(ref_loader.reference_root() is None, reason="reference not staged")


def _mp():
    from ebsdtorch_b200 import synthetic

    return synthetic.synthetic_master_pattern(65, seed=0, device="cpu")


def test_pcfit_baseline_runs_one_step():
    from oracle import ref_baselines as RB

    kw = dict(pc_x_min=0.45, pc_x_max=0.55, pc_y_min=0.45, pc_y_max=0.55, pc_z_min=0.5, pc_z_max=0.6,
              pc_z_steps=4, primary_tilt_deg=70.0, secondary_tilt_deg=0.0, dictionary_resolution_deg=15.0,
              dictionary_indexing_batch_size=64)
    r = RB.pcfit_cpu(_mp(), torch.rand((2, 1, 12, 12)), kw, kw["pc_z_steps"])
    assert r["kind"] == "reference" and r["unit"] == "fits/s" and r["value"] > 0 and r["cores"] >= 1


def test_preprocess_baseline_runs_on_a_crop():
    from oracle import ref_baselines as RB

    r = RB.preprocess_cpu(torch.poisson(torch.full((4, 5, 16, 16), 80.0)), 1, 0.375)
    assert r["kind"] == "reference" and r["unit"] == "patterns/s" and r["value"] > 0


def test_refine_baseline_runs_on_a_sample():
    from ebsdtorch_b200 import synthetic
    from oracle import ref_baselines as RB

    q = synthetic.random_quaternions(4, 1)
    r = RB.refine_cpu(_mp(), (12, 12), torch.rand((4, 12, 12)), q, 3.0, n_iter=1)
    assert r["kind"] == "reference" and r["unit"] == "patterns/s" and r["value"] > 0
