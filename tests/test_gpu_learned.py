"""The learned-proposal part on the GPU: 6-D rotation kernels against the
reference goldens and the oracle; CNN forward / backward kernels against the
FP64 oracle; and a short training run."""

import math

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def test_rot6d_kernels_match_reference(golden):
    from ebsdtorch_b200._capi import call

    g = golden("rot6d")
    zh = torch.from_numpy(g["zh"]).float().to(DEV)
    qu = torch.empty((zh.shape[0], 4), device=DEV)
    om = torch.empty((zh.shape[0], 9), device=DEV)
    s = torch.cuda.current_stream().cuda_stream
    call("ebsd_zh_to_qu", zh.data_ptr(), zh.shape[0], qu.data_ptr(), om.data_ptr(), s)
    assert np.abs(om.cpu().numpy().reshape(-1, 3, 3) - g["om"]).max() < 2e-5
    ref = g["qu"]
    got = qu.cpu().numpy()
    assert np.minimum(np.abs(got - ref).max(1), np.abs(got + ref).max(1)).max() < 5e-5
    q_in = torch.from_numpy(g["qu_in"]).float().to(DEV)
    z = torch.empty((q_in.shape[0], 6), device=DEV)
    call("ebsd_qu_to_zh", q_in.data_ptr(), q_in.shape[0], z.data_ptr(), s)
    assert np.abs(z.cpu().numpy() - g["zh_out"]).max() < 2e-6


def test_rot6d_loss_kernel_matches_oracle():
    from ebsdtorch_b200._capi import call

    rng = np.random.default_rng(4)
    zh = rng.standard_normal((500, 6))
    q = rng.standard_normal((500, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    loss_ref, grad_ref = O.rot6d_sym_loss(zh, q, 11)
    z_t, q_t = torch.from_numpy(zh).float().to(DEV), torch.from_numpy(q).float().to(DEV)
    loss = torch.empty(500, device=DEV)
    grad = torch.empty((500, 6), device=DEV)
    call("ebsd_rot6d_sym_loss", z_t.data_ptr(), q_t.data_ptr(), 500, 11, 0.5, loss.data_ptr(), grad.data_ptr(),
         torch.cuda.current_stream().cuda_stream)
    assert np.abs(loss.cpu().numpy() - loss_ref).max() < 1e-4
    assert np.abs(grad.cpu().numpy() - 0.5 * grad_ref).max() < 2e-3 * (1 + np.abs(grad_ref).max())


def test_cnn_gradients_match_oracle():
    """bf16 forward / backward of the full architecture (32 x 32 input) vs the
    FP64 oracle with the same weights: outputs and every parameter gradient
    agree to bf16 accuracy."""
    from ebsdtorch_b200.learned import OrientationCNN

    torch.manual_seed(0)
    model = OrientationCNN((32, 32), 11, seed=3, device=DEV)
    assert OrientationCNN((128, 128), 11, seed=0, device=DEV).n_params() == 1240518
    B = 128
    x = torch.randn((B, 32, 32), device=DEV)
    q = torch.nn.functional.normalize(torch.randn((B, 4), device=DEV), dim=1)
    out = model.forward(x)
    loss, grad = model.loss_and_grad(out, q)
    model.backward(grad)
    params = {k: v.double().cpu().numpy() for k, v in model.state_dict().items()}
    # same upstream gradient on both sides (the nearest symmetric target can
    # differ between bf16 and FP64 outputs; the loss kernel is checked alone)
    z, L, g = O.cnn_forward_backward(params, x.double().cpu().numpy(), q.double().cpu().numpy(), 11,
                                     grad_out=grad.double().cpu().numpy())
    zo = out.double().cpu().numpy()
    assert np.linalg.norm(zo - z) <= 0.03 * np.linalg.norm(z)
    assert abs(float(loss.mean()) - L) <= 0.03 * abs(L)
    gpu_g = {}
    for i, c in enumerate(model.convs):
        gpu_g[f"conv{i}.w"], gpu_g[f"conv{i}.b"] = c.gw, c.gb
    gpu_g["fc1.w"], gpu_g["fc1.b"] = model.fc1.gw, model.fc1.gb
    gpu_g["fc2.w"], gpu_g["fc2.b"] = model.fc2.gw, model.fc2.gb
    report = {}
    for k, ref in g.items():
        got = gpu_g[k].double().cpu().numpy()
        cos = float(np.sum(got * ref) / (np.linalg.norm(got) * np.linalg.norm(ref) + 1e-30))
        rel = float(np.linalg.norm(got - ref) / (np.linalg.norm(ref) + 1e-30))
        report[k] = (round(cos, 4), round(rel, 4))
    print(report)
    assert all(c > 0.99 and r < 0.15 for c, r in report.values()), report
    assert report["fc2.b"][1] < 1e-5  # FP32 head: exact


@pytest.mark.parametrize("cin,cout,hw,batch", [(1, 32, 64, 1024), (64, 128, 16, 256), (256, 256, 8, 128),
                                                (32, 64, 32, 256), (64, 128, 15, 64)])
def test_conv_forward_matches_fp32_convolution(cin, cout, hw, batch):
    """Fused im2col GEMM + bias + ReLU (ebsd_cnn_conv_fwd) against an FP32
    convolution of the same bf16-rounded input and weights; the first case
    streams ~14 pixel tiles per work unit, the third uses two channel tiles,
    the fourth pads K (288 -> 320), the last has an odd input size."""
    from ebsdtorch_b200.learned import _Conv

    gen = torch.Generator().manual_seed(cin + cout)
    conv = _Conv(cin, cout, gen, torch.device(DEV))
    conv.b.copy_(torch.randn(cout, generator=gen).to(DEV) * 0.1)
    x = torch.randn((batch, hw, hw, cin), generator=gen).to(DEV).bfloat16()
    out, out32, ho, wo = conv.forward(x, batch, hw, hw, {}, want32=True)
    torch.cuda.synchronize()
    assert int(conv.status.item()) == 0
    w = conv.w.bfloat16().float().view(cout, 3, 3, cin).permute(0, 3, 1, 2)
    prev = torch.backends.cudnn.allow_tf32
    torch.backends.cudnn.allow_tf32 = False
    try:
        ref = torch.nn.functional.conv2d(x.float().permute(0, 3, 1, 2), w, conv.b, stride=2, padding=1)
    finally:
        torch.backends.cudnn.allow_tf32 = prev
    ref = torch.relu(ref).permute(0, 2, 3, 1).reshape(batch * ho * wo, cout)
    scale = float(ref.abs().max())
    assert float((out32 - ref).abs().max()) <= 1e-4 * scale
    assert float((out.float() - ref).abs().max()) <= 8e-3 * scale


def test_cnn_training_learns_orientations():
    """A short training run on projector-generated patterns lowers the
    symmetric rotation loss (400 steps of 128 fresh 64 x 64 patterns)."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry
    from ebsdtorch_b200.learned import train_proposal_cnn

    mp = synthetic.synthetic_master_pattern(257, seed=1, device=DEV)
    geom = EBSDGeometry((64, 64), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    model, losses = train_proposal_cnn(mp, geom, 11, steps=400, batch=128, lr=1e-3, mean_counts=200.0, seed=0)
    assert torch.isfinite(losses).all()
    assert float(losses[-50:].mean()) < 0.88 * float(losses[:50].mean())
