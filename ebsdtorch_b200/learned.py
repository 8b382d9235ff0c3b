"""Learned orientation proposals: a small CNN trained only on patterns the
projector generates, running on this package's own kernels.

Architecture: five 3x3 / stride-2 / pad-1 convolutions with ReLU
(1 -> 32 -> 64 -> 128 -> 256 -> 256 channels; a 128 x 128 pattern becomes
4 x 4 x 256), then a two-layer head (4096 -> 64 with ReLU, 64 -> 6) that
predicts the 6-D rotation representation of Zhou et al. (orientations.py:940);
1.24 M parameters. Convolutions run in bf16 on the tcgen05 GEMM (im2col
forward with bias, ReLU and the activation stores fused into the GEMM
epilogue; weight- and column-gradient GEMMs + col2im backward), except the
single-channel first layer, computed directly on the CUDA cores; the head in
FP32. The loss is the symmetry-aware rotation loss min_g ||R(z) - R(g q)||_F^2
(ebsd_rot6d_sym_loss), optimiser Adam on FP32 master weights.

This part has no counterpart in the reference (ebsdtorch has no learned
indexer); it feeds local dictionary search (ebsdtorch_b200.local_search).
"""

from __future__ import annotations

import math
from typing import List, Optional

import torch

from . import _capi, kernels
from ._capi import call, ptr
from .kernels import round_up


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


class _Conv:
    """3x3 / stride 2 / pad 1 convolution + ReLU, NHWC bf16 activations."""

    def __init__(self, cin: int, cout: int, gen: torch.Generator, device):
        self.cin, self.cout = cin, cout
        self.K = 9 * cin
        self.K_pad = round_up(self.K, 64)
        w = torch.randn((cout, self.K), generator=gen) * math.sqrt(2.0 / self.K)
        self.w = w.to(device)
        self.b = torch.zeros(cout, device=device)
        self.state = [torch.zeros_like(self.w), torch.zeros_like(self.w), torch.zeros_like(self.b),
                      torch.zeros_like(self.b)]
        # bf16 copies read by the GEMMs: W (cout_pad128 x K_pad) and W^T (K_pad256 x cout_pad64)
        self.w16 = torch.zeros((round_up(cout, 128), self.K_pad), dtype=torch.bfloat16, device=device)
        self.w16[:cout, :self.K] = self.w.bfloat16()
        self.ld_t = round_up(cout, 64)
        self.w16t = torch.zeros((round_up(self.K_pad, 256), self.ld_t), dtype=torch.bfloat16, device=device)
        self.w16t[:self.K, :cout] = self.w.t().bfloat16()
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        # device status word of the forward GEMM (non-zero after a timeout)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        sms = torch.cuda.get_device_properties(device).multi_processor_count if self.w.is_cuda else 148
        self.fwd_splits = max(1, 2 * sms // (self.w16.shape[0] // 128))

    def params(self):
        return [self.w, self.b]

    def _im2col(self, x: torch.Tensor, B: int, H: int, W: int) -> torch.Tensor:
        M = B * ((H + 1) // 2) * ((W + 1) // 2)
        cols = torch.empty((round_up(M, 256), self.K_pad), dtype=torch.bfloat16, device=x.device)
        call("ebsd_cnn_im2col", ptr(x), B, H, W, self.cin, cols.shape[0], self.K_pad, ptr(cols), _stream(x))
        return cols

    def forward(self, x: torch.Tensor, B: int, H: int, W: int, keep: dict, want32: bool = False):
        Ho, Wo = (H + 1) // 2, (W + 1) // 2
        M = B * Ho * Wo
        out = torch.empty((M, self.cout), dtype=torch.bfloat16, device=x.device)
        out32 = torch.empty((M, self.cout), dtype=torch.float32, device=x.device) if want32 else None
        if self.cin == 1:
            # 9 taps: a direct SIMT convolution beats a GEMM padded to K = 64
            call("ebsd_cnn_conv_c1", ptr(x), B, H, W, ptr(self.w16), self.K_pad, ptr(self.b), self.cout, 1, ptr(out),
                 ptr(out32), _stream(x))
            keep.update(x=x)
        else:
            # one tcgen05 GEMM with the output channels on the 128-row side and
            # the long pixel axis streamed in a few hundred units; bias, ReLU
            # and the bf16 (and FP32) activation stores are fused into its epilogue
            cols = self._im2col(x, B, H, W)
            call("ebsd_cnn_conv_fwd", ptr(self.w16), self.w16.shape[0], ptr(cols), cols.shape[0], self.K_pad,
                 ptr(self.b), self.cout, M, 1, ptr(out), self.cout, ptr(out32), self.fwd_splits, ptr(self.status),
                 _stream(x))
            keep.update(cols=cols)
        keep.update(out=out, M=M, H=H, W=W, B=B)
        return out, out32, Ho, Wo

    def backward(self, dout: torch.Tensor, keep: dict, need_dx: bool) -> Optional[torch.Tensor]:
        M, B, H, W = keep["M"], keep["B"], keep["H"], keep["W"]
        dev = dout.device
        s = _stream(dout)
        g32 = torch.empty((M, self.cout), dtype=torch.float32, device=dev)
        ld16 = round_up(self.cout, 64)
        g16 = torch.empty((M, ld16), dtype=torch.bfloat16, device=dev)
        call("ebsd_cnn_relu_grad", ptr(dout), self.cout, ptr(keep["out"]), self.cout, M, self.cout, ptr(g32),
             ptr(g16), ld16, s)
        call("ebsd_cnn_col_sum", ptr(g32), M, self.cout, ptr(self.gb), s)
        # weight gradient: (cout x K) = g^T (cout x M) . cols (M x K)
        gT = torch.empty((round_up(self.cout, 128), M), dtype=torch.bfloat16, device=dev)
        call("ebsd_cnn_transpose", ptr(g16), 0, M, self.cout, ld16, ptr(gT), gT.shape[0], M, s)
        colsT = torch.empty((round_up(self.K_pad, 256), M), dtype=torch.bfloat16, device=dev)
        cols = keep["cols"] if "cols" in keep else self._im2col(keep["x"], B, H, W)
        call("ebsd_cnn_transpose", ptr(cols), 0, M, self.K_pad, self.K_pad, ptr(colsT), colsT.shape[0], M, s)
        kernels.gemm_nt(gT, colsT, self.gw, m_valid=self.cout, n_valid=self.K)
        if not need_dx:
            return None
        dcols = torch.empty((M, self.K), dtype=torch.float32, device=dev)
        kernels.gemm_nt(g16, self.w16t, dcols, m_valid=M, n_valid=self.K)
        dx = torch.empty((B, H, W, self.cin), dtype=torch.float32, device=dev)
        call("ebsd_cnn_col2im", ptr(dcols), self.K, B, H, W, self.cin, ptr(dx), s)
        return dx


class _Dense:
    def __init__(self, nin: int, nout: int, gen: torch.Generator, device, relu: bool):
        self.nin, self.nout, self.relu = nin, nout, relu
        scale = math.sqrt((2.0 if relu else 1.0) / nin)
        self.w = (torch.randn((nout, nin), generator=gen) * scale).to(device)
        self.b = torch.zeros(nout, device=device)
        self.state = [torch.zeros_like(self.w), torch.zeros_like(self.w), torch.zeros_like(self.b),
                      torch.zeros_like(self.b)]
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)

    def forward(self, x: torch.Tensor, keep: dict, tf32: bool = False):
        """y = act(x W^T + b). tf32 (inference): the product on the tensor
        cores (ebsd_gemm_f32) when the layer is wide, then bias and ReLU;
        training keeps the FP32 SIMT kernel."""
        B = x.shape[0]
        y = torch.empty((B, self.nout), dtype=torch.float32, device=x.device)
        y16 = torch.empty((B, self.nout), dtype=torch.bfloat16, device=x.device) if self.relu else None
        if tf32 and self.nin >= 512 and self.nin % 4 == 0 and x.stride(1) == 1 and x.stride(0) % 4 == 0:
            kernels.gemm_f32(x, self.w, y)
            if self.relu:
                call("ebsd_cnn_bias_act", ptr(y), self.nout, ptr(self.b), B, self.nout, 1, ptr(y16), self.nout,
                     ptr(y), _stream(x))
            else:
                y += self.b
        else:
            call("ebsd_cnn_dense_fwd", ptr(x), x.stride(0), ptr(self.w), ptr(self.b), B, self.nout, self.nin,
                 int(self.relu), ptr(y), ptr(y16), _stream(x))
        keep.update(x=x, y16=y16)
        return y

    def backward(self, dy: torch.Tensor, keep: dict, need_dx: bool):
        B = dy.shape[0]
        s = _stream(dy)
        if self.relu:
            g = torch.empty_like(dy)
            call("ebsd_cnn_relu_grad", ptr(dy), self.nout, ptr(keep["y16"]), self.nout, B, self.nout, ptr(g), None,
                 self.nout, s)
            dy = g
        dx = torch.empty((B, self.nin), dtype=torch.float32, device=dy.device) if need_dx else None
        x = keep["x"]
        call("ebsd_cnn_dense_bwd", ptr(dy), ptr(x), x.stride(0), ptr(self.w), B, self.nout, self.nin, ptr(self.gw),
             ptr(self.gb), ptr(dx), s)
        return dx


class OrientationCNN:
    """Orientation-proposal network (see module doc). Inputs: (B, H, W)
    patterns, zero-mean with unit per-pixel variance, B a multiple of 128."""

    CHANNELS = (1, 32, 64, 128, 256, 256)

    def __init__(self, detector_shape=(128, 128), laue_id: int = 11, seed: int = 0, device="cuda", hidden: int = 64):
        self.device = torch.device(device)
        self.H, self.W = detector_shape
        self.laue = int(laue_id)
        gen = torch.Generator().manual_seed(seed)
        self.convs = [_Conv(a, b, gen, self.device) for a, b in zip(self.CHANNELS[:-1], self.CHANNELS[1:])]
        h, w = self.H, self.W
        for _ in self.convs:
            h, w = (h + 1) // 2, (w + 1) // 2
        self.feat = h * w * self.CHANNELS[-1]
        self.fc1 = _Dense(self.feat, hidden, gen, self.device, relu=True)
        self.fc2 = _Dense(hidden, 6, gen, self.device, relu=False)
        self.step_count = 0
        self._keep: List[dict] = []

    def n_params(self) -> int:
        return sum(t.numel() for c in self.convs for t in c.params()) + sum(
            t.numel() for d in (self.fc1, self.fc2) for t in (d.w, d.b))

    def forward(self, x: torch.Tensor, keep: bool = True) -> torch.Tensor:
        """x: (B, H, W) float32 -> (B, 6) float32 6-D rotation outputs. With
        keep=False the activations needed by backward() are not retained."""
        B = x.shape[0]
        if B % 128:
            raise ValueError("batch size must be a multiple of 128")
        x16 = torch.empty((B, self.H, self.W), dtype=torch.bfloat16, device=x.device)
        call("ebsd_cnn_scale_cast", ptr(x.contiguous()), x.numel(), 1.0, ptr(x16), _stream(x))
        self._keep = []
        a, h, w = x16, self.H, self.W
        a32 = None
        for i, conv in enumerate(self.convs):
            saved = {}
            a, a32, h, w = conv.forward(a, B, h, w, saved, want32=(i == len(self.convs) - 1))
            if keep:
                self._keep.append(saved)
        k1, k2 = {}, {}
        hid = self.fc1.forward(a32.view(B, -1), k1, tf32=not keep)
        out = self.fc2.forward(hid, k2)
        if keep:
            self._keep += [k1, k2]
        return out

    def check_status(self) -> None:
        """Raise if a forward GEMM reported a device timeout (reads the
        status words, so it synchronises)."""
        for i, c in enumerate(self.convs):
            st = int(c.status.item())
            if st:
                c.status.zero_()
                raise RuntimeError(f"convolution {i} GEMM reported device status {st:#x}")

    def backward(self, dout: torch.Tensor) -> None:
        k1, k2 = self._keep[-2], self._keep[-1]
        dh = self.fc2.backward(dout, k2, need_dx=True)
        dfeat = self.fc1.backward(dh, k1, need_dx=True)
        d = dfeat
        for i in range(len(self.convs) - 1, -1, -1):
            conv = self.convs[i]
            keep = self._keep[i]
            d = conv.backward(d.reshape(keep["M"], conv.cout), keep, need_dx=(i > 0))

    def adam_step(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8, wd: float = 0.0):
        self.step_count += 1
        t = self.step_count
        s = torch.cuda.current_stream(self.device).cuda_stream
        for c in self.convs:
            m, v, mb, vb = c.state
            call("ebsd_cnn_adam", ptr(c.w), ptr(m), ptr(v), ptr(c.gw), c.cout, c.K, lr, b1, b2, eps, t, wd,
                 ptr(c.w16), c.K_pad, ptr(c.w16t), c.ld_t, s)
            call("ebsd_cnn_adam", ptr(c.b), ptr(mb), ptr(vb), ptr(c.gb), 1, c.cout, lr, b1, b2, eps, t, 0.0, None, 0,
                 None, 0, s)
        for d in (self.fc1, self.fc2):
            m, v, mb, vb = d.state
            call("ebsd_cnn_adam", ptr(d.w), ptr(m), ptr(v), ptr(d.gw), d.nout, d.nin, lr, b1, b2, eps, t, wd, None, 0,
                 None, 0, s)
            call("ebsd_cnn_adam", ptr(d.b), ptr(mb), ptr(vb), ptr(d.gb), 1, d.nout, lr, b1, b2, eps, t, 0.0, None, 0,
                 None, 0, s)

    def loss_and_grad(self, out: torch.Tensor, q_true: torch.Tensor):
        B = out.shape[0]
        loss = torch.empty(B, dtype=torch.float32, device=out.device)
        grad = torch.empty_like(out)
        call("ebsd_rot6d_sym_loss", ptr(out), ptr(q_true.contiguous()), B, self.laue, 1.0 / B, ptr(loss), ptr(grad),
             _stream(out))
        return loss, grad

    def predict_quaternions(self, x: torch.Tensor, keep: bool = False) -> torch.Tensor:
        out = self.forward(x, keep=keep)
        qu = torch.empty((x.shape[0], 4), dtype=torch.float32, device=x.device)
        call("ebsd_zh_to_qu", ptr(out), out.shape[0], ptr(qu), None, _stream(out))
        return qu

    def state_dict(self) -> dict:
        d = {}
        for i, c in enumerate(self.convs):
            d[f"conv{i}.w"], d[f"conv{i}.b"] = c.w.clone(), c.b.clone()
        for n, l in (("fc1", self.fc1), ("fc2", self.fc2)):
            d[f"{n}.w"], d[f"{n}.b"] = l.w.clone(), l.b.clone()
        return d


def unit_variance_patterns(patterns: torch.Tensor) -> torch.Tensor:
    """(B, H, W) -> zero-mean patterns with unit per-pixel variance, the
    network's input normalisation (row preparation by the K2 kernel)."""
    B, H, W = patterns.shape
    P = H * W
    f32 = torch.empty((B, P), dtype=torch.float32, device=patterns.device)
    norm = torch.empty(B, dtype=torch.float32, device=patterns.device)
    kernels.prep_patterns(patterns.float().contiguous(), kernels.RowBuffers(f32=f32, norm=norm))
    return (f32 * (math.sqrt(P) / norm.clamp_min(1e-12))[:, None]).view(B, H, W)


def train_proposal_cnn(master_pattern: torch.Tensor, geometry, laue_id: int = 11, steps: int = 1000,
                       batch: int = 256, lr: float = 2e-3, mean_counts: float = 100.0, seed: int = 0,
                       model: Optional[OrientationCNN] = None, log_every: int = 0):
    """Train on freshly projected noisy patterns (random orientations, blur,
    Poisson noise) every step. Returns (model, per-step mean losses)."""
    from .synthetic import random_quaternions, synthetic_patterns

    dev = master_pattern.device
    H, W = geometry.detector_shape
    if model is None:
        model = OrientationCNN((H, W), laue_id, seed=seed, device=dev)
    losses = []
    for it in range(steps):
        q = random_quaternions(batch, seed * 1000003 + it).to(dev)
        pats = synthetic_patterns(master_pattern, geometry, q, mean_counts=mean_counts, seed=seed + 7 * it,
                                  chunk=batch)
        x = pats * math.sqrt(H * W)
        out = model.forward(x)
        loss, grad = model.loss_and_grad(out, q)
        model.backward(grad)
        frac = it / max(1, steps - 1)
        model.adam_step(lr=lr * (0.5 * (1 + math.cos(math.pi * frac))) + 1e-5)
        losses.append(loss.mean())
        if log_every and it % log_every == 0:
            print(f"step {it} loss {float(loss.mean()):.4f}", flush=True)
    return model, torch.stack(losses).cpu()
