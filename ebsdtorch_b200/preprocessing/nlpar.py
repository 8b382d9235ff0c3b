"""Non-local pattern averaging (mirror of ebsdtorch/preprocessing/nlpar.py:
19-192; Brewick, Wright and Rowenhorst, Ultramicroscopy 200 (2019) 50-61).

`nlpar` keeps the reference's signature and result. The two passes that read
the patterns, the squared distances to every window neighbour and the
weighted average, are CUDA kernels that stage an 8 x 8 tile of the scan plus
its halo in shared memory once per 32-pixel chunk (`ebsd_nlpar_dists`,
`ebsd_nlpar_average`). The per-point arithmetic between them, on
(scan_h, scan_w, window) tensors, follows the reference's formulas with
torch on the same device: noise estimate from window offsets 1..8,
normalised distances, the Newton fit of the global coefficient on offsets
0..8 (run for its 10 iterations with a done flag instead of a
host-side break, so nothing synchronises) and the masked softmax.
"""

from __future__ import annotations

import torch
import torch.nn.functional as F
from torch import Tensor

from .._capi import call, ptr
from .patterns import _stream, device_rows

MAX_RADIUS = 7        # the kernels' halo limit
OFFSETS_PER_CALL = 128


def nlpar_offsets(k_rad: int) -> Tensor:
    """(K, 2) window offsets (di, dj), K = (2 k_rad + 1)^2, in the reference's
    order (nlpar.py:77-91): sorted by L1 norm with torch.argsort, so offset 0
    is the point itself, 1..4 the axial neighbours and 5..8 four offsets of
    L1 norm 2, chosen by how argsort breaks ties (the reference's "8 nearest
    neighbours")."""
    oc = torch.stack(torch.meshgrid(torch.arange(-k_rad, k_rad + 1), torch.arange(-k_rad, k_rad + 1), indexing="ij"),
                     dim=-1).reshape(-1, 2)
    return oc[torch.argsort(torch.sum(torch.abs(oc), dim=-1))]


def nlpar(data: Tensor, k_rad: int = 5, coeff: float = 0.375, coeff_fit_tol: float = 1e-6,
          center_logit_bias: float = 0.0) -> Tensor:
    """Denoise a (scan_h, scan_w, H, W) scan; returns the same shape on the
    input's device (FP32)."""
    if len(data.shape) != 4:
        raise ValueError("The EBSD pattern data tensor must have 4 dimensions.")
    if not 1 <= k_rad <= MAX_RADIUS:
        raise ValueError(f"k_rad must be in [1, {MAX_RADIUS}], got {k_rad}")
    hs, ws, hp, wp = data.shape
    n_pix = hp * wp
    x, back = device_rows(data, n_pix)
    dev = x.device
    stream = _stream(x)
    off = nlpar_offsets(k_rad)
    K = off.shape[0]
    off_d = off.to(device=dev, dtype=torch.int32).contiguous()

    dists = torch.empty((hs * ws, K), dtype=torch.float32, device=dev)
    for o0 in range(0, K, OFFSETS_PER_CALL):
        call("ebsd_nlpar_dists", ptr(x), hs, ws, n_pix, x.stride(0), k_rad, ptr(off_d), o0,
             min(OFFSETS_PER_CALL, K - o0), K, ptr(dists), stream)
    dists = dists.view(hs, ws, K)

    # neighbour coordinates of every (point, offset) and the out-of-scan mask
    off_l = off.to(dev)
    yy = torch.arange(hs, device=dev).view(hs, 1, 1) + off_l[:, 0].view(1, 1, K)
    xx = torch.arange(ws, device=dev).view(1, ws, 1) + off_l[:, 1].view(1, 1, K)
    out_of_scan = (yy < 0) | (yy >= hs) | (xx < 0) | (xx >= ws)

    # noise level per point from window offsets 1..8 (nlpar.py:123-126)
    sigma_hat = torch.sqrt(torch.min(dists[:, :, 1:9], dim=-1).values / (2 * n_pix))
    sigma_pad = F.pad(sigma_hat, (k_rad,) * 4, mode="constant", value=1.0)
    sigma_other = sigma_pad[yy + k_rad, xx + k_rad]
    s2 = sigma_hat[..., None] ** 2 + sigma_other**2
    dists = (dists - n_pix * s2) / (2**0.5 * n_pix**0.5 * s2)
    weights = -dists.clamp_min_(0.0)

    # Newton fit of the global coefficient: the mean softmax weight of the
    # point itself over offsets 0..8 equals coeff (nlpar.py:150-173)
    nn_w = weights[:, :, :9]
    g = torch.ones((), dtype=torch.float32, device=dev)
    done = torch.zeros((), dtype=torch.bool, device=dev)
    for _ in range(10):
        g2 = g**2
        e = torch.exp(nn_w / g2)
        obj = torch.mean(torch.softmax(nn_w / g2, dim=-1)[:, :, 0]) - coeff
        grad = torch.mean(-2 * torch.exp(nn_w[:, :, 0] / g2)
                          * (torch.sum(nn_w[:, :, [0]] * e, dim=-1) - torch.sum(nn_w * e, dim=-1))
                          / (g**3 * torch.sum(e, dim=-1) ** 2))
        g = torch.where(done, g, g - obj / grad)
        done = done | (torch.abs(obj) < coeff_fit_tol)
    weights = weights / g**2
    if center_logit_bias > 0:
        weights[:, :, 0] += center_logit_bias
    weights = torch.softmax(weights.masked_fill_(out_of_scan, -torch.inf), dim=-1).contiguous()

    out = torch.empty_like(x)
    for o0 in range(0, K, OFFSETS_PER_CALL):
        call("ebsd_nlpar_average", ptr(x), hs, ws, n_pix, x.stride(0), k_rad, ptr(off_d), o0,
             min(OFFSETS_PER_CALL, K - o0), K, ptr(weights), int(o0 > 0), ptr(out), out.stride(0), stream)
    return back(out).view(hs, ws, hp, wp)
