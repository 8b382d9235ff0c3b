"""Non-local pattern averaging (mirror of ebsdtorch/preprocessing/nlpar.py:
19-192; Brewick, Wright and Rowenhorst, Ultramicroscopy 200 (2019) 50-61).

`nlpar` keeps the reference's signature and result. The two passes that read
the patterns, the squared distances to every window neighbour and the
weighted average, are CUDA kernels that stage an 8 x 8 tile of the scan plus
its halo in shared memory once per 32-pixel chunk (`ebsd_nlpar_dists`,
`ebsd_nlpar_average`). The per-point arithmetic between them follows the
reference's formulas in FP32 (`ebsd_nlpar_weights`): noise estimate from
window offsets 1..8, normalised distances, the Newton fit of the global
coefficient on offsets 0..8 (each iteration one launch whose last block
updates the coefficient on the device, so nothing synchronises with the
host) and the masked softmax.
"""

from __future__ import annotations

import torch
from torch import Tensor

from .._capi import call, load, ptr
from .patterns import _stream, device_rows
from .._device import on_data_device

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


@on_data_device
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
    # noise estimate, normalised distances, Newton fit of the coefficient
    # and the masked softmax, in place: dists becomes the weights
    ws_bytes = int(load().ebsd_nlpar_workspace_bytes(hs, ws))
    workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    call("ebsd_nlpar_weights", ptr(dists), hs, ws, n_pix, ptr(off_d), K, float(coeff), float(coeff_fit_tol),
         float(center_logit_bias), ptr(workspace), ws_bytes, stream)
    weights = dists

    out = torch.empty_like(x)
    for o0 in range(0, K, OFFSETS_PER_CALL):
        call("ebsd_nlpar_average", ptr(x), hs, ws, n_pix, x.stride(0), k_rad, ptr(off_d), o0,
             min(OFFSETS_PER_CALL, K - o0), K, ptr(weights), int(o0 > 0), ptr(out), out.stride(0), stream)
    return back(out).view(hs, ws, hp, wp)
