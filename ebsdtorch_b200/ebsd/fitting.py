"""Pattern-centre fitting by the spatial FFT search (mirror of
ebsdtorch/ebsd/fitting.py:54-540).

`spatial_fft_pc_fitter` keeps the reference's signature and result. For
each pc_z of linspace(pc_z_min, pc_z_max, pc_z_steps) the orientation
dictionary is simulated on the detector enlarged by the pc_x / pc_y search
range (`ebsd_project_dictionary`, the same projector as dictionary
indexing) and circularly cross-correlated with every zero-padded
experimental pattern, which scores all (pc_x, pc_y) shifts at once.
Up to 127 x 127 enlarged pixels the correlation runs in the project's
kernels: 2-D DFTs as tensor-core matrix products (`ebsd_pcfit_spectra`
for the spectra, `ebsd_pcfit_xcorr_max` for the inverse transforms of the
spectrum products fused with the max over the batch per (pattern, shift),
`ebsd_pcfit_fold` for the running best per pc_z); no correlation map
reaches memory. Larger detectors use cuFFT (torch.fft) and
`ebsd_pcfit_reduce`, which applies the fftshift, takes the max and argmax
over the chunk and folds them into the running best. A second kernel
prepares the patterns (`ebsd_pcfit_prep`): min-max, zero-mean and zero
padding in one pass. The fit is the argmax of the mean over patterns;
nothing synchronises with the host before it.

Differences, by design:

* Widths of the enlarged detector may be odd (irfft2 gets the output size;
  the reference raises a shape error).
* The caller's patterns are not modified (the reference scales them in
  place).
* `orientation_index="global"` (keyword-only) returns the winning
  orientation by its index in the whole dictionary. The default
  "reference" reproduces the reference, which indexes the dictionary with
  the position inside the winning batch of `dictionary_indexing_batch_size`
  orientations.
* metric="mi" (mutual information) raises NotImplementedError.
"""

from __future__ import annotations

from typing import Tuple

import numpy as np
import torch
from torch import Tensor

from .. import kernels
from .._capi import call, load, ptr
from ..kernels import RowBuffers
from ..s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle
from .geometry import bruker_geometry_to_SE3
from .indexing import _device, _master_pattern_tensor
from .._device import on_data_device

MAX_PRODUCT_BYTES = 4 << 30  # spectrum product of one correlation launch


def bruker_geometries_to_SE3(pattern_centers: Tensor, primary_tilt_deg: Tensor, secondary_tilt_deg: Tensor,
                             detector_shape: Tuple[int, int]) -> Tuple[Tensor, Tensor]:
    """Rotations (N, 3, 3) and translations (N, 3) of Bruker pattern centres
    (N, 3) (fitting.py:54-115)."""
    pcs = pattern_centers.reshape(-1, 3).double().cpu().numpy()
    rots, ts = [], []
    for pc in pcs:
        r, t = bruker_geometry_to_SE3(pc, float(primary_tilt_deg), float(secondary_tilt_deg), detector_shape)
        rots.append(r)
        ts.append(t)
    dev, dt = pattern_centers.device, pattern_centers.dtype
    return (torch.from_numpy(np.stack(rots)).to(dev, dt), torch.from_numpy(np.stack(ts)).to(dev, dt))


def bruker_geometry_from_SE3(rotation_matrix: Tensor, translation_vector: Tensor,
                             detector_shape: Tuple[int, int]):
    """Pattern centres and the two tilts (degrees) of SE(3) detector maps
    (fitting.py:118-157, the inverse of bruker_geometries_to_SE3)."""
    tx, ty, tz = torch.unbind(translation_vector, dim=-1)
    rows, cols = float(detector_shape[0]), float(detector_shape[1])
    cos_sx = rotation_matrix[..., 1, 1]
    dt = torch.acos((rotation_matrix[..., 0, 2] / cos_sx).clamp(-1, 1))
    sx = torch.acos(cos_sx.clamp(-1, 1))
    pcx = (tx * torch.sin(sx) * torch.cos(dt) - ty * torch.cos(sx) - tz * torch.sin(dt) * torch.sin(sx) + 0.5) / cols
    pcy = (tx * torch.sin(dt) + tz * torch.cos(dt) + 0.5) / rows
    pcz = (tx * torch.cos(dt) * torch.cos(sx) + ty * torch.sin(sx) - tz * torch.sin(dt) * torch.cos(sx)) / rows
    return torch.stack([pcx, pcy, pcz], dim=-1), torch.rad2deg(dt), torch.rad2deg(sx)


def get_3D_pixel_coords(detector_shape: Tuple[int, int], device: torch.device, binning: int = 1,
                        dtype: torch.dtype = torch.float32) -> Tensor:
    """(H/b * W/b, 3) detector-frame coordinates of the binned pixel centres,
    z = 0 (fitting.py:160-217)."""
    return get_3D_pixel_coords_with_periphery(detector_shape, device, 0.5, 0.5, 0.5, 0.5, binning, dtype)[0]


def get_3D_pixel_coords_with_periphery(detector_shape: Tuple[int, int], device: torch.device, pc_x_min: float,
                                       pc_x_max: float, pc_y_min: float, pc_y_max: float, binning: int = 1,
                                       dtype: torch.dtype = torch.float32):
    """Pixel coordinates of the detector enlarged by the pattern-centre
    search range, the padding (w_prior, w_after, h_prior, h_after) and the
    enlarged shape (fitting.py:219-289): per axis linspace(0.5 (b - 1) -
    prior, size + after - 0.5 (b - 1), n) with the reference's int()
    truncation of the padding."""
    bf = float(binning)
    wpp = int((0.5 - pc_x_min) * detector_shape[1] / bf)
    wpa = int((pc_x_max - 0.5) * detector_shape[1] / bf)
    hpp = int((0.5 - pc_y_min) * detector_shape[0] / bf)
    hpa = int((pc_y_max - 0.5) * detector_shape[0] / bf)
    shape = (detector_shape[0] // binning + hpp + hpa, detector_shape[1] // binning + wpp + wpa)
    ii = torch.linspace(0.5 * (bf - 1) - hpp, detector_shape[0] + hpa - 0.5 * (bf - 1), shape[0], dtype=dtype,
                        device=device)
    jj = torch.linspace(0.5 * (bf - 1) - wpp, detector_shape[1] + wpa - 0.5 * (bf - 1), shape[1], dtype=dtype,
                        device=device)
    pix = torch.stack(torch.meshgrid(ii, jj, indexing="ij"), dim=-1).reshape(-1, 2)
    pix = torch.cat([pix, torch.zeros_like(pix[..., :1])], dim=-1)
    return pix, (wpp, wpa, hpp, hpa), shape


def apply_geometry(pixel_coords: Tensor, rotation_matrix: Tensor, translation: Tensor) -> Tensor:
    """Unit sample-frame directions of detector pixels (fitting.py:292-321)."""
    c = torch.matmul(rotation_matrix, pixel_coords[..., None]).squeeze(-1) + translation
    return c / torch.norm(c, dim=-1, keepdim=True)


def generate_dictionary_coords(pixel_coords: Tensor, quats: Tensor, rotation_matrix: Tensor,
                               translation: Tensor) -> Tensor:
    """(N_ori, N_pix, 3) pixel directions rotated by each orientation,
    q (0, v) q* (fitting.py:324-356)."""
    c = apply_geometry(pixel_coords, rotation_matrix, translation)[None, :, :].expand(quats.shape[0], -1, -1)
    w, u = quats[:, None, :1], quats[:, None, 1:].expand_as(c)
    t = 2.0 * torch.cross(u, c, dim=-1)
    return c + w * t + torch.cross(u, t, dim=-1)


def _rays_soa(pix64: np.ndarray, pc_z: float, primary_tilt_deg: float, secondary_tilt_deg: float,
              detector_shape, device) -> Tensor:
    rot, t = bruker_geometry_to_SE3((0.5, 0.5, pc_z), -primary_tilt_deg, secondary_tilt_deg, detector_shape)
    c = pix64 @ rot.T + t
    c = c / np.linalg.norm(c, axis=1, keepdims=True)
    return torch.from_numpy(c.T.copy()).float().to(device).contiguous()


@on_data_device
def spatial_fft_pc_fitter(
    mp,
    patterns: Tensor,
    pc_x_min: float = 0.0,
    pc_x_max: float = 1.0,
    pc_y_min: float = 0.0,
    pc_y_max: float = 1.0,
    pc_z_min: float = 0.3,
    pc_z_max: float = 0.7,
    pc_z_steps: int = 16,
    primary_tilt_deg: float = 70.0,
    secondary_tilt_deg: float = 0.0,
    dictionary_resolution_deg: float = 1.0,
    dictionary_indexing_batch_size: int = 1024,
    virtual_binning: int = 1,
    metric: str = "dot",
    *,
    orientation_index: str = "reference",
    device=None,
) -> Tuple[Tensor, Tensor]:
    """Fit the pattern centre (pc_x, pc_y, pc_z) and the orientations of
    (B, 1, H, W) patterns; returns (pc (3,), quaternions (B, 4)) on the
    patterns' device."""
    if patterns.dim() != 4:
        raise ValueError("Pattern must be 4D (B, C, H, W).")
    if metric != "dot":
        raise NotImplementedError(f"metric '{metric}' is not supported (only 'dot')")
    if orientation_index not in ("reference", "global"):
        raise ValueError("orientation_index must be 'reference' or 'global'")
    B, C, H, W = patterns.shape
    if C != 1:
        raise ValueError("Only single channel patterns are supported.")
    b = int(virtual_binning)
    if H % b or W % b:
        raise ValueError("H and W must be divisible by virtual binning.")
    hb, wb = H // b, W // b
    dev = _device(mp, device)
    stream = torch.cuda.current_stream(dev).cuda_stream

    x = patterns.detach().to(dev, torch.float32).reshape(B, H, W).contiguous()
    if b > 1:
        x = kernels.avg_pool(x, b)
    pix, pad, (hp, wp) = get_3D_pixel_coords_with_periphery((H, W), torch.device("cpu"), pc_x_min, pc_x_max,
                                                            pc_y_min, pc_y_max, b)
    padded = torch.empty((B, hp, wp), dtype=torch.float32, device=dev)
    call("ebsd_pcfit_prep", ptr(x), B, hb, wb, hp, wp, pad[2], pad[0], 1, ptr(padded), stream)

    quats = sample_ori_fz_laue_angle(mp.laue_group, dictionary_resolution_deg, dev).float().contiguous()
    mp_t = _master_pattern_tensor(mp, b, dev)
    pix64 = pix.double().numpy()
    z_vals = torch.linspace(pc_z_min, pc_z_max, pc_z_steps)  # float32, as the reference's
    best = torch.zeros((pc_z_steps, B, hp, wp), dtype=torch.float32, device=dev)
    best_idx = torch.zeros((pc_z_steps, B, hp, wp), dtype=torch.int64, device=dev)

    bs = int(dictionary_indexing_batch_size)
    if xcorr_supported(hp, wp):
        _search_dft(mp_t, padded, quats, pix64, z_vals, float(primary_tilt_deg), float(secondary_tilt_deg), (H, W),
                    bs, orientation_index == "reference", best, best_idx, stream)
    else:
        _search_fft(mp_t, padded, quats, pix64, z_vals, float(primary_tilt_deg), float(secondary_tilt_deg), (H, W),
                    bs, orientation_index == "reference", best, best_idx, stream)

    avg = best.mean(dim=1)
    zi, yi, xi = (int(v) for v in torch.unravel_index(avg.argmax(), avg.shape))
    pc_x = 0.5 + float(xi - pad[0] - (wb + 1) // 2) / wb
    pc_y = 0.5 + float(yi - pad[2] - (hb + 1) // 2) / hb
    best_pc = torch.tensor([pc_x, pc_y, float(z_vals[zi])], device=patterns.device)
    best_quats = quats[best_idx[zi, :, yi, xi]].to(patterns.device)
    return best_pc, best_quats


def xcorr_supported(hp: int, wp: int) -> bool:
    """Whether the enlarged detector fits the tensor-core correlation
    kernels (2..127 rows and columns); larger ones use cuFFT."""
    return int(load().ebsd_pcfit_xcorr_table_bytes(int(hp), int(wp))) > 0


# sub-batch of the dictionary projected and transformed at once (the
# correlation itself runs per dictionary batch on the spectra)
MAX_SIM_BYTES = 2 << 30


def _search_dft(mp_t, padded, quats, pix64, z_vals, tilt, sec_tilt, det, bs, batch_local, best, best_idx, stream):
    """The search with the correlation in the project's kernels: spectra of
    the patterns and of each projected dictionary sub-batch
    (ebsd_pcfit_spectra), the per-batch max over all shifts
    (ebsd_pcfit_xcorr_max) and the running best (ebsd_pcfit_fold)."""
    dev = padded.device
    B, hp, wp = padded.shape
    n_dict = quats.shape[0]
    spec_len = 4 * (hp // 2 + 1) * (wp // 2 + 1)
    tables = torch.empty((int(load().ebsd_pcfit_xcorr_table_bytes(hp, wp)),), dtype=torch.uint8, device=dev)
    call("ebsd_pcfit_xcorr_tables", hp, wp, ptr(tables), tables.numel(), stream)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    pspec = torch.empty((B, spec_len), dtype=torch.float32, device=dev)
    call("ebsd_pcfit_spectra", ptr(padded), hp * wp, B, hp, wp, ptr(tables), ptr(pspec), ptr(status), stream)
    terms = torch.empty_like(pspec)
    call("ebsd_pcfit_pattern_terms", ptr(pspec), B, hp, wp, ptr(terms), stream)
    keys = torch.zeros((B * hp * wp,), dtype=torch.int64, device=dev)
    sub = max(1, min(bs, n_dict, MAX_SIM_BYTES // (hp * wp * 4)))
    sims = torch.empty((sub, hp * wp), dtype=torch.float32, device=dev)
    spec = torch.empty((sub, spec_len), dtype=torch.float32, device=dev)
    for zi in range(len(z_vals)):
        rays = _rays_soa(pix64, float(z_vals[zi]), tilt, sec_tilt, det, dev)
        for j in range(0, n_dict, bs):
            j_end = min(j + bs, n_dict)
            for s in range(j, j_end, sub):
                n = min(sub, j_end - s)
                kernels.project(mp_t, rays, quats[s:s + n], RowBuffers(f32=sims[:n]), subtract_mean=False)
                call("ebsd_pcfit_spectra", ptr(sims), hp * wp, n, hp, wp, ptr(tables), ptr(spec), ptr(status), stream)
                call("ebsd_pcfit_xcorr_max", ptr(spec), n, ptr(terms), B, hp, wp, ptr(tables), ptr(keys),
                     (s - j) if batch_local else s, ptr(status), stream)
            call("ebsd_pcfit_fold", ptr(keys), keys.numel(), ptr(best[zi]), ptr(best_idx[zi]), stream)
    if int(status.item()) != 0:
        raise RuntimeError("pattern-centre correlation kernels reported a device timeout")


def _search_fft(mp_t, padded, quats, pix64, z_vals, tilt, sec_tilt, det, bs, batch_local, best, best_idx, stream):
    """The search with cuFFT (torch.fft) for detectors beyond the
    tensor-core kernels' 127 x 127: rfft2 of each chunk, spectrum product
    with the patterns' conjugate spectra, irfft2, then the max over the
    chunk (ebsd_pcfit_reduce)."""
    dev = padded.device
    B, hp, wp = padded.shape
    n_dict = quats.shape[0]
    pat_fft = torch.fft.rfft2(padded).conj()  # (B, hp, wp // 2 + 1)
    wf = wp // 2 + 1
    sub = max(1, min(bs, MAX_PRODUCT_BYTES // (B * hp * wf * 8)))
    sims = torch.empty((min(sub, n_dict), hp * wp), dtype=torch.float32, device=dev)
    for zi in range(len(z_vals)):
        rays = _rays_soa(pix64, float(z_vals[zi]), tilt, sec_tilt, det, dev)
        for j in range(0, n_dict, bs):
            j_end = min(j + bs, n_dict)
            for s in range(j, j_end, sub):
                n = min(sub, j_end - s)
                kernels.project(mp_t, rays, quats[s:s + n], RowBuffers(f32=sims[:n]), subtract_mean=False)
                spec = torch.fft.rfft2(sims[:n].view(n, hp, wp))
                corr = torch.fft.irfft2(spec[:, None] * pat_fft[None], s=(hp, wp)).contiguous()
                base = (s - j) if batch_local else s
                call("ebsd_pcfit_reduce", ptr(corr), n, B, hp, wp, base, ptr(best[zi]), ptr(best_idx[zi]), stream)
                del spec, corr
