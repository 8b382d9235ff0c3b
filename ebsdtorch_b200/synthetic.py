"""Seeded synthetic EBSD data (stands in for the reference demo's kikuchipy
nickel master pattern and scans, which are not available offline).

Master pattern: sum of Gaussian-profile Kikuchi bands centred on the great
circles of the cubic {111}, {200}, {220} and {311} planes, band width
proportional to 1/d (so to |hkl|), one intensity per family drawn from
U[0.3, 1], plus 5 % Gaussian noise; evaluated at every modified-Lambert pixel
of both hemispheres (inverse Rosca-Lambert map, sphere.py:95-142) and laid
out side by side (H, 2W). For a non-cubic Laue group the band families are
seeded random plane normals closed under the group's rotations, so the
pattern has exactly that symmetry. Queries: patterns projected at seeded uniform random
orientations (Shoemake, sampling.py:135-176), Gaussian blurred (sigma 1 px),
scaled to a mean count, Poisson sampled, then zero-mean / unit-norm.
"""

from __future__ import annotations

import itertools
import math
from typing import Tuple

import torch

from . import kernels
from .kernels import RowBuffers

FAMILIES = ((1, 1, 1), (2, 0, 0), (2, 2, 0), (3, 1, 1))


def _family_normals(hkl):
    out = set()
    for perm in set(itertools.permutations(hkl)):
        for signs in itertools.product((1, -1), repeat=3):
            v = tuple(p * s for p, s in zip(perm, signs))
            if v == (0, 0, 0):
                continue
            # a plane and its opposite normal are the same great circle
            first = next(x for x in v if x != 0)
            if first < 0:
                v = tuple(-x for x in v)
            out.add(v)
    return sorted(out)


def inv_lambert_north(u: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """Square [-1, 1]^2 -> northern unit hemisphere (Rosca 2010)."""
    pi = math.pi
    xa = u.abs() * math.sqrt(pi / 2)
    ya = v.abs() * math.sqrt(pi / 2)
    cond = xa >= ya
    xn = torch.where(cond, xa, ya)
    yn = torch.where(cond, ya, xa)
    ang = torch.where(xn > 0, pi * yn / (4 * xn.clamp_min(1e-30)), torch.zeros_like(xn))
    rr = (2 * xn / pi) * torch.sqrt((pi - xn * xn).clamp_min(0.0))
    xh, yh = rr * torch.cos(ang), rr * torch.sin(ang)
    z = 1 - 2 * xn * xn / pi
    x = torch.copysign(torch.where(cond, xh, yh), u)
    y = torch.copysign(torch.where(cond, yh, xh), v)
    return torch.stack((x, y, z), dim=-1)


def _axis_angle_quat(axis, angle):
    a = torch.tensor(axis, dtype=torch.float64)
    a = a / a.norm()
    return torch.cat((torch.tensor([math.cos(angle / 2)], dtype=torch.float64), math.sin(angle / 2) * a))


def _qmul(a, b):
    w1, x1, y1, z1 = a.unbind(-1)
    w2, x2, y2, z2 = b.unbind(-1)
    return torch.stack((w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                        w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2), dim=-1)


# generators of the proper rotation group of each Laue class (axis, order)
_LAUE_GENERATORS = {
    1: [], 2: [((0, 1, 0), 2)], 3: [((0, 0, 1), 2), ((1, 0, 0), 2)], 4: [((0, 0, 1), 4)],
    5: [((0, 0, 1), 4), ((1, 0, 0), 2)], 6: [((0, 0, 1), 3)], 7: [((0, 0, 1), 3), ((1, 0, 0), 2)],
    8: [((0, 0, 1), 6)], 9: [((0, 0, 1), 6), ((1, 0, 0), 2)], 10: [((0, 0, 1), 2), ((1, 1, 1), 3)],
    11: [((0, 0, 1), 4), ((1, 1, 1), 3)],
}


def laue_rotations(laue_group: int) -> torch.Tensor:
    """(n, 4) float64 quaternions of the proper rotations of a Laue class
    (closure of its generators)."""
    elems = [torch.tensor([1.0, 0.0, 0.0, 0.0], dtype=torch.float64)]
    gens = [_axis_angle_quat(ax, 2 * math.pi / order) for ax, order in _LAUE_GENERATORS[laue_group]]
    changed = True
    while changed:
        changed = False
        for a in list(elems):
            for g in gens:
                c = _qmul(a, g)
                if not any(torch.allclose(c, e, atol=1e-9) or torch.allclose(c, -e, atol=1e-9) for e in elems):
                    elems.append(c)
                    changed = True
    return torch.stack(elems)


def _qrot(q, v):
    w, x, y, z = q.unbind(-1)
    t = 2 * torch.stack((y * v[2] - z * v[1], z * v[0] - x * v[2], x * v[1] - y * v[0]))
    return v + w * t + torch.stack((y * t[2] - z * t[1], z * t[0] - x * t[2], x * t[1] - y * t[0]))


def synthetic_master_pattern(n: int, seed: int = 0, width_per_hkl: float = 0.012, noise: float = 0.05,
                             device="cpu", laue_group: int = 11, n_families: int = 6) -> torch.Tensor:
    """(n, 2n) float32 side-by-side master pattern (north | south). Laue group
    11 (m-3m) uses the cubic {111}, {200}, {220}, {311} families; any other
    group `n_families` seeded random plane normals, each closed under the
    group's rotations."""
    g = torch.Generator().manual_seed(seed)
    c = (2 * torch.arange(n, dtype=torch.float64) + 1) / n - 1
    vv, uu = torch.meshgrid(c, c, indexing="ij")  # rows <-> v, columns <-> u
    north = inv_lambert_north(uu, vv)
    south = north * torch.tensor([1.0, 1.0, -1.0], dtype=torch.float64)
    pts = torch.cat((north, south), dim=1)  # (n, 2n, 3)
    img = torch.zeros(pts.shape[:2], dtype=torch.float64)
    if laue_group == 11:
        families = [(0.3 + 0.7 * torch.rand((), generator=g, dtype=torch.float64),
                     width_per_hkl * math.sqrt(sum(h * h for h in hkl)),
                     [torch.tensor(nrm, dtype=torch.float64) for nrm in _family_normals(hkl)]) for hkl in FAMILIES]
    else:
        rots = laue_rotations(laue_group)
        families = []
        for _ in range(n_families):
            nv = torch.randn(3, generator=g, dtype=torch.float64)
            inten = 0.3 + 0.7 * torch.rand((), generator=g, dtype=torch.float64)
            hkl_len = 1.5 + 2.0 * torch.rand((), generator=g, dtype=torch.float64)
            orbit = []
            for q in rots:
                m = _qrot(q, nv / nv.norm())
                if not any(abs(float(m @ o)) > 1 - 1e-9 for o in orbit):
                    orbit.append(m)
            families.append((inten, width_per_hkl * float(hkl_len), orbit))
    for inten, sigma, normals in families:
        for nv in normals:
            nv = nv / nv.norm()
            s = pts @ nv  # sine of the angular distance to the great circle
            img += inten * torch.exp(-0.5 * (s / sigma) ** 2)
    img = img / img.max()
    img = img + noise * torch.randn(img.shape, generator=g, dtype=torch.float64)
    return img.float().to(device)


def random_quaternions(n: int, seed: int) -> torch.Tensor:
    """Uniform random unit quaternions (Shoemake), w >= 0, float32."""
    g = torch.Generator().manual_seed(seed)
    u, v, w = (torch.rand(n, generator=g, dtype=torch.float64) for _ in range(3))
    q = torch.stack((torch.sqrt(1 - u) * torch.sin(2 * math.pi * v), torch.sqrt(1 - u) * torch.cos(2 * math.pi * v),
                     torch.sqrt(u) * torch.sin(2 * math.pi * w), torch.sqrt(u) * torch.cos(2 * math.pi * w)), dim=1)
    q = torch.where(q[:, :1] < 0, -q, q)
    return q.float()


def _gaussian_blur(x: torch.Tensor, sigma: float) -> torch.Tensor:
    r = max(1, int(math.ceil(3 * sigma)))
    t = torch.arange(-r, r + 1, dtype=torch.float32, device=x.device)
    k = torch.exp(-0.5 * (t / sigma) ** 2)
    k = k / k.sum()
    y = x.unsqueeze(1)
    y = torch.nn.functional.conv2d(torch.nn.functional.pad(y, (r, r, 0, 0), mode="replicate"), k.view(1, 1, 1, -1))
    y = torch.nn.functional.conv2d(torch.nn.functional.pad(y, (0, 0, r, r), mode="replicate"), k.view(1, 1, -1, 1))
    return y.squeeze(1)


def synthetic_patterns(master_pattern: torch.Tensor, geometry, quats: torch.Tensor, mean_counts: float = 200.0,
                       blur_sigma: float = 1.0, seed: int = 0, chunk: int = 8192, out: torch.Tensor = None,
                       counts: bool = False) -> torch.Tensor:
    """(n, H, W) float32 noisy, zero-mean, unit-norm patterns on the master
    pattern's device (or written into `out`, which may be pinned host memory).
    With counts=True the Poisson detector counts themselves are returned
    (uint16, not normalised), as a camera delivers them."""
    dev = master_pattern.device
    h, w = geometry.detector_shape
    coords = geometry.get_coords_sample_frame(binning=(1, 1)).double().cpu()
    rays = (coords / coords.norm(dim=-1, keepdim=True)).t().contiguous().float().to(dev)
    n = quats.shape[0]
    if out is None:
        out = torch.empty((n, h, w), dtype=torch.uint16 if counts else torch.float32, device=dev)
    g = torch.Generator(device=dev).manual_seed(seed)
    for s0 in range(0, n, chunk):
        s1 = min(n, s0 + chunk)
        raw = torch.empty((s1 - s0, h * w), dtype=torch.float32, device=dev)
        kernels.project(master_pattern, rays, quats[s0:s1].to(dev).contiguous(), RowBuffers(f32=raw),
                        subtract_mean=False)
        x = raw.view(-1, h, w)
        x = x - x.amin(dim=(1, 2), keepdim=True)
        if blur_sigma > 0:
            x = _gaussian_blur(x, blur_sigma)
        x = x * (mean_counts / x.mean(dim=(1, 2), keepdim=True).clamp_min(1e-12))
        x = torch.poisson(x, generator=g)
        if counts:
            out[s0:s1].copy_(x.clamp_max(65535).to(torch.int32).to(torch.uint16), non_blocking=True)
            continue
        x = x - x.mean(dim=(1, 2), keepdim=True)
        x = x / x.flatten(1).norm(dim=1).clamp_min(1e-12).view(-1, 1, 1)
        out[s0:s1].copy_(x, non_blocking=True)
    return out


def make_case(mp_size: int, detector: Tuple[int, int], n_queries: int, seed: int = 0, mean_counts: float = 200.0,
              proj_center=(0.5, 0.5, 0.6), device="cuda"):
    """(MasterPattern, EBSDGeometry, ExperimentPatterns, true orientations)."""
    from .ebsd.experiment_pats import ExperimentPatterns
    from .ebsd.geometry import EBSDGeometry
    from .ebsd.master_pattern import MasterPattern

    mp_t = synthetic_master_pattern(mp_size, seed=seed, device=device)
    mp = MasterPattern(mp_t, laue_group=11)
    geom = EBSDGeometry(detector, tilts_degrees=(0.0, 70.0, 0.0), proj_center=proj_center)
    q = random_quaternions(n_queries, seed + 1).to(device)
    pats = synthetic_patterns(mp_t, geom, q, mean_counts=mean_counts, seed=seed + 2)
    return mp, geom, ExperimentPatterns(pats), q
