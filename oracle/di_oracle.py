"""CPU oracle for the dictionary-indexing (DI) hot path.

TEST INFRASTRUCTURE ONLY. This module is the checker: the CUDA product path
never imports, calls or falls back to it. Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it.

It is a NumPy restatement of ebsdtorch's DI algorithm (reference package
``ebsdtorch``), written so that every step can run in float64 (the accuracy
oracle) or float32 (the timed CPU baseline, mirroring the reference's own CPU
arithmetic width). Each function names the reference file:line it follows.

Parity pins: ``tests/golden/make_golden.py`` runs the reference itself (exec-
loaded from its source tree, CPU torch) on small seeded cases and commits the
inputs and outputs as ``tests/golden/*.npz``; ``tests/test_oracle_golden.py``
checks this module against every one of those fixtures.
"""

from __future__ import annotations

import math
from typing import Optional, Tuple

import numpy as np

# --------------------------------------------------------------------------
# Laue groups
# --------------------------------------------------------------------------

# Group orders including inversion, ebsdtorch/s2_and_so3/laue_generators.py:14-51
LAUE_MULT = {1: 2, 2: 4, 3: 8, 4: 8, 5: 16, 6: 6, 7: 12, 8: 12, 9: 24, 10: 24, 11: 48}


def laue_mult(laue_id: int) -> int:
    """Multiplicity of a Laue group (laue_generators.py:14-51)."""
    if laue_id not in LAUE_MULT:
        raise ValueError(f"Laue group {laue_id} is not supported")
    return LAUE_MULT[laue_id]


def _qmul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Hamilton product of (w, x, y, z) quaternions (quaternions.py:60-75)."""
    aw, ax, ay, az = np.moveaxis(a, -1, 0)
    bw, bx, by, bz = np.moveaxis(b, -1, 0)
    return np.stack(
        (
            aw * bw - ax * bx - ay * by - az * bz,
            aw * bx + ax * bw + ay * bz - az * by,
            aw * by - ax * bz + ay * bw + az * bx,
            aw * bz + ax * by - ay * bx + az * bw,
        ),
        axis=-1,
    )


def _rot_quat(axis, angle_deg) -> np.ndarray:
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    h = math.radians(angle_deg) / 2.0
    return np.concatenate(([math.cos(h)], math.sin(h) * axis))


def _close_group(gens) -> np.ndarray:
    """Closure of a set of rotation quaternions under multiplication (w >= 0)."""
    elems = [np.array([1.0, 0.0, 0.0, 0.0])]

    def canon(q):
        q = np.where(np.abs(q) < 1e-12, 0.0, q)
        if q[0] < 0 or (q[0] == 0 and tuple(-q[1:]) > tuple(q[1:])):
            q = -q
        return q

    def known(q):
        return any(abs(abs(float(np.dot(q, e))) - 1.0) < 1e-9 for e in elems)

    frontier = [canon(g) for g in gens]
    while frontier:
        nxt = []
        for g in frontier:
            if not known(g):
                elems.append(g)
                nxt.append(g)
        new = []
        for a in list(elems):
            for b in nxt:
                for c in (canon(_qmul(a, b)), canon(_qmul(b, a))):
                    if not known(c):
                        new.append(c)
        frontier = new
    return np.array(elems)


def laue_elements(laue_id: int) -> np.ndarray:
    """Rotation operators of the 11 Laue groups as (n, 4) float64 quaternions.

    Same groups as ebsdtorch/s2_and_so3/laue_generators.py:54-249, built here
    by closing each group's generators (hexagonal/trigonal axes: c along z,
    a along x), so the set, not the row order, is what matches.
    """
    z4 = _rot_quat((0, 0, 1), 90)
    z2 = _rot_quat((0, 0, 1), 180)
    z3 = _rot_quat((0, 0, 1), 120)
    z6 = _rot_quat((0, 0, 1), 60)
    x2 = _rot_quat((1, 0, 0), 180)
    d3 = _rot_quat((1, 1, 1), 120)
    gens = {
        1: [],
        2: [z2],
        3: [z2, x2],
        4: [z4],
        5: [z4, x2],
        6: [z3],
        7: [z3, x2],
        8: [z6],
        9: [z6, x2],
        10: [z2, x2, d3],
        11: [z4, x2, d3],
    }[laue_id]
    g = _close_group(gens)
    assert len(g) == laue_mult(laue_id) // 2
    return g


# --------------------------------------------------------------------------
# Cubochoric grid -> quaternions (A1)
# --------------------------------------------------------------------------

CU_HALF_EDGE = 0.5 * math.pi ** (2.0 / 3.0)


def cu2ho(cu: np.ndarray) -> np.ndarray:
    """Cubochoric -> homochoric (orientations.py:293-349).

    Restates the closed-form Rosca et al. (2014) square-to-sphere step used by
    the reference: per point, the components are ordered by magnitude
    (s <= m <= b), the magnitudes are mapped, and the signs of the input are
    copied back. Works in the dtype of ``cu``.
    """
    cu = np.asarray(cu)
    dt = cu.dtype
    a = np.abs(cu)
    order = np.argsort(a, axis=-1, kind="stable")
    srt = np.take_along_axis(a, order, axis=-1)
    s, m, b = srt[..., 0], srt[..., 1], srt[..., 2]
    r2 = dt.type(math.sqrt(2.0))
    pi = dt.type(math.pi)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = s * pi / (dt.type(12.0) * m)
        t = np.where(np.isnan(t), dt.type(0.0), t)
        c = np.cos(t)
        fac = (
            dt.type(2.0 ** (1.0 / 12.0) * 3.0 ** (1.0 / 3.0))
            * m
            * np.sqrt(
                (dt.type(4.0) * b * b * (c - r2) + r2 * m * m * (dt.type(-2.0) * r2 * c + dt.type(3.0)))
                / (c - r2)
            )
            / (dt.type(math.pi ** (1.0 / 3.0)) * b * np.sqrt(r2 - c))
        )
        hx = fac * np.sin(t)
        hy = fac * dt.type(2.0 ** -0.5) * (r2 * c - dt.type(1.0))
        hz = (
            dt.type(2.0 * 6.0 ** (1.0 / 3.0)) * b * b * (c - r2)
            + dt.type(2.0 ** (5.0 / 6.0) * 3.0 ** (1.0 / 3.0)) * m * m * (dt.type(-2.0) * r2 * c + dt.type(3.0))
        ) / (dt.type(2.0 * math.pi ** (1.0 / 3.0)) * b * (c - r2))
    hs = np.stack((hx, hy, hz), axis=-1)
    ho = np.empty_like(hs)
    np.put_along_axis(ho, order, hs, axis=-1)
    ho = np.where(np.isnan(ho), dt.type(0.0), ho)
    return np.copysign(ho, cu)


def _omega_from_ho_norm(t: np.ndarray) -> np.ndarray:
    """Rotation angle w from |h| by solving |h|^3 = 3/4 (w - sin w) (float64).

    The reference fits cos(w/2) with a polynomial (orientations.py:419-517);
    the oracle instead solves the defining equation with Newton's method to
    float64 accuracy. w - sin w and 1 - cos w use series / half-angle forms to
    avoid cancellation near 0.
    """
    t = np.asarray(t, dtype=np.float64)
    g = (4.0 / 3.0) * t**3  # = w - sin w
    w = np.cbrt(6.0 * g)  # small-angle start
    w = np.minimum(w, math.pi)
    for _ in range(40):
        small = w < 0.25
        w2 = w * w
        wms_series = w * w2 / 6.0 * (1 - w2 / 20.0 * (1 - w2 / 42.0 * (1 - w2 / 72.0 * (1 - w2 / 110.0))))
        wms = np.where(small, wms_series, w - np.sin(w))
        omc = 2.0 * np.sin(0.5 * w) ** 2
        with np.errstate(divide="ignore", invalid="ignore"):
            step = np.where(omc > 0, (wms - g) / omc, 0.0)
        w_new = np.clip(w - step, 0.0, math.pi)
        if np.all(np.abs(w_new - w) <= 1e-16 * np.maximum(1.0, w)):
            w = w_new
            break
        w = w_new
    return w


# Reference fp32 polynomial for cos(w/2) in |h|^2 (orientations.py:440-456).
_HO2AX_FP32_POLY = np.array(
    [
        1.0000000000000009e00,
        -4.9999943403867775e-01,
        -2.5015165060149020e-02,
        -3.8120131548551729e-03,
        -1.2106188330642162e-03,
        4.9329295993155416e-04,
        -7.0089385526450620e-04,
        3.0979774923589078e-04,
        -7.3023474963298843e-05,
    ]
)


def ho2qu(ho: np.ndarray, mode: str = "exact") -> np.ndarray:
    """Homochoric -> unit quaternion (w, x, y, z) (ho2ax orientations.py:419-517
    followed by ax2qu orientations.py:730-746).

    ``mode="exact"`` (float64): w solved from |h| (see _omega_from_ho_norm).
    ``mode="fp32poly"``: the reference's float32 polynomial for cos(w/2),
    evaluated in float32 exactly as the reference sums it.
    Rotations with |h|^2 < 1e-6 become the identity, as in the reference
    (orientations.py:511-515).
    """
    if mode == "exact":
        ho = np.asarray(ho, dtype=np.float64)
        n2 = np.sum(ho * ho, axis=-1)
        t = np.sqrt(n2)
        w = _omega_from_ho_norm(t)
        cw, sw = np.cos(0.5 * w), np.sin(0.5 * w)
        with np.errstate(divide="ignore", invalid="ignore"):
            axis = ho / t[..., None]
    elif mode == "fp32poly":
        ho = np.asarray(ho, dtype=np.float32)
        n2 = np.sum(ho * ho, axis=-1, dtype=np.float32)
        s = np.zeros_like(n2)
        for i, c in enumerate(_HO2AX_FP32_POLY.astype(np.float32)):
            s = s + c * n2 ** np.float32(i)
        w = np.float32(2.0) * np.arccos(np.clip(s, -1.0, 1.0))
        cw = np.cos(w / np.float32(2.0))
        sw = np.sin(w / np.float32(2.0))
        with np.errstate(divide="ignore", invalid="ignore"):
            axis = ho * (np.float32(1.0) / np.sqrt(n2))[..., None]
    else:
        raise ValueError(mode)
    qu = np.concatenate((cw[..., None], axis * sw[..., None]), axis=-1)
    ident = np.abs(n2) < 1e-6
    qu[ident] = np.array([1.0, 0.0, 0.0, 0.0], dtype=qu.dtype)
    return qu


def qu_std(qu: np.ndarray) -> np.ndarray:
    """Make the real part non-negative (quaternions.py:27-38)."""
    return np.where(qu[..., 0:1] >= 0, qu, -qu)


def cu2qu(cu: np.ndarray, mode: str = "exact") -> np.ndarray:
    """Cubochoric -> quaternion (orientations.py:1136-1147)."""
    return ho2qu(cu2ho(cu), mode=mode)


def qu2ho(qu: np.ndarray) -> np.ndarray:
    """Quaternion -> homochoric vector h = axis * (3/4 (w - sin w))^(1/3)
    (orientations.py:28-48), float64, series form near w = 0."""
    qu = np.asarray(qu, dtype=np.float64)
    w = 2.0 * np.arccos(np.clip(qu[..., 0], -1.0, 1.0))
    n = np.linalg.norm(qu[..., 1:], axis=-1, keepdims=True)
    with np.errstate(divide="ignore", invalid="ignore"):
        axis = np.where(n > 0, qu[..., 1:] / n, 0.0)
    w2 = w * w
    wms = np.where(w < 0.25, w * w2 / 6.0 * (1 - w2 / 20.0 * (1 - w2 / 42.0 * (1 - w2 / 72.0))), w - np.sin(w))
    return axis * np.cbrt(0.75 * wms)[..., None]


def ho2cu(ho: np.ndarray) -> np.ndarray:
    """Homochoric -> cubochoric, the inverse of cu2ho (orientations.py:352-416,
    Rosca et al. 2014): magnitudes ordered ascending, inverse square-to-sphere
    and squircle steps, signs copied back."""
    ho = np.asarray(ho, dtype=np.float64)
    a = np.abs(ho)
    order = np.argsort(a, axis=-1, kind="stable")
    srt = np.take_along_axis(a, order, axis=-1)
    x3, y3, z3 = srt[..., 0], srt[..., 1], srt[..., 2]
    r = np.linalg.norm(ho, axis=-1)
    with np.errstate(divide="ignore", invalid="ignore"):
        pf = np.sqrt(2 * r / (r + z3))
        x2, y2 = x3 * pf, y3 * pf
        z2 = math.sqrt(math.pi / 6) * r
        q = np.sqrt(x2 * x2 + 2 * y2 * y2)
        pf2 = math.sqrt(math.pi / 6) * np.sqrt(x2 * x2 + y2 * (q + 2 * y2)) / math.sqrt(2.0)
        x1 = pf2 * 12.0 / math.pi * np.arccos(np.clip((x2 * x2 + y2 * q) / (math.sqrt(2.0) * (x2 * x2 + y2 * y2)),
                                                        -1.0, 1.0))
        y1 = pf2
    cs = np.stack((x1, y1, z2), axis=-1) / (math.pi / 6) ** (1.0 / 6.0)
    cs = np.where(np.isnan(cs), 0.0, cs)
    cu = np.empty_like(cs)
    np.put_along_axis(cu, order, cs, axis=-1)
    return np.copysign(cu, ho)


def qu2cu(qu: np.ndarray) -> np.ndarray:
    """Quaternion -> cubochoric (orientations.py:1024-1035)."""
    return ho2cu(qu2ho(qu))


def grid_edge_length(laue_id: int, angular_resolution_deg: float) -> int:
    """Cubochoric edge length for a target resolution (laue_fz_ori.py:540-547).

    The empirical fit and the int truncation are the reference's; they set how
    many grid points exist, so they are kept identical.
    """
    n_so3 = (2 * 131.97049 / (angular_resolution_deg - 0.03732) + 1) ** 3
    return int((n_so3 / (0.5 * laue_mult(laue_id))) ** (1.0 / 3.0) + 1.0)


def cubochoric_axis(edge_length: int, dtype=np.float64) -> np.ndarray:
    """Per-axis grid coordinates (sampling.py:193-200): edge+1 points spanning
    [-a/2, a/2], the last dropped. Coordinate i is a/2 * (2i - edge) / edge:
    exactly 0 at the centre and antisymmetric, like the reference's
    symmetric linspace (the FZ test of 180-degree rotations needs the exact 0)."""
    i = np.arange(edge_length, dtype=np.float64)
    return (CU_HALF_EDGE * (2.0 * i - edge_length) / edge_length).astype(dtype)


def so3_cubochoric_grid(edge_length: int, mode: str = "exact") -> np.ndarray:
    """All edge^3 grid quaternions in 'ij' meshgrid order (sampling.py:179-205)."""
    ax = cubochoric_axis(edge_length, np.float64 if mode == "exact" else np.float32)
    cu = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), axis=-1).reshape(-1, 3)
    return qu_std(cu2qu(cu, mode=mode))


def ori_in_fz_laue(qu: np.ndarray, laue_id: int) -> np.ndarray:
    """Orientation fundamental-zone membership, inclusive bounds
    (laue_fz_ori.py:144-239). ``qu`` must have w >= 0."""
    w = qu[..., 0]
    x, y, z = np.abs(qu[..., 1]), np.abs(qu[..., 2]), np.abs(qu[..., 3])
    r2m1 = math.sqrt(2.0) - 1.0
    r3 = math.sqrt(3.0)
    if laue_id == 11:
        return (np.maximum(np.maximum(x, y), z) <= w * r2m1) & (x + y + z <= w)
    if laue_id == 10:
        return x + y + z <= w
    if laue_id == 9:
        m, n = np.maximum(x, y), np.minimum(x, y)
        rot = np.where(m > (2 + r3) * n, m, (r3 / 2) * m + 0.5 * n)
        return (z <= (2 - r3) * w) & (rot <= w)
    if laue_id == 8:
        return z <= (2 - r3) * w
    if laue_id == 7:
        rot = np.where(x >= y * r3, x, (r3 / 2) * y + 0.5 * x)
        return (z <= (1.0 / r3) * w) & (rot <= w)
    if laue_id == 6:
        return z <= (1.0 / r3) * w
    if laue_id == 5:
        m, n = np.maximum(x, y), np.minimum(x, y)
        rot = np.where(m > (math.sqrt(2.0) + 1) * n, m, (1 / math.sqrt(2.0)) * (m + n))
        return (z <= r2m1 * w) & (rot <= w)
    if laue_id == 4:
        return z <= r2m1 * w
    if laue_id == 3:
        return np.maximum(np.maximum(x, y), z) <= w
    if laue_id == 2:
        return z <= w
    if laue_id == 1:
        return np.ones(qu.shape[:-1], dtype=bool)
    raise ValueError(f"Laue group {laue_id} is not supported")


def sample_ori_fz_laue_angle(
    laue_id: int,
    angular_resolution_deg: float,
    permutation: Optional[np.ndarray] = None,
    mode: str = "exact",
) -> np.ndarray:
    """FZ dictionary (laue_fz_ori.py:516-557): grid, FZ filter, optional
    permutation (the reference draws it with torch.randperm on the global CPU
    generator; the caller passes that permutation in)."""
    edge = grid_edge_length(laue_id, angular_resolution_deg)
    q = so3_cubochoric_grid(edge, mode=mode)
    q = q[ori_in_fz_laue(q, laue_id)]
    if permutation is not None:
        q = q[permutation]
    return q


# --------------------------------------------------------------------------
# Detector geometry (A3)
# --------------------------------------------------------------------------


def bruker_geometry_to_SE3(pc, primary_tilt_deg: float, secondary_tilt_deg: float, detector_shape):
    """Bruker pattern centre -> detector-to-sample rotation and translation
    (geometry.py:31-92)."""
    pcx, pcy, pcz = (float(v) for v in pc)
    rows, cols = float(detector_shape[0]), float(detector_shape[1])
    d = math.radians(primary_tilt_deg)
    sx = math.radians(secondary_tilt_deg)
    sd, cd, ss, cs = math.sin(d), math.cos(d), math.sin(sx), math.cos(sx)
    rot = np.array(
        [
            [-sd, -ss * cd, cs * cd],
            [0.0, cs, ss],
            [-cd, ss * sd, -sd * cs],
        ]
    )
    tx = pcx * cols * ss * cd + pcy * rows * sd + pcz * rows * cs * cd - ss * cd / 2 - sd / 2
    ty = -cols * pcx * cs + pcz * rows * ss + cs / 2
    tz = -cols * pcx * ss * sd + pcy * rows * cd - pcz * rows * sd * cs + ss * sd / 2 - cd / 2
    return rot, np.array([tx, ty, tz])


def detector_coords_sample_frame(
    detector_shape: Tuple[int, int],
    proj_center=(0.5, 0.5, 0.5),
    tilts_degrees=(0.0, 70.0, 0.0),
    binning=(1, 1),
) -> np.ndarray:
    """Un-normalised sample-frame coordinates of each (binned) detector pixel,
    (P, 3) float64, row-major over (i, j) (geometry.py:422-503 with
    project2sample :282-347; the SE(3) correction is the identity)."""
    h, w = detector_shape
    if h % binning[0] or w % binning[1]:
        raise ValueError("binning must evenly divide the detector shape")
    bh, bw = h // binning[0], w // binning[1]
    ii = np.linspace(0.5 * (binning[0] - 1), h - 0.5 * (binning[0] - 1), bh)
    jj = np.linspace(0.5 * (binning[1] - 1), w - 0.5 * (binning[1] - 1), bw)
    pix = np.stack(np.meshgrid(ii, jj, indexing="ij"), axis=-1).reshape(-1, 2)
    rot, t = bruker_geometry_to_SE3(
        proj_center, tilts_degrees[2] - tilts_degrees[1], tilts_degrees[0], detector_shape
    )
    p3 = np.concatenate((pix, np.zeros((pix.shape[0], 1))), axis=-1)
    return p3 @ rot.T + t


def unit_rays(coords: np.ndarray) -> np.ndarray:
    """Normalise rays (indexing.py:106)."""
    return coords / np.linalg.norm(coords, axis=-1, keepdims=True)


# --------------------------------------------------------------------------
# Projector (A4-A7)
# --------------------------------------------------------------------------


def qu_apply(qu: np.ndarray, v: np.ndarray) -> np.ndarray:
    """Rotate vectors by unit quaternions, q (0, v) q* (quaternions.py:186-213).
    Broadcasts (..., 4) against (..., 3)."""
    w, x, y, z = (qu[..., i] for i in range(4))
    vx, vy, vz = v[..., 0], v[..., 1], v[..., 2]
    # t = 2 (q_vec x v); v' = v + w t + q_vec x t  (same rotation, fewer terms)
    tx = 2.0 * (y * vz - z * vy)
    ty = 2.0 * (z * vx - x * vz)
    tz = 2.0 * (x * vy - y * vx)
    return np.stack(
        (
            vx + w * tx + (y * tz - z * ty),
            vy + w * ty + (z * tx - x * tz),
            vz + w * tz + (x * ty - y * tx),
        ),
        axis=-1,
    )


def rosca_lambert_side_by_side(p: np.ndarray) -> np.ndarray:
    """Unit sphere -> side-by-side square Lambert coordinates in [-1, 1]^2
    (sphere.py:145-185). x in [-1, 0] for z >= 0 (north), [0, 1] for z < 0;
    y in [-1, 1]. Same branch structure and sign conventions as the reference."""
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    dt = p.dtype.type
    fac = np.sqrt(np.maximum(dt(2.0) * (dt(1.0) - np.abs(z)), dt(0.0)))
    cond = np.abs(y) <= np.abs(x)
    big = np.where(cond, x, y)
    sml = np.where(cond, y, x)
    sgn = np.where(big < 0, dt(-1.0), dt(1.0))
    simple = sgn * fac * dt(2.0 / 8.0**0.5)
    arct = sgn * fac * np.arctan2(sml * sgn, np.abs(big)) * dt(2.0 * 2.0**0.5 / math.pi)
    u = np.where(cond, simple, arct)
    v = np.where(cond, arct, simple)
    u = u / dt(2.0) - dt(0.5) + np.where(z < 0, dt(1.0), dt(0.0))
    return np.stack((u, v), axis=-1)


def grid_sample_border(img: np.ndarray, uv: np.ndarray, align_corners: bool = False) -> np.ndarray:
    """Bilinear sampling of a (H, W) image at normalised (x, y) in [-1, 1],
    padding_mode='border' -- the semantics of torch.nn.functional.grid_sample
    used by master_pattern.py:197-206. Pixel coordinate ((c + 1) * size - 1) / 2
    (align_corners=False, dictionary indexing) or (c + 1) / 2 * (size - 1)
    (align_corners=True, refining.py:206), clamped to [0, size - 1]."""
    H, W = img.shape
    dt = uv.dtype.type
    if align_corners:
        fx = (uv[..., 0] + dt(1.0)) / dt(2.0) * dt(W - 1)
        fy = (uv[..., 1] + dt(1.0)) / dt(2.0) * dt(H - 1)
    else:
        fx = ((uv[..., 0] + dt(1.0)) * dt(W) - dt(1.0)) / dt(2.0)
        fy = ((uv[..., 1] + dt(1.0)) * dt(H) - dt(1.0)) / dt(2.0)
    fx = np.clip(fx, 0, W - 1)
    fy = np.clip(fy, 0, H - 1)
    x0 = np.floor(fx).astype(np.int64)
    y0 = np.floor(fy).astype(np.int64)
    tx = (fx - x0).astype(uv.dtype)
    ty = (fy - y0).astype(uv.dtype)
    x1 = np.minimum(x0 + 1, W - 1)
    y1 = np.minimum(y0 + 1, H - 1)
    im = img.astype(uv.dtype, copy=False)
    v00 = im[y0, x0]
    v01 = im[y0, x1]
    v10 = im[y1, x0]
    v11 = im[y1, x1]
    return (v00 * (1 - tx) + v01 * tx) * (1 - ty) + (v10 * (1 - tx) + v11 * tx) * ty


def avg_pool(img: np.ndarray, b: int) -> np.ndarray:
    """b x b average pooling with stride b over the last two axes
    (torch avg_pool2d, master_pattern.py:94-113, experiment_pats.py:338-341)."""
    if b == 1:
        return img
    *lead, H, W = img.shape
    Hb, Wb = H // b, W // b
    v = img[..., : Hb * b, : Wb * b].reshape(*lead, Hb, b, Wb, b)
    return v.mean(axis=(-3, -1))


def project_patterns(master_pattern: np.ndarray, rays: np.ndarray, quats: np.ndarray) -> np.ndarray:
    """Simulated patterns (n, P): rotate unit rays by each orientation, map to
    the side-by-side Lambert square and bilinearly sample the (H, 2W) master
    pattern (indexing.py:117-130, master_pattern.py:141-209)."""
    rot = qu_apply(quats[:, None, :], rays[None, :, :])
    uv = rosca_lambert_side_by_side(rot)
    return grid_sample_border(master_pattern, uv)


def zero_mean_rows(x: np.ndarray) -> np.ndarray:
    """Row mean subtraction (indexing.py:139-143)."""
    return x - x.mean(axis=-1, keepdims=True)


# --------------------------------------------------------------------------
# Matcher (A9, A10)
# --------------------------------------------------------------------------


def topk_dot(queries: np.ndarray, data: np.ndarray, k: int, chunk: int = 4096):
    """Top-k by raw dot product, sorted descending (knn.py:80-103 angular,
    ChunkedKNN merge and retrieve_topk :219-287). Ties resolve to the lower
    dictionary index. Returns (indices int64 (Q, k), values (Q, k))."""
    Q = queries.shape[0]
    best_v = np.full((Q, k), -np.inf, dtype=np.result_type(queries, data))
    best_i = np.zeros((Q, k), dtype=np.int64)
    for d0 in range(0, data.shape[0], chunk):
        blk = data[d0 : d0 + chunk]
        sim = queries @ blk.T
        kk = min(k, blk.shape[0])
        part = np.argpartition(-sim, kk - 1, axis=1)[:, :kk]
        pv = np.take_along_axis(sim, part, axis=1)
        allv = np.concatenate((best_v, pv), axis=1)
        alli = np.concatenate((best_i, part + d0), axis=1)
        # order by (-value, index) so equal values keep the lower index
        o = np.lexsort((alli, -allv), axis=1)[:, :k]
        best_v = np.take_along_axis(allv, o, axis=1)
        best_i = np.take_along_axis(alli, o, axis=1)
    return best_i, best_v


def topk_euclidean(queries: np.ndarray, data: np.ndarray, k: int, chunk: int = 4096):
    """Top-k by the smallest squared euclidean distance |q|^2 + |d|^2 - 2 q.d,
    sorted ascending (knn.py:85-91 with largest=False, ChunkedKNN merge and
    retrieve_topk :219-287). Ties resolve to the lower dictionary index.
    Returns (indices int64 (Q, k), distances (Q, k))."""
    Q = queries.shape[0]
    qn = (queries.astype(np.float64) ** 2).sum(axis=1).astype(queries.dtype)
    best_v = np.full((Q, k), np.inf, dtype=np.result_type(queries, data))
    best_i = np.zeros((Q, k), dtype=np.int64)
    for d0 in range(0, data.shape[0], chunk):
        blk = data[d0 : d0 + chunk]
        dn = (blk.astype(np.float64) ** 2).sum(axis=1).astype(blk.dtype)
        dist = qn[:, None] + dn[None, :] - 2.0 * (queries @ blk.T)
        kk = min(k, blk.shape[0])
        part = np.argpartition(dist, kk - 1, axis=1)[:, :kk]
        pv = np.take_along_axis(dist, part, axis=1)
        allv = np.concatenate((best_v, pv), axis=1)
        alli = np.concatenate((best_i, part + d0), axis=1)
        o = np.lexsort((alli, allv), axis=1)[:, :k]
        best_v = np.take_along_axis(allv, o, axis=1)
        best_i = np.take_along_axis(alli, o, axis=1)
    return best_i, best_v


def topk_manhattan(queries: np.ndarray, data: np.ndarray, k: int, chunk: int = 256):
    """Top-k by the smallest L1 distance sum |q - d| (knn.py:92-93 with
    largest=False), sorted ascending; ties resolve to the lower index.
    Returns (indices int64 (Q, k), distances (Q, k))."""
    Q = queries.shape[0]
    best_v = np.full((Q, k), np.inf, dtype=np.result_type(queries, data))
    best_i = np.zeros((Q, k), dtype=np.int64)
    for d0 in range(0, data.shape[0], chunk):
        blk = data[d0 : d0 + chunk]
        dist = np.abs(queries[:, None, :] - blk[None, :, :]).sum(axis=2)
        kk = min(k, blk.shape[0])
        part = np.argpartition(dist, kk - 1, axis=1)[:, :kk]
        pv = np.take_along_axis(dist, part, axis=1)
        allv = np.concatenate((best_v, pv), axis=1)
        alli = np.concatenate((best_i, part + d0), axis=1)
        o = np.lexsort((alli, allv), axis=1)[:, :k]
        best_v = np.take_along_axis(allv, o, axis=1)
        best_i = np.take_along_axis(alli, o, axis=1)
    return best_i, best_v


# --------------------------------------------------------------------------
# End-to-end plain DI (A1-A13)
# --------------------------------------------------------------------------


def prep_patterns(patterns: np.ndarray, binning: int = 1, mask: Optional[np.ndarray] = None,
                  subtract_mean: bool = True, dtype=np.float64) -> np.ndarray:
    """Query preparation (indexing.py:175-187, experiment_pats.py:318-346):
    bin, flatten, mask, zero-mean."""
    x = avg_pool(np.asarray(patterns, dtype=dtype), binning)
    x = x.reshape(x.shape[0], -1)
    if mask is not None:
        x = x[:, mask.reshape(-1)]
    if subtract_mean:
        x = zero_mean_rows(x)
    return x


def dictionary_rows(master_pattern, rays_unit, quats, mask=None, dtype=np.float64, chunk=2048):
    """Zero-mean simulated dictionary rows (n, P') in ``dtype``."""
    mp = np.asarray(master_pattern, dtype=dtype)
    r = rays_unit.astype(dtype)
    if mask is not None:
        r = r[mask.reshape(-1)]
    out = np.empty((quats.shape[0], r.shape[0]), dtype=dtype)
    for i in range(0, quats.shape[0], chunk):
        out[i : i + chunk] = zero_mean_rows(project_patterns(mp, r, quats[i : i + chunk].astype(dtype)))
    return out


def dictionary_index(
    master_pattern: np.ndarray,
    laue_id: int,
    patterns: np.ndarray,
    detector_shape,
    proj_center=(0.5, 0.5, 0.5),
    tilts_degrees=(0.0, 70.0, 0.0),
    resolution_deg: float = 10.0,
    permutation: Optional[np.ndarray] = None,
    top_k: int = 1,
    mask: Optional[np.ndarray] = None,
    binning: int = 1,
    dtype=np.float64,
    dictionary: Optional[np.ndarray] = None,
    distance_metric: str = "angular",
):
    """Plain DI for one phase (indexing.py:14-211). Returns
    (orientations (Q, k, 4), metrics (Q, k), indices (Q, k), dictionary (D, 4));
    distance_metric "angular" (largest raw dot first), "euclidean"
    (smallest squared distance first, knn.py:85-91) or "manhattan" (smallest
    L1 distance first, knn.py:92-93)."""
    if dictionary is None:
        dictionary = sample_ori_fz_laue_angle(laue_id, resolution_deg, permutation)
    mp = avg_pool(np.asarray(master_pattern, dtype=np.float64), binning)
    coords = detector_coords_sample_frame(detector_shape, proj_center, tilts_degrees, (binning, binning))
    rays = unit_rays(coords)
    d = dictionary_rows(mp, rays, dictionary, mask, dtype)
    q = prep_patterns(patterns, binning, mask, True, dtype)
    if distance_metric == "euclidean":
        idx, val = topk_euclidean(q, d, top_k)
    elif distance_metric == "manhattan":
        idx, val = topk_manhattan(q, d, top_k)
    elif distance_metric == "angular":
        idx, val = topk_dot(q, d, top_k)
    else:
        raise NotImplementedError(f"'{distance_metric}' not supported.")
    return dictionary[idx], val, idx, dictionary


# --------------------------------------------------------------------------
# PCA (A11, A12)
# --------------------------------------------------------------------------


def covariance_chan(rows_iter, n_features: int) -> np.ndarray:
    """Streaming covariance with Chan/Welford batch updates, float64
    (pca_covmat.py:53-91 update, :139-147 normalisation by obs - 1)."""
    mean = np.zeros((1, n_features))
    agg = np.zeros((n_features, n_features))
    obs = 0
    for x in rows_iter:
        x = np.asarray(x, dtype=np.float64)
        n = x.shape[0]
        bmean = x.mean(axis=0, keepdims=True)
        new_mean = (mean * obs + bmean * n) / (obs + n)
        agg += (x - mean).T @ (x - new_mean)
        obs += n
        mean = new_mean
    return agg / (obs - 1)


def pca_components(cov: np.ndarray, n_components: int, slice_mode: str = "top") -> np.ndarray:
    """Eigenvectors (ascending eigenvalue, pca_covmat.py:149-158) and the
    component slice. ``slice_mode="reference"`` reproduces indexing.py:355
    exactly (``[:, -n : -n + 300]``); ``"top"`` keeps the n leading vectors."""
    _, vecs = np.linalg.eigh(cov)
    if slice_mode == "reference":
        return vecs[:, -n_components : (-n_components + 300)]
    return vecs[:, -n_components:]


def pca_dictionary_index(
    master_pattern: np.ndarray,
    patterns: np.ndarray,
    detector_shape,
    proj_center,
    learn_dictionary: np.ndarray,
    index_dictionary: np.ndarray,
    n_components: int,
    slice_mode: str = "top",
    top_k: int = 1,
    tilts_degrees=(0.0, 70.0, 0.0),
    chunk: int = 4096,
):
    """PCA DI for one phase, float64 (indexing.py:214-476): Chan covariance of
    the zero-mean learn patterns, eigenvectors, slice, projection of the
    zero-mean dictionary and query rows, top-k by the projected dot.
    Returns (orientations (Q, k, 4), metrics (Q, k), indices (Q, k))."""
    rays = unit_rays(detector_coords_sample_frame(detector_shape, proj_center, tilts_degrees))
    learn = dictionary_rows(master_pattern, rays, learn_dictionary)
    cov = covariance_chan((learn[i:i + chunk] for i in range(0, learn.shape[0], chunk)), learn.shape[1])
    V = pca_components(cov, n_components, slice_mode)
    d = dictionary_rows(master_pattern, rays, index_dictionary) @ V
    q = prep_patterns(patterns) @ V
    idx, val = topk_dot(q, d, top_k)
    return index_dictionary[idx], val, idx


# --------------------------------------------------------------------------
# Disorientation (A14)
# --------------------------------------------------------------------------


def disori_angle(q1: np.ndarray, q2: np.ndarray, laue_id: int) -> np.ndarray:
    """Disorientation angle (rad) under one Laue group
    (laue_fz_misori.py:148-203): max |w| over g2 (q1 q2*) g1."""
    g = laue_elements(laue_id)
    q2c = q2 * np.array([1.0, -1.0, -1.0, -1.0])
    mis = _qmul(q1, q2c)
    best = np.zeros(mis.shape[:-1])
    for a in g:
        left = _qmul(np.broadcast_to(a, mis.shape), mis)
        for b in g:
            w = np.abs(_qmul(left, np.broadcast_to(b, mis.shape))[..., 0])
            best = np.maximum(best, w)
    return 2.0 * np.arccos(np.clip(best, -1.0, 1.0))


# --------------------------------------------------------------------------
# 6-D rotation representation (A15)
# --------------------------------------------------------------------------


def zh2om(zh: np.ndarray) -> np.ndarray:
    """6-D (Zhou et al. 2019) -> rotation matrix with Gram-Schmidt rows
    b1, b2, b3 (orientations.py:940-963)."""
    a1, a2 = zh[..., :3], zh[..., 3:]
    b1 = a1 / np.linalg.norm(a1, axis=-1, keepdims=True)
    b2 = a2 - np.sum(b1 * a2, axis=-1, keepdims=True) * b1
    b2 = b2 / np.linalg.norm(b2, axis=-1, keepdims=True)
    b3 = np.cross(b1, b2)
    b3 = b3 / np.linalg.norm(b3, axis=-1, keepdims=True)
    return np.stack((b1, b2, b3), axis=-2)


def qu2om(qu: np.ndarray) -> np.ndarray:
    """Quaternion (w, x, y, z) -> rotation matrix (orientations.py:913-937)."""
    w, x, y, z = (qu[..., i] for i in range(4))
    qb = w * w - (x * x + y * y + z * z)
    m = np.empty(qu.shape[:-1] + (3, 3))
    m[..., 0, 0] = qb + 2 * x * x
    m[..., 0, 1] = 2 * (x * y - w * z)
    m[..., 0, 2] = 2 * (x * z + w * y)
    m[..., 1, 0] = 2 * (y * x + w * z)
    m[..., 1, 1] = qb + 2 * y * y
    m[..., 1, 2] = 2 * (y * z - w * x)
    m[..., 2, 0] = 2 * (z * x - w * y)
    m[..., 2, 1] = 2 * (z * y + w * x)
    m[..., 2, 2] = qb + 2 * z * z
    return m


def om2qu(m: np.ndarray) -> np.ndarray:
    """Rotation matrix -> quaternion with w >= 0 (orientations.py:52-132):
    the largest-diagonal branch of Farrell's method, then the axis signs from
    the antisymmetric part."""
    m00, m11, m22 = m[..., 0, 0], m[..., 1, 1], m[..., 2, 2]
    m01, m02, m10, m12, m20, m21 = m[..., 0, 1], m[..., 0, 2], m[..., 1, 0], m[..., 1, 2], m[..., 2, 0], m[..., 2, 1]
    q = np.empty(m.shape[:-2] + (4,))
    b1 = (m22 < 0) & (m00 > m11)
    b2 = (m22 < 0) & ~(m00 > m11)
    b3 = ~(m22 < 0) & (m00 < -m11)
    b4 = ~(m22 < 0) & ~(m00 < -m11)
    for br, t, comp in (
        (b1, 1 + m00 - m11 - m22, (m12 - m21, None, m01 + m10, m20 + m02)),
        (b2, 1 - m00 + m11 - m22, (m20 - m02, m01 + m10, None, m12 + m21)),
        (b3, 1 - m00 - m11 + m22, (m01 - m10, m20 + m02, m12 + m21, None)),
        (b4, 1 + m00 + m11 + m22, (None, m12 - m21, m20 - m02, m01 - m10)),
    ):
        r = 0.5 / np.sqrt(np.where(br, t, 1.0))
        for i, c in enumerate(comp):
            val = t * r if c is None else c * r
            q[..., i] = np.where(br, val, q[..., i])
    q[..., 0] = np.abs(q[..., 0])
    q[..., 1] = np.copysign(q[..., 1], m21 - m12)
    q[..., 2] = np.copysign(q[..., 2], m02 - m20)
    q[..., 3] = np.copysign(q[..., 3], m10 - m01)
    return q


def zh2qu(zh: np.ndarray) -> np.ndarray:
    return om2qu(zh2om(zh))


def qu2zh(qu: np.ndarray) -> np.ndarray:
    """First two rows of the rotation matrix (orientations.py:1008-1020)."""
    return qu2om(qu)[..., :2, :].reshape(qu.shape[:-1] + (6,))


def rot6d_sym_loss(zh: np.ndarray, q_true: np.ndarray, laue_id: int):
    """Per-sample loss min over Laue operators g of ||zh2om(zh) - om(g q_true)||_F^2
    and its gradient with respect to zh (Gram-Schmidt backward), float64.
    The CNN head's training objective (a new part: the reference has no
    learned indexer)."""
    g = laue_elements(laue_id)
    R = zh2om(zh)
    best = np.full(zh.shape[0], np.inf)
    target = np.zeros_like(R)
    for op in g:
        Rt = qu2om(_qmul(np.broadcast_to(op, q_true.shape), q_true))
        d = np.sum((R - Rt) ** 2, axis=(-2, -1))
        sel = d < best
        best = np.where(sel, d, best)
        target[sel] = Rt[sel]
    gR = 2.0 * (R - target)
    a1, a2 = zh[:, :3], zh[:, 3:]
    n1 = np.linalg.norm(a1, axis=1, keepdims=True)
    b1 = a1 / n1
    u = a2 - np.sum(b1 * a2, axis=1, keepdims=True) * b1
    n2 = np.linalg.norm(u, axis=1, keepdims=True)
    b2 = u / n2
    c = np.cross(b1, b2)
    nc = np.linalg.norm(c, axis=1, keepdims=True)
    b3 = c / nc
    gb1, gb2, gb3 = gR[:, 0], gR[:, 1], gR[:, 2]
    gc = (gb3 - np.sum(gb3 * b3, axis=1, keepdims=True) * b3) / nc
    gb1 = gb1 + np.cross(b2, gc)
    gb2 = gb2 + np.cross(gc, b1)
    gu = (gb2 - np.sum(gb2 * b2, axis=1, keepdims=True) * b2) / n2
    gub1 = np.sum(gu * b1, axis=1, keepdims=True)
    ga2 = gu - gub1 * b1
    gb1 = gb1 - gub1 * a2 - np.sum(b1 * a2, axis=1, keepdims=True) * gu
    ga1 = (gb1 - np.sum(gb1 * b1, axis=1, keepdims=True) * b1) / n1
    return best, np.concatenate((ga1, ga2), axis=1)


# --------------------------------------------------------------------------
# Orientation-proposal CNN (checker for the GPU forward / backward kernels)
# --------------------------------------------------------------------------


def _im2col(x: np.ndarray) -> np.ndarray:
    """(B, H, W, C) -> (B*Ho*Wo, 9*C) for 3x3 / stride 2 / pad 1, columns
    ordered (ky, kx, c)."""
    B, H, W, C = x.shape
    Ho, Wo = (H + 1) // 2, (W + 1) // 2
    xp = np.zeros((B, H + 2, W + 2, C), dtype=x.dtype)
    xp[:, 1:H + 1, 1:W + 1] = x
    cols = np.empty((B, Ho, Wo, 3, 3, C), dtype=x.dtype)
    for ky in range(3):
        for kx in range(3):
            cols[:, :, :, ky, kx] = xp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Wo:2]
    return cols.reshape(B * Ho * Wo, 9 * C)


def _col2im(dcols: np.ndarray, shape) -> np.ndarray:
    B, H, W, C = shape
    Ho, Wo = (H + 1) // 2, (W + 1) // 2
    d = dcols.reshape(B, Ho, Wo, 3, 3, C)
    dxp = np.zeros((B, H + 2, W + 2, C))
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Wo:2] += d[:, :, :, ky, kx]
    return dxp[:, 1:H + 1, 1:W + 1]


def cnn_forward_backward(params: dict, x: np.ndarray, q_true: np.ndarray, laue_id: int, grad_out=None):
    """FP64 forward + backward of the proposal CNN (ebsdtorch_b200/learned.py
    layout: conv{i}.w (Cout, 9*Cin) over (ky, kx, cin), conv{i}.b, fc1, fc2).
    grad_out, if given, replaces the loss gradient dL/dz (already divided by
    the batch size). Returns (outputs (B, 6), mean loss, gradients dict)."""
    B = x.shape[0]
    a = x.reshape(B, x.shape[1], x.shape[2], 1).astype(np.float64)
    cache = []
    i = 0
    while f"conv{i}.w" in params:
        w, b = params[f"conv{i}.w"], params[f"conv{i}.b"]
        cols = _im2col(a)
        y = cols @ w.T + b
        out = np.maximum(y, 0.0)
        Ho, Wo = (a.shape[1] + 1) // 2, (a.shape[2] + 1) // 2
        cache.append((a.shape, cols, out))
        a = out.reshape(B, Ho, Wo, w.shape[0])
        i += 1
    feat = a.reshape(B, -1)
    h_pre = feat @ params["fc1.w"].T + params["fc1.b"]
    h = np.maximum(h_pre, 0.0)
    z = h @ params["fc2.w"].T + params["fc2.b"]
    loss, gz = rot6d_sym_loss(z, q_true, laue_id)
    gz = gz / B if grad_out is None else grad_out
    grads = {"fc2.w": gz.T @ h, "fc2.b": gz.sum(0)}
    gh = (gz @ params["fc2.w"]) * (h > 0)
    grads["fc1.w"], grads["fc1.b"] = gh.T @ feat, gh.sum(0)
    g = (gh @ params["fc1.w"]).reshape(-1, params[f"conv{i - 1}.w"].shape[0])
    for j in range(i - 1, -1, -1):
        shape, cols, out = cache[j]
        g = g * (out > 0)
        grads[f"conv{j}.w"] = g.T @ cols
        grads[f"conv{j}.b"] = g.sum(0)
        if j > 0:
            dx = _col2im(g @ params[f"conv{j}.w"], shape)
            g = dx.reshape(-1, shape[3])
    return z, float(loss.mean()), grads


def local_search_bruteforce(q_rows: np.ndarray, proposals: np.ndarray, dictionary: np.ndarray,
                            d_rows: np.ndarray, laue_id: int, max_angle_rad: float):
    """Checker of ebsd_local_search: for each query, every dictionary
    orientation whose disorientation from the proposal is at most
    max_angle_rad, scored by the exact dot; best index (ties: lower index) and
    score, -1 / -inf when none."""
    Q = q_rows.shape[0]
    best_i = np.full(Q, -1, dtype=np.int64)
    best_v = np.full(Q, -np.inf)
    for i in range(Q):
        ang = disori_angle(np.broadcast_to(proposals[i], dictionary.shape), dictionary, laue_id)
        cand = np.nonzero(ang <= max_angle_rad)[0]
        if cand.size == 0:
            continue
        sc = d_rows[cand] @ q_rows[i]
        j = np.lexsort((cand, -sc))[0]
        best_i[i], best_v[i] = cand[j], sc[j]
    return best_i, best_v


# --------------------------------------------------------------------------
# Synthetic data (stands in for the reference's kikuchipy demo data)
# --------------------------------------------------------------------------


def inv_rosca_lambert_north(uv: np.ndarray) -> np.ndarray:
    """Square [-1, 1]^2 -> northern unit hemisphere (sphere.py:95-142)."""
    pi = math.pi
    xa = np.abs(uv[..., 0]) * math.sqrt(pi / 2)
    ya = np.abs(uv[..., 1]) * math.sqrt(pi / 2)
    cond = xa >= ya
    xn = np.where(cond, xa, ya)
    yn = np.where(cond, ya, xa)
    with np.errstate(divide="ignore", invalid="ignore"):
        ang = np.where(xn > 0, pi * yn / (4 * xn), 0.0)
    rr = (2 * xn / pi) * np.sqrt(np.maximum(pi - xn * xn, 0.0))
    xh, yh = rr * np.cos(ang), rr * np.sin(ang)
    zo = 1 - 2 * xn * xn / pi
    xo = np.copysign(np.where(cond, xh, yh), uv[..., 0])
    yo = np.copysign(np.where(cond, yh, xh), uv[..., 1])
    return np.stack((xo, yo, zo), axis=-1)


# --------------------------------------------------------------------------
# Orientation grid refinement (the first "next" step after DI)
# --------------------------------------------------------------------------


def local_orientation_grid(semi_edge_deg: float, radius: int, axial: int = 3) -> np.ndarray:
    """(G, 3) cubochoric offsets of the local grid (refining.py:13-68): a
    (2 radius + 1)^3 cube of semi-edge semi_edge_deg * pi^(2/3) / 360, all
    points (axial 3), points with a zero coordinate (2) or on the axes (1)."""
    s = semi_edge_deg * math.pi ** (2.0 / 3.0) / 360.0
    c = np.linspace(-s, s, 2 * radius + 1)
    cu = np.stack(np.meshgrid(c, c, c, indexing="ij"), axis=-1).reshape(-1, 3)
    if axial == 2:
        cu = cu[np.any(cu == 0, axis=-1)]
    elif axial == 1:
        cu = cu[np.sum(cu == 0, axis=-1) >= 2]
    elif axial != 3:
        raise ValueError("axial_grid_dimension must be 1, 2, or 3.")
    return cu


def ori_to_fz_laue_right(q: np.ndarray, laue_id: int) -> np.ndarray:
    """The reference's orientation FZ reduction (laue_fz_ori.py:36-81): the
    operator g maximising |(q g).w| is applied on the RIGHT, q g (qu_prod
    then w >= 0)."""
    g = laue_elements(laue_id)
    prods = _qmul(q[..., None, :], g)
    best = np.argmax(np.abs(prods[..., 0]), axis=-1)
    return qu_std(np.take_along_axis(prods, best[..., None, None], axis=-2)[..., 0, :])


def ori_to_fz_laue_left(q: np.ndarray, laue_id: int) -> np.ndarray:
    """FZ reduction by the left product g q (the operator maximising |w|),
    which keeps the simulated pattern: pattern(g q) == pattern(q)."""
    g = laue_elements(laue_id)
    prods = _qmul(g, q[..., None, :])
    best = np.argmax(np.abs(prods[..., 0]), axis=-1)
    return qu_std(np.take_along_axis(prods, best[..., None, None], axis=-2)[..., 0, :])


def orientation_grid_refinement(master_pattern: np.ndarray, coords: np.ndarray, exp_rows: np.ndarray,
                                q0: np.ndarray, laue_id: int, semi_edge_deg: float, n_iter: int = 3,
                                axial: int = 3, radius: int = 1, shrink: float = 0.5,
                                offsets: Optional[np.ndarray] = None, fz: str = "reference"):
    """Grid refinement of one phase (refining.py:71-244), float64.

    coords: (P, 3) detector coordinates in the sample frame (unit rays when
    offsets is None; with offsets (n, 2), per pattern normalize(coords +
    (offset, 0)), refining.py:117-128). exp_rows: (n, P) zero-mean patterns.
    Each iteration composes the grid with the current orientation
    (cu2qu(grid) q), reduces to the FZ (fz "reference": ori_to_fz_laue_right,
    "left": ori_to_fz_laue_left), simulates with align_corners=True sampling,
    subtracts each simulation's mean, takes the best dot product, moves there
    and halves (shrink) the pattern's grid when the centre stayed best.
    Returns (orientations (n, 4), best dots (n, n_iter))."""
    grid = local_orientation_grid(semi_edge_deg, radius, axial)
    n_grid = grid.shape[0]
    centre = (n_grid - 1) // 2
    n = q0.shape[0]
    scale = np.ones(n)
    q = np.asarray(q0, dtype=np.float64)
    dots = np.zeros((n, n_iter))
    reduce = ori_to_fz_laue_right if fz == "reference" else ori_to_fz_laue_left
    for j in range(n_iter):
        qg = cu2qu(grid[None] * scale[:, None, None])
        qa = reduce(qu_std(_qmul(qg, q[:, None, :])), laue_id)
        best_v = np.empty(n)
        best_i = np.empty(n, dtype=np.int64)
        for i in range(n):
            if offsets is None:
                rays = coords
            else:
                c = coords + np.concatenate((offsets[i], [0.0]))[None]
                rays = c / np.linalg.norm(c, axis=-1, keepdims=True)
            rot = qu_apply(qa[i][:, None, :], rays[None])
            sims = grid_sample_border(master_pattern, rosca_lambert_side_by_side(rot), align_corners=True)
            sims = sims - sims.mean(axis=-1, keepdims=True)
            d = sims @ exp_rows[i]
            best_i[i] = int(np.argmax(d))
            best_v[i] = d[best_i[i]]
        dots[:, j] = best_v
        q = qa[np.arange(n), best_i]
        scale = np.where(best_i == centre, scale * shrink, scale)
    return q, dots


# --------------------------------------------------------------------------
# Pattern preprocessing (experiment_pats.py:223-316, preprocessing/)
# --------------------------------------------------------------------------


def subtract_overall_background(pats: np.ndarray) -> np.ndarray:
    """Subtract the mean pattern of the scan (experiment_pats.py:223-232)."""
    return pats - pats.mean(axis=0, keepdims=True)


def normalize_per_pattern(pats: np.ndarray, norm_type: str = "minmax") -> np.ndarray:
    """Per-pattern normalisation (experiment_pats.py:255-285); 'standard'
    divides by the unbiased standard deviation, as torch.std does."""
    x = pats.reshape(pats.shape[0], -1)
    if norm_type == "minmax":
        mn, mx = x.min(axis=1, keepdims=True), x.max(axis=1, keepdims=True)
        x = (x - mn) / (1e-4 + mx - mn)
    elif norm_type == "zeromean":
        x = x - x.mean(axis=1, keepdims=True)
    elif norm_type == "standard":
        x = x - x.mean(axis=1, keepdims=True)
        x = x / x.std(axis=1, ddof=1, keepdims=True)
    else:
        raise ValueError(norm_type)
    return x.reshape(pats.shape)


def clahe(x: np.ndarray, clip_limit: float = 40.0, n_bins: int = 64, grid=(4, 4)) -> np.ndarray:
    """Contrast-limited adaptive histogram equalisation of (B, H, W) images
    in [0, 1] (preprocessing/clahe.py:17-130): per tile (the image reflect-
    padded on the bottom/right to a multiple of the grid) a histogram of
    floor(x (n_bins - 1)), clipped at max(clip_limit tile_px // n_bins, 1)
    with the excess spread evenly and the remainder one count to each of the
    first bins, cumulated into a CDF; each pixel is then read from the
    (tile-y, tile-x, bin) CDF volume by trilinear interpolation with
    align_corners=False / border semantics (grid_sample)."""
    B, H, W = x.shape
    gh, gw = grid
    th, tw = math.ceil(H / gh), math.ceil(W / gw)
    vpt = th * tw
    ph = gh - H % gh if H % gh else 0
    pw = gw - W % gw if W % gw else 0
    xp = np.pad(x, ((0, 0), (0, ph), (0, pw)), mode="reflect")
    cdfs = np.zeros((B, gh, gw, n_bins))
    for ty in range(gh):
        for tx in range(gw):
            tile = xp[:, ty * th:(ty + 1) * th, tx * tw:(tx + 1) * tw].reshape(B, -1)
            idx = (tile.astype(np.float32) * np.float32(n_bins - 1)).astype(np.int64)
            hist = np.stack([np.bincount(r, minlength=n_bins)[:n_bins] for r in idx]).astype(np.float64)
            hist = hist / hist.sum(axis=1, keepdims=True) * vpt
            if clip_limit > 0:
                limit = max(clip_limit * vpt // n_bins, 1)
                hist = np.minimum(hist, limit)
                clipped = vpt - hist.sum(axis=1)
                residual = np.remainder(clipped, n_bins)
                hist = hist + ((clipped - residual) / n_bins)[:, None]
                hist = hist + (np.arange(n_bins)[None] < residual[:, None])
            cdfs[:, ty, tx] = np.clip(np.cumsum(hist, axis=1) / vpt, 0.0, 1.0)

    def coord(c, size):
        return np.clip(((c + 1.0) * size - 1.0) / 2.0, 0.0, size - 1.0)

    fb = coord(x * 2.0 - 1.0, n_bins)                        # (B, H, W)
    fx = coord(np.linspace(-1.0, 1.0, W, dtype=np.float32).astype(np.float64), gw)  # (W,)
    fy = coord(np.linspace(-1.0, 1.0, H, dtype=np.float32).astype(np.float64), gh)  # (H,)
    b0 = np.floor(fb).astype(np.int64)
    x0 = np.floor(fx).astype(np.int64)
    y0 = np.floor(fy).astype(np.int64)
    b1, x1, y1 = np.minimum(b0 + 1, n_bins - 1), np.minimum(x0 + 1, gw - 1), np.minimum(y0 + 1, gh - 1)
    wb, wx, wy = fb - b0, (fx - x0)[None, None, :], (fy - y0)[None, :, None]
    bi = np.arange(B)[:, None, None]
    yy0, yy1 = y0[None, :, None], y1[None, :, None]
    xx0, xx1 = x0[None, None, :], x1[None, None, :]
    out = 0.0
    for yv, wyv in ((yy0, 1 - wy), (yy1, wy)):
        for xv, wxv in ((xx0, 1 - wx), (xx1, wx)):
            for bv, wbv in ((b0, 1 - wb), (b1, wb)):
                out = out + cdfs[bi, yv, xv, bv] * wyv * wxv * wbv
    return out


def standard_clean(pats: np.ndarray) -> np.ndarray:
    """Background, min-max, CLAHE, min-max (experiment_pats.py:287-297)."""
    x = normalize_per_pattern(subtract_overall_background(pats), "minmax")
    return normalize_per_pattern(clahe(x), "minmax")


def nlpar_offsets(k_rad: int):
    """Window offsets in the reference's order (nlpar.py:77-91): sorted by
    L1 norm with torch.argsort, whose order among equal norms is the one the
    reference gets (it decides which 8 offsets estimate the noise)."""
    import torch

    oc = torch.stack(torch.meshgrid(torch.arange(-k_rad, k_rad + 1), torch.arange(-k_rad, k_rad + 1),
                                    indexing="ij"), dim=-1).reshape(-1, 2)
    return oc[torch.argsort(torch.sum(torch.abs(oc), dim=-1))].numpy()


def nlpar(data: np.ndarray, k_rad: int = 5, coeff: float = 0.375, coeff_fit_tol: float = 1e-6,
          center_logit_bias: float = 0.0) -> np.ndarray:
    """Non-local pattern averaging of a (h, w, H, W) scan (nlpar.py:19-192,
    Brewick et al. 2019), float64."""
    hs, ws = data.shape[:2]
    P = data.shape[2] * data.shape[3]
    off = nlpar_offsets(k_rad)
    K = off.shape[0]
    flat = data.reshape(hs, ws, P).astype(np.float64)
    pad = np.zeros((hs + 2 * k_rad, ws + 2 * k_rad, P))
    pad[k_rad:k_rad + hs, k_rad:k_rad + ws] = flat
    oob = np.ones((hs + 2 * k_rad, ws + 2 * k_rad), dtype=bool)
    oob[k_rad:k_rad + hs, k_rad:k_rad + ws] = False
    dists = np.empty((hs, ws, K))
    mask = np.empty((hs, ws, K), dtype=bool)
    for i, (di, dj) in enumerate(off):
        nb = pad[k_rad + di:k_rad + di + hs, k_rad + dj:k_rad + dj + ws]
        dists[:, :, i] = ((nb - flat) ** 2).sum(-1)
        mask[:, :, i] = oob[k_rad + di:k_rad + di + hs, k_rad + dj:k_rad + dj + ws]
    sigma = np.sqrt(dists[:, :, 1:9].min(-1) / (2 * P))
    sp = np.ones((hs + 2 * k_rad, ws + 2 * k_rad))
    sp[k_rad:k_rad + hs, k_rad:k_rad + ws] = sigma
    for i, (di, dj) in enumerate(off):
        so = sp[k_rad + di:k_rad + di + hs, k_rad + dj:k_rad + dj + ws]
        s2 = sigma ** 2 + so ** 2
        dists[:, :, i] = (dists[:, :, i] - P * s2) / (2 ** 0.5 * P ** 0.5 * s2)
    weights = -np.maximum(dists, 0.0)
    g = 1.0
    nn = weights[:, :, :9]
    # on degenerate scans (most of the window outside) the fit runs away, as
    # the reference's does; the large coefficient then flattens the weights
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        for _ in range(10):
            g2 = g ** 2
            e = np.exp(nn / g2)
            obj = np.mean(e[:, :, 0] / e.sum(-1)) - coeff
            grad = np.mean(-2 * np.exp(nn[:, :, 0] / g2) * ((nn[:, :, :1] * e).sum(-1) - (nn * e).sum(-1))
                           / (g ** 3 * e.sum(-1) ** 2))
            g -= obj / grad
            if abs(obj) < coeff_fit_tol:
                break
    weights = weights / g ** 2
    if center_logit_bias > 0:
        weights[:, :, 0] += center_logit_bias
    weights = np.where(mask, -np.inf, weights)
    weights = np.exp(weights - weights.max(-1, keepdims=True))
    weights /= weights.sum(-1, keepdims=True)
    out = np.zeros_like(flat)
    for i, (di, dj) in enumerate(off):
        out += pad[k_rad + di:k_rad + di + hs, k_rad + dj:k_rad + dj + ws] * weights[:, :, i:i + 1]
    return out.reshape(data.shape)


# --------------------------------------------------------------------------
# Pattern-centre fitting (ebsd/fitting.py:54-540, spatial FFT fitter)
# --------------------------------------------------------------------------


def pixel_coords_with_periphery(detector_shape, pc_x_min, pc_x_max, pc_y_min, pc_y_max, binning=1):
    """(Hp * Wp, 3) detector-frame pixel coordinates of the detector enlarged
    by the pattern-centre search range, the padding (w_prior, w_after,
    h_prior, h_after) and the enlarged shape (fitting.py:219-289): per axis
    linspace(0.5 (b - 1) - prior, size + after - 0.5 (b - 1), n), row-major,
    z = 0. The padding uses the reference's float expressions and int()
    truncation."""
    import torch

    H, W = detector_shape
    bf = float(binning)
    wpp = int((0.5 - pc_x_min) * W / bf)
    wpa = int((pc_x_max - 0.5) * W / bf)
    hpp = int((0.5 - pc_y_min) * H / bf)
    hpa = int((pc_y_max - 0.5) * H / bf)
    shape = (H // binning + hpp + hpa, W // binning + wpp + wpa)
    # float32 linspace as torch builds it
    ii = torch.linspace(0.5 * (bf - 1) - hpp, H + hpa - 0.5 * (bf - 1), shape[0], dtype=torch.float32).double()
    jj = torch.linspace(0.5 * (bf - 1) - wpp, W + wpa - 0.5 * (bf - 1), shape[1], dtype=torch.float32).double()
    gi, gj = np.meshgrid(ii.numpy(), jj.numpy(), indexing="ij")
    pix = np.stack((gi.reshape(-1), gj.reshape(-1), np.zeros(gi.size)), axis=1)
    return pix, (wpp, wpa, hpp, hpa), shape


def bruker_se3(pc, primary_tilt_deg, secondary_tilt_deg, detector_shape):
    """Rotation and translation of the Bruker pattern-centre convention
    (fitting.py:54-115), float64."""
    pcx, pcy, pcz = pc
    rows, cols = float(detector_shape[0]), float(detector_shape[1])
    d, sx = math.radians(primary_tilt_deg), math.radians(secondary_tilt_deg)
    sd, cd, ss, cs = math.sin(d), math.cos(d), math.sin(sx), math.cos(sx)
    rot = np.array([[-sd, -ss * cd, cs * cd], [0.0, cs, ss], [-cd, ss * sd, -sd * cs]])
    t = np.array([
        pcx * cols * ss * cd + pcy * rows * sd + pcz * rows * cs * cd - ss * cd / 2 - sd / 2,
        -cols * pcx * cs + pcz * rows * ss + cs / 2,
        -cols * pcx * ss * sd + pcy * rows * cd - pcz * rows * sd * cs + ss * sd / 2 - cd / 2,
    ])
    return rot, t


def spatial_fft_pc_fit(master_pattern, patterns, quats_dict, pc_x_min=0.0, pc_x_max=1.0, pc_y_min=0.0,
                       pc_y_max=1.0, pc_z_min=0.3, pc_z_max=0.7, pc_z_steps=16, primary_tilt_deg=70.0,
                       secondary_tilt_deg=0.0, batch_size=1024, virtual_binning=1, batch_local_index=False):
    """The spatial FFT pattern-centre fitter (fitting.py:359-540), float64:
    patterns (B, 1, H, W) binned, min-max scaled, zero-mean, zero-padded to
    the enlarged detector; for each pc_z of linspace(min, max, steps) the
    dictionary (quats_dict, in the fitter's order) is simulated on the
    enlarged detector (pc_x = pc_y = 0.5, primary tilt negated) and
    circularly cross-correlated with every pattern by FFT (fftshifted); the
    running maximum over the dictionary starts at 0 per (pc_z, pattern,
    shift). The fit is the argmax of the mean over patterns; pc_x / pc_y
    follow from the shift. batch_local_index reproduces the reference's
    orientation index, which is local to the dictionary batch that won.
    Returns (pc (3,), orientation indices (B,), mean best dots (steps, Hp, Wp))."""
    import torch

    B, C, H, W = patterns.shape
    b = virtual_binning
    Hb, Wb = H // b, W // b
    x = avg_pool(patterns[:, 0].astype(np.float64), b)
    x = x - x.reshape(B, -1).min(axis=1)[:, None, None]
    x = x / x.reshape(B, -1).max(axis=1)[:, None, None]
    x = x - x.reshape(B, -1).mean(axis=1)[:, None, None]
    pix, pad, (Hp, Wp) = pixel_coords_with_periphery((H, W), pc_x_min, pc_x_max, pc_y_min, pc_y_max, b)
    xp = np.zeros((B, Hp, Wp))
    xp[:, pad[2]:pad[2] + Hb, pad[0]:pad[0] + Wb] = x
    xf = np.conj(np.fft.rfft2(xp))
    mp = avg_pool(master_pattern.astype(np.float64), b)
    z_vals = torch.linspace(pc_z_min, pc_z_max, pc_z_steps, dtype=torch.float32).double().numpy()
    best = np.zeros((pc_z_steps, B, Hp, Wp))
    best_i = np.zeros((pc_z_steps, B, Hp, Wp), dtype=np.int64)
    for zi, z in enumerate(z_vals):
        rot, t = bruker_se3((0.5, 0.5, z), -primary_tilt_deg, secondary_tilt_deg, (H, W))
        rays = unit_rays(pix @ rot.T + t)
        for j in range(0, quats_dict.shape[0], batch_size):
            q = quats_dict[j:j + batch_size].astype(np.float64)
            sims = project_patterns(mp, rays, q).reshape(-1, Hp, Wp)
            corr = np.fft.irfft2(np.fft.rfft2(sims)[:, None] * xf[None], s=(Hp, Wp))
            corr = np.fft.fftshift(corr, axes=(-2, -1))
            vals, idx = corr.max(axis=0), corr.argmax(axis=0)
            best[zi] = np.maximum(best[zi], vals)
            best_i[zi] = np.where(best[zi] == vals, idx + (0 if batch_local_index else j), best_i[zi])
    avg = best.mean(axis=1)
    zi, yi, xi = np.unravel_index(int(avg.argmax()), avg.shape)
    pc = np.array([0.5 + float(xi - pad[0] - (Wb + 1) // 2) / Wb, 0.5 + float(yi - pad[2] - (Hb + 1) // 2) / Hb,
                   float(z_vals[zi])])
    return pc, best_i[zi, :, yi, xi], avg


# --------------------------------------------------------------------------
# EMsoft master-pattern reader (io/read_master_pattern.py:7-53)
# --------------------------------------------------------------------------


def emsoft_master_pattern(accum_e: np.ndarray, north: np.ndarray, south: np.ndarray) -> np.ndarray:
    """The energy-weighted hemispheres side by side, float64: weights =
    accum_e summed over its first two axes, normalised; each hemisphere
    (1, n_e, H, W) squeezed and summed over energies with those weights
    (read_master_pattern.py:35-47)."""
    w = accum_e.astype(np.float64).sum(axis=(0, 1))
    w = w / w.sum()
    out = []
    for hemi in (north, south):
        h = hemi.astype(np.float64).reshape(-1, *hemi.shape[-2:])
        out.append((w[:, None, None] * h).sum(axis=0))
    return np.concatenate(out, axis=-1)
