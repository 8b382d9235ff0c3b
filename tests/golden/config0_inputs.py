"""Inputs of the config-0 golden case, regenerated deterministically on the CPU.

Plain dictionary indexing at the small configuration: a 2 x 257 x 257
synthetic master pattern (Gaussian Kikuchi bands on the cubic {111}, {200},
{220}, {311} great circles), a 60 x 60 detector (PC 0.5, 0.5, 0.6; 70 deg
tilt), the m-3m 1.0 deg dictionary (36,829 orientations) and 4,096 patterns
projected at seeded uniform orientations, Gaussian-blurred (sigma 1 px),
scaled to a mean of 200 counts and Poisson sampled.

Only the seeds, the reference's outputs and the SHA-256 of the inputs are
committed (``config0.npz``); the inputs (0.5 MB master pattern, 59 MB of
patterns) are rebuilt here, on whichever machine runs the test. Every step
that could round differently on another CPU (vectorised transcendental
functions) happens in float64 before a float32 cast of the master pattern or
before the Poisson draw, whose integer outcome does not move for a last-bit
change of its mean; the checksums make any mismatch loud.
"""

from __future__ import annotations

import hashlib
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

CASE = dict(mp_size=257, mp_seed=5, det=(60, 60), pc=(0.5, 0.5, 0.6), tilts=(0.0, 70.0, 0.0), n=4096,
            quat_seed=6, mean_counts=200.0, blur_sigma=1.0, poisson_seed=7, res=1.0, k=4, perm_seed=8,
            dictionary_chunk_size=4096, experiment_chunk_size=1024)


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def uniform_quaternions(n: int, seed: int) -> np.ndarray:
    """(n, 4) float64 uniform unit quaternions (Shoemake), w >= 0."""
    rng = np.random.default_rng(seed)
    u, v, w = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack((np.sqrt(1 - u) * np.sin(2 * math.pi * v), np.sqrt(1 - u) * np.cos(2 * math.pi * v),
                  np.sqrt(u) * np.sin(2 * math.pi * w), np.sqrt(u) * np.cos(2 * math.pi * w)), axis=1)
    return np.where(q[:, :1] < 0, -q, q)


def _blur(x: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian blur of (n, H, W) float64 with replicate padding."""
    r = max(1, int(math.ceil(3 * sigma)))
    k = np.array([math.exp(-0.5 * (t / sigma) ** 2) for t in range(-r, r + 1)])
    k /= k.sum()
    p = np.pad(x, ((0, 0), (0, 0), (r, r)), mode="edge")
    y = sum(k[i] * p[:, :, i:i + x.shape[2]] for i in range(2 * r + 1))
    p = np.pad(y, ((0, 0), (r, r), (0, 0)), mode="edge")
    return sum(k[i] * p[:, i:i + x.shape[1], :] for i in range(2 * r + 1))


def make_inputs(case: dict = CASE, chunk: int = 512) -> dict:
    """master_pattern (H, 2W) float32, counts (n, h, w) uint16, truth (n, 4)
    float64, and their checksums."""
    from ebsdtorch_b200.synthetic import synthetic_master_pattern
    from oracle import di_oracle as O

    mp = synthetic_master_pattern(case["mp_size"], seed=case["mp_seed"]).numpy()
    h, w = case["det"]
    rays = O.unit_rays(O.detector_coords_sample_frame((h, w), case["pc"], case["tilts"]))
    truth = uniform_quaternions(case["n"], case["quat_seed"])
    rng = np.random.default_rng(case["poisson_seed"])
    mp64 = mp.astype(np.float64)
    counts = np.empty((case["n"], h, w), dtype=np.uint16)
    for s0 in range(0, case["n"], chunk):
        x = O.project_patterns(mp64, rays, truth[s0:s0 + chunk]).reshape(-1, h, w)
        x = x - x.min(axis=(1, 2), keepdims=True)
        x = _blur(x, case["blur_sigma"])
        x = x * (case["mean_counts"] / np.maximum(x.mean(axis=(1, 2), keepdims=True), 1e-12))
        counts[s0:s0 + chunk] = np.minimum(rng.poisson(x), 65535).astype(np.uint16)
    return {"master_pattern": mp, "counts": counts, "truth": truth,
            "sha256_master_pattern": sha256(mp), "sha256_counts": sha256(counts)}
