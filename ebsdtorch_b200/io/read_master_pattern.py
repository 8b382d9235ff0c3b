"""EMsoft master-pattern reader (mirror of ebsdtorch/io/read_master_pattern.py:
7-53).

An EMsoft EBSD master-pattern file holds, per electron energy, the modified
square-Lambert projections of both hemispheres (EMData/EBSDmaster/mLPNH and
mLPSH, stored (1, n_energies, H, W)). It also holds the Monte Carlo energy
histogram over the Lambert square (EMData/MCOpenCL/accum_e, stored (H', W',
n_energies)) and the space group (CrystalData/SpaceGroupNumber). The master
pattern used for indexing is the energy-weighted sum of each hemisphere, the
weights being the histogram summed over the square and normalised. The
hemispheres are placed side by side (north | south) as MasterPattern expects.

This is a one-time host-side load of a few images, so it runs in NumPy and
returns the pattern on the host, as the reference does; move the
MasterPattern to the GPU afterwards. Reading the file needs h5py, as in the
reference. `h5py_module` lets a caller pass an object with the same `File`
API instead.
"""

from __future__ import annotations

import numpy as np
import torch

from ..ebsd.master_pattern import MasterPattern

ACCUM_E = "EMData/MCOpenCL/accum_e"
NORTH = "EMData/EBSDmaster/mLPNH"
SOUTH = "EMData/EBSDmaster/mLPSH"
SPACE_GROUP = "CrystalData/SpaceGroupNumber"


def master_pattern_from_emsoft(accum_e, north, south, space_group: int) -> MasterPattern:
    """MasterPattern from EMsoft arrays as stored: accum_e (H', W', n_e),
    north / south (1, n_e, H, W) (or (n_e, H, W), or (H, W) for one energy).
    Weights: accum_e summed over its first two axes, normalised to sum 1;
    result: (H, 2W) float32, north | south."""
    acc = np.asarray(accum_e, dtype=np.float32)
    counts = acc.reshape(-1, acc.shape[-1]).sum(axis=0)
    weights = counts / counts.sum()
    halves = []
    for hemi in (north, south):
        h = np.asarray(hemi, dtype=np.float32).squeeze()
        if h.ndim == 2:
            h = h[None]
        if h.shape[0] != weights.shape[0]:
            raise ValueError(f"{h.shape[0]} energy bins in the master pattern, {weights.shape[0]} in accum_e")
        halves.append(np.tensordot(weights, h, axes=(0, 0)).astype(np.float32))
    return MasterPattern(torch.from_numpy(np.concatenate(halves, axis=-1)), space_group=int(space_group))


def read_master_pattern(file_path, *, h5py_module=None) -> MasterPattern:
    """Read an EMsoft master-pattern file into a MasterPattern (host
    tensor), as read_master_pattern.py:7-53 does."""
    if h5py_module is None:
        try:
            import h5py as h5py_module
        except ImportError as exc:  # the reference needs h5py too
            raise ImportError("reading EMsoft HDF5 master-pattern files needs h5py") from exc
    with h5py_module.File(file_path, "r") as f:
        accum_e = f[ACCUM_E][:]
        north = f[NORTH][:]
        south = f[SOUTH][:]
        space_group = f[SPACE_GROUP][0]
    return master_pattern_from_emsoft(accum_e, north, south, int(space_group))
