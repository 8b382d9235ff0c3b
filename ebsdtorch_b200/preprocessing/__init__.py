"""Experimental-pattern preprocessing (mirror of ebsdtorch/preprocessing/
and the preprocessing methods of ebsdtorch/ebsd/experiment_pats.py)."""

from .clahe import clahe_grayscale
from .nlpar import nlpar, nlpar_offsets
from .patterns import normalize_per_pattern, pattern_mean, standard_clean, subtract_overall_background
from .radial_mask import get_radial_mask

__all__ = [
    "clahe_grayscale",
    "get_radial_mask",
    "nlpar",
    "nlpar_offsets",
    "normalize_per_pattern",
    "pattern_mean",
    "standard_clean",
    "subtract_overall_background",
]
