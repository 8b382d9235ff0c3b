from .experiment_pats import ExperimentPatterns
from .fitting import spatial_fft_pc_fitter
from .geometry import EBSDGeometry
from .indexing import dictionary_index_orientations, pca_dictionary_index_orientations
from .master_pattern import MasterPattern
from .refining import get_local_orientation_grid, orientation_grid_refinement

__all__ = [
    "EBSDGeometry",
    "ExperimentPatterns",
    "MasterPattern",
    "dictionary_index_orientations",
    "get_local_orientation_grid",
    "orientation_grid_refinement",
    "pca_dictionary_index_orientations",
    "spatial_fft_pc_fitter",
]
