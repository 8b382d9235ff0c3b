from .experiment_pats import ExperimentPatterns
from .geometry import EBSDGeometry
from .indexing import dictionary_index_orientations, pca_dictionary_index_orientations
from .master_pattern import MasterPattern

__all__ = [
    "EBSDGeometry",
    "ExperimentPatterns",
    "MasterPattern",
    "dictionary_index_orientations",
    "pca_dictionary_index_orientations",
]
