"""ebsdtorch_b200: B200-native (sm_100a) dictionary indexing for EBSD patterns.

Drop-in replacements for ebsdtorch's dictionary-indexing entry points:

    from ebsdtorch_b200.ebsd.indexing import (
        dictionary_index_orientations, pca_dictionary_index_orientations)

with the same containers (MasterPattern, EBSDGeometry, ExperimentPatterns)
under ebsdtorch_b200.ebsd. All compute runs in hand-written CUDA kernels of
the C-ABI library ebsdtorch_b200/_lib/libebsd_b200.so.
"""

__version__ = "0.1.0"
