"""Load the reference ebsdtorch (staged in ``oracle/_ref/`` or from a root).

TEST INFRASTRUCTURE ONLY (golden vectors, timed baselines); the product path
never imports this module.

The reference's ``ebsdtorch/ebsd/indexing.py`` ends (lines 479-578) in a
module-level demo script that imports ``kikuchipy``, which is not installed,
so the two dictionary-indexing functions are loaded by executing only the
file's lines 1-477 into a fresh module. Nothing in the reference is modified.
``load_indexing(top_slice=True)`` additionally replaces line 355's PCA slice
``eigenvectors[:, -n : -n + 300]`` by ``eigenvectors[:, -n:]`` (the n leading
components).
"""

from __future__ import annotations

import os
import sys
import types
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
STAGED = os.path.join(HERE, "_ref")

SHIPPED_PCA_SLICE = "pca_matrix = eigenvectors[:, -n_pca_components : (-n_pca_components + 300)]"
TOP_PCA_SLICE = "pca_matrix = eigenvectors[:, -n_pca_components:]"


def reference_root(root: Optional[str] = None) -> Optional[str]:
    """The directory holding the reference's ebsdtorch/: `root`, else
    $EBSD_REFERENCE_ROOT, else the staged copy; None when none exists."""
    for cand in (root, os.environ.get("EBSD_REFERENCE_ROOT"), STAGED):
        if cand and os.path.isfile(os.path.join(cand, "ebsdtorch", "__init__.py")):
            return cand
    return None


def import_reference(root: Optional[str] = None):
    """Put the reference on sys.path and import its package; returns the root."""
    r = reference_root(root)
    if r is None:
        raise FileNotFoundError("the reference ebsdtorch is not staged (run oracle/stage_ref.py) "
                                "and EBSD_REFERENCE_ROOT is not set")
    if r not in sys.path:
        sys.path.insert(0, r)
    import ebsdtorch  # noqa: F401

    mod_dir = os.path.dirname(os.path.abspath(ebsdtorch.__file__))
    if os.path.dirname(mod_dir) != os.path.abspath(r):
        raise RuntimeError(f"an ebsdtorch from {mod_dir} shadows the reference at {r}")
    return r


def load_indexing(root: Optional[str] = None, top_slice: bool = False) -> types.ModuleType:
    """Module holding the reference's dictionary_index_orientations and
    pca_dictionary_index_orientations (indexing.py lines 1-477)."""
    r = import_reference(root)
    path = os.path.join(r, "ebsdtorch", "ebsd", "indexing.py")
    with open(path) as f:
        src = "".join(f.readlines()[:477])
    if top_slice:
        if SHIPPED_PCA_SLICE not in src:
            raise RuntimeError("the reference's PCA slice (indexing.py:355) was not found")
        src = src.replace(SHIPPED_PCA_SLICE, TOP_PCA_SLICE)
    mod = types.ModuleType("ref_indexing_top" if top_slice else "ref_indexing")
    mod.__file__ = path
    exec(compile(src, path, "exec"), mod.__dict__)
    return mod


class quiet_stdout:
    """Silence file descriptor 1 (the reference's progress bar binds
    sys.stdout at import time, so only an fd-level redirect hides it)."""

    def __enter__(self):
        sys.stdout.flush()
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False
