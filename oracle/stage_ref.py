"""Stage the reference ebsdtorch package into ``oracle/_ref/`` (git-ignored).

TEST INFRASTRUCTURE ONLY: the staged copy is the reference itself, run as the
checker (golden vectors) and as the timed baselines of ``bench.py`` (the
reference's own CPU dictionary indexing, and its plain FP32 dictionary
indexing on the GPU). The product path never imports it.

The reference is pure Python on PyTorch, so "building" it is copying its
``ebsdtorch/`` package tree (``*.py`` files only, unmodified) next to this
file; ``oracle/_ref/`` is listed in ``.gitignore`` so nothing of it enters
the history, but it is not excluded from the GPU-box snapshot, so the
baselines can run there. ``oracle/_ref/MANIFEST.txt`` records the SHA-256 of
every staged file.

    python oracle/stage_ref.py REFERENCE_ROOT
    EBSD_REFERENCE_ROOT=... python oracle/stage_ref.py

REFERENCE_ROOT is the directory holding the reference's ``ebsdtorch/``.
"""

from __future__ import annotations

import hashlib
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEST = os.path.join(HERE, "_ref")


def stage(root: str, dest: str = DEST) -> str:
    """Copy root/ebsdtorch/**/*.py to dest/ebsdtorch/; returns dest."""
    src_pkg = os.path.join(root, "ebsdtorch")
    if not os.path.isfile(os.path.join(src_pkg, "__init__.py")):
        raise FileNotFoundError(f"no ebsdtorch package under {root!r}")
    dst_pkg = os.path.join(dest, "ebsdtorch")
    if os.path.isdir(dst_pkg):
        shutil.rmtree(dst_pkg)
    lines = []
    for dirpath, dirnames, filenames in os.walk(src_pkg):
        dirnames[:] = sorted(d for d in dirnames if d != "__pycache__")
        rel = os.path.relpath(dirpath, root)
        os.makedirs(os.path.join(dest, rel), exist_ok=True)
        for name in sorted(filenames):
            if not name.endswith(".py"):
                continue
            src = os.path.join(dirpath, name)
            dst = os.path.join(dest, rel, name)
            shutil.copyfile(src, dst)
            with open(dst, "rb") as f:
                lines.append(f"{hashlib.sha256(f.read()).hexdigest()}  {os.path.join(rel, name)}")
    with open(os.path.join(dest, "MANIFEST.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    return dest


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EBSD_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: python oracle/stage_ref.py REFERENCE_ROOT (or set EBSD_REFERENCE_ROOT)")
    print("staged into", stage(root))
