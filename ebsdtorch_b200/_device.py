"""Device guard for the public entry points.

The C library launches its kernels on the current CUDA device, so an entry
point whose data lives on another GPU must make that GPU current for the
call. `on_data_device` does this: the device is the `device=` argument when
given, else that of the first CUDA tensor among the arguments (directly, in a
list or tuple, or as the `master_pattern` / `patterns` of a container). The
previous current device is restored on return. With no CUDA data the call
runs unchanged (host data goes to the current device).
"""

from __future__ import annotations

import functools

import torch


def _find(obj, depth: int = 0):
    if isinstance(obj, torch.Tensor):
        return obj.device if obj.is_cuda else None
    if depth > 1:
        return None
    if isinstance(obj, (list, tuple)):
        for o in obj:
            d = _find(o, depth + 1)
            if d is not None:
                return d
        return None
    for attr in ("master_pattern", "patterns"):
        t = getattr(obj, attr, None)
        if isinstance(t, torch.Tensor) and t.is_cuda:
            return t.device
    return None


def on_data_device(fn):
    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        dev = kwargs.get("device")
        if dev is None:
            for a in list(args) + list(kwargs.values()):
                dev = _find(a)
                if dev is not None:
                    break
        if dev is None:
            return fn(*args, **kwargs)
        dev = torch.device(dev)
        if dev.type != "cuda" or dev.index is None:
            return fn(*args, **kwargs)
        with torch.cuda.device(dev):
            return fn(*args, **kwargs)

    return wrapper
