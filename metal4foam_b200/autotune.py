"""Persistent choice of the SpMV launch shape per (device, mesh).

cf_autotune times every launch shape of the FP32 SpMV on a context's matrix
and returns the fastest; this module keeps the answer in a JSON file so a
mesh is timed once per device, not once per run:

    cfg = autotune.tuned_config(ctx, addr)     # times on first use, then cached

The key is the device description plus a structural fingerprint of the addressing
(cell and face counts and a CRC of lowerAddr / upperAddr) and the cell
reordering mode; coefficients do not enter it because the shapes move the
same bytes whatever the values.  The file is
``$CUDAFOAM_TUNE_CACHE`` or ``~/.cache/cudafoam/autotune.json``.
"""
from __future__ import annotations

import json
import os
import tempfile
import zlib
from typing import Optional

import numpy as np

from . import _lib

__all__ = ["cache_path", "mesh_key", "load_cache", "tuned_config"]


def cache_path() -> str:
    p = os.environ.get("CUDAFOAM_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "cudafoam", "autotune.json")


def mesh_key(device: str, addr, reorder: str = "auto") -> str:
    low = np.ascontiguousarray(addr.lowerAddr, np.int32)
    upp = np.ascontiguousarray(addr.upperAddr, np.int32)
    crc = zlib.crc32(upp.tobytes(), zlib.crc32(low.tobytes()))
    return f"{device}|n={addr.n}|nf={addr.nf}|crc={crc:08x}|reorder={reorder}"


def load_cache(path: Optional[str] = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(key: str, entry: dict, path: Optional[str] = None) -> None:
    path = path or cache_path()
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    d = load_cache(path)
    d[key] = entry
    # write-then-rename so concurrent readers never see a partial file
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(os.path.abspath(path)), suffix=".tmp")
    with os.fdopen(fd, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tuned_config(ctx: "_lib.Context", addr, reps: int = 20, path: Optional[str] = None,
                 retune: bool = False) -> dict:
    """Apply the cached shape for this mesh on ctx, or time all shapes
    (ctx must hold the mesh's topology and coefficients) and cache the
    winner.  Returns the applied shape as a dict."""
    key = mesh_key(ctx.description, addr, getattr(ctx, "reorder", "auto"))
    entry = None if retune else load_cache(path).get(key)
    if entry is not None:
        cfg = entry["config"]
        ctx.set_spmv_config(**cfg)
        return cfg
    best, table = ctx.autotune(reps=reps, apply=True)
    cfg = best.as_dict()
    _store(key, {"config": cfg, "timings_ms": [[t, ms] for t, ms in table]}, path)
    return cfg
