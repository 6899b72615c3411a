"""Time-series files: a compressed ``.npz`` archive of the arrays plus one member
holding the metadata as JSON text.

This is the file format of critmc (``src/critmc/io.py:33-48``), kept exactly so
that series and task caches written here load with critmc's
``TimeSeries.load`` and the other way round: the metadata member is called
``__meta__`` and holds a 0-d unicode array with the JSON document.
"""

from __future__ import annotations

import json
import math
from collections.abc import Mapping
from pathlib import Path
from typing import Any

import numpy as np

META_MEMBER = "__meta__"


def to_jsonable(obj: Any) -> Any:
    """A copy of ``obj`` that ``json.dumps`` accepts, with critmc's conventions:
    mapping keys become strings, tuples lists, arrays nested lists, numpy
    scalars Python numbers, paths strings, and a non-finite Python float its
    ``str`` ("nan", "inf", "-inf").  (A non-finite numpy scalar or array entry
    stays a float and is written as JSON's NaN / Infinity, as critmc does.)
    """
    if isinstance(obj, Mapping):
        return {str(key): to_jsonable(val) for key, val in obj.items()}
    if isinstance(obj, np.generic):
        return obj.item()
    if isinstance(obj, np.ndarray):
        return obj.tolist()
    if isinstance(obj, (list, tuple)):
        return list(map(to_jsonable, obj))
    if isinstance(obj, Path):
        return str(obj)
    if isinstance(obj, float) and not math.isfinite(obj):
        return str(obj)
    return obj


def save_npz(path: str | Path, arrays: dict[str, np.ndarray], meta: dict[str, Any]) -> Path:
    """Write ``arrays`` and ``meta`` to ``path`` (numpy adds ``.npz`` when missing)."""
    if META_MEMBER in arrays:
        raise ValueError(f"{META_MEMBER!r} holds the metadata and cannot name an array")
    members = {name: np.asarray(values) for name, values in arrays.items()}
    members[META_MEMBER] = np.array(json.dumps(to_jsonable(meta)))
    target = Path(path)
    target.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(target, **members)
    return target


def load_npz(path: str | Path) -> tuple[dict[str, np.ndarray], dict[str, Any]]:
    """The arrays and the metadata (empty when the file has none) of a series file."""
    with np.load(Path(path), allow_pickle=False) as archive:
        names = [name for name in archive.files if name != META_MEMBER]
        arrays = {name: archive[name] for name in names}
        meta = json.loads(archive[META_MEMBER].item()) if META_MEMBER in archive.files else {}
    return arrays, meta
