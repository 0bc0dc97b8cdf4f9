"""Measured choice among launch configurations, with an optional on-disk cache.

The dense local stage of uneven batches (polygon macrocells, ``PolygonP2Plan``) has two
schedule parameters that trade padding against launch count and concurrency: the bin
width (local systems are padded to the next multiple of it, one launch chain per bin)
and the number of streams the bins' chains are spread over.  ``choose`` times every
candidate with the caller's measurement, keeps the fastest and records it under a key
(device name and the problem's size signature), so that a later plan of the same shape
on the same device skips the search.
"""

from __future__ import annotations

import hashlib
import json
import os
from collections.abc import Callable, Hashable, Iterable
from pathlib import Path

import numpy as np


def shape_key(device_name: str, *arrays) -> str:
    """A stable key for a device and the integer arrays that fix a problem's layout."""
    h = hashlib.sha256(device_name.encode())
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.int64).tobytes())
    return h.hexdigest()[:32]


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def choose(candidates: Iterable[Hashable], measure: Callable[[Hashable], float], *, key: str | None = None,
           cache: str | os.PathLike | None = None) -> tuple[Hashable, dict]:
    """Time every candidate (``measure`` returns milliseconds, lower is better) and
    return the fastest with all timings.  With ``cache`` and ``key``, a recorded choice
    that is still among the candidates is returned without measuring, and a new choice
    is recorded."""
    cands = list(candidates)
    if not cands:
        raise ValueError("no candidate configurations")
    path = Path(cache) if cache is not None else None
    if path is not None and key is not None:
        hit = _load(path).get(key)
        if hit is not None:
            for c in cands:
                if json.dumps(c) == json.dumps(hit["choice"]):
                    return c, {"cached": True, "timings_ms": hit.get("timings_ms", {})}
    timings = {}
    for c in cands:
        ms = float(measure(c))
        if not ms == ms or ms < 0:  # NaN or negative: a failed measurement
            raise RuntimeError(f"measurement of {c!r} failed")
        timings[json.dumps(c)] = ms
    best = min(cands, key=lambda c: timings[json.dumps(c)])
    if path is not None and key is not None:
        data = _load(path)
        data[key] = {"choice": best, "timings_ms": timings}
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(path.suffix + ".tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(path)
    return best, {"cached": False, "timings_ms": timings}
