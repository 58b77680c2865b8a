"""Launch-shape autotuner for the evaluation kernel.

The evaluation kernel has two shape parameters that trade occupancy against
work per block: threads per block (the lane count the contraction programs
are scheduled for; it also sets how many threads share a neighbour in the
force phase) and atoms evaluated together per block (they share every
program entry but multiply the shared-memory value space).  The best pair
depends on the basis level, the species count, the row length, the precision
and the GPU, so it is measured: every candidate is timed on the caller's own
device inputs with CUDA events around the evaluation kernel, and the winner is
cached in a JSON file keyed by those properties (default
``$MTP_B200_TUNE_CACHE`` or ``~/.cache/mtp_b200/launch.json``).
"""

from __future__ import annotations

import json
import os
from typing import Dict, Iterable, Optional, Tuple

import torch

from .engine import MTPEngine

__all__ = ["tune", "apply_cached", "cache_key", "DEFAULT_CANDIDATES"]

DEFAULT_CANDIDATES = ((128, 1), (256, 1), (512, 1), (128, 2), (256, 2), (512, 2), (256, 4), (512, 4))


def _cache_path() -> str:
    p = os.environ.get("MTP_B200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "mtp_b200", "launch.json")


def cache_key(engine: MTPEngine, stride: int) -> str:
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return (f"{name}|S{engine.species_count}R{engine.radial_funcs_count}K{engine.radial_basis_size}"
            f"M{engine.alpha_moments_count}B{engine.alpha_index_basic_count}T{engine.alpha_index_times_count}"
            f"|n{stride}|{engine.precision}")


def _load() -> Dict[str, dict]:
    try:
        with open(_cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(key: str, entry: dict) -> None:
    data = _load()
    data[key] = entry
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(data, fh, indent=1)
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home: the choice still applies to this engine


def apply_cached(engine: MTPEngine, stride: int) -> Optional[Tuple[int, int]]:
    e = _load().get(cache_key(engine, stride))
    if not e:
        return None
    engine.set_launch(e["threads"], 0, e["atoms_per_block"])
    return e["threads"], e["atoms_per_block"]


def tune(engine: MTPEngine, itypes, rijs, js, jtypes, counts, candidates: Iterable[Tuple[int, int]] = DEFAULT_CANDIDATES,
         calls: int = 3, use_cache: bool = True) -> dict:
    """Time each (threads, atoms_per_block) candidate on these inputs; keep the fastest.

    Returns {"threads", "atoms_per_block", "ms", "timings": {...}}; the engine
    is left configured with the winner.
    """
    stride = int(rijs.shape[1])
    key = cache_key(engine, stride)
    if use_cache:
        got = _load().get(key)
        if got:
            engine.set_launch(got["threads"], 0, got["atoms_per_block"])
            return dict(got, cached=True)
    timings = {}
    best = None
    for threads, apb in candidates:
        if engine.precision == "fp64" and apb > 2:
            continue
        try:
            engine.set_launch(threads, 0, apb)
            engine.compute_device(itypes, rijs, js, jtypes, counts)     # warm-up (and incoming lists)
            engine.profile(True)
            for _ in range(calls):
                engine.compute_device(itypes, rijs, js, jtypes, counts, reuse_neighbors=True)
            ms, n = engine.profile_read()
            engine.profile(False)
            engine.sync_status()
        except RuntimeError as exc:        # a shape that does not fit this basis
            timings[f"{threads}x{apb}"] = str(exc)
            continue
        launch = engine.launch()
        per = ms / max(1, n)
        timings[f"{threads}x{apb}"] = {"ms": per, "ran": launch}
        if best is None or per < best["ms"]:
            best = {"threads": threads, "atoms_per_block": apb, "ms": per, "ran": launch}
    if best is None:
        raise RuntimeError("no launch shape fits this basis")
    engine.set_launch(best["threads"], 0, best["atoms_per_block"])
    out = dict(best, timings=timings)
    _store(key, {"threads": best["threads"], "atoms_per_block": best["atoms_per_block"], "ms": best["ms"]})
    return out
