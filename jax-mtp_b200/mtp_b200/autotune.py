"""Launch-shape autotuner for the evaluation and training kernels.

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

Training batches add a third parameter, the neighbour tile: the row length
`n_pad` the batch's neighbour rows are padded to (at least the longest row).
It sets the shared-memory staging of both kernels, and the evaluation kernel
stages whole warps of slots per atom, so a tile of 96 slots stages 3 warps and
one of 136 stages 5.  `tune_batch` searches (n_pad, threads, atoms per block)
for the batched forward (mtp_compute_batch_device, one persistent launch over
every configuration's atoms), `tune_adjoint` (n_pad, threads) for the training
gradient (mtp_adjoint_batch_device; it evaluates one atom per block).  Both
time every candidate with CUDA events on the caller's own batch and return
the winner, the batch restrided to its tile, and the table of candidates.  The
uneven configurations of a training batch (the reference pads atoms with NaN,
motep_jax_train_import.py:271) are padded here only in their rows' tails,
which the kernels never read.
"""

from __future__ import annotations

import json
import os
from typing import Dict, Iterable, Optional, Tuple

import torch

from .engine import MTPEngine

__all__ = ["tune", "tune_batch", "tune_adjoint", "tune_step", "apply_cached", "cache_key", "DEFAULT_CANDIDATES",
           "tile_candidates"]

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


def tile_candidates(longest_row: int) -> Tuple[int, ...]:
    """Row lengths worth trying: the smallest multiples of 8, 16 and 32 that hold the longest row."""
    out = []
    for m in (8, 16, 32):
        n = -(-max(1, longest_row) // m) * m
        if n not in out:
            out.append(n)
    return tuple(sorted(out))


def _timed(fn, calls: int) -> float:
    fn()                                         # warm-up (lazy buffers, schedules)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(calls):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / max(1, calls)


def _search(engine: MTPEngine, batch, tiles, candidates, run, calls: int):
    timings = {}
    best = None
    for n in tiles:
        b = batch.with_stride(n)
        for threads, apb in candidates:
            if engine.precision == "fp64" and apb > 2:
                continue
            tag = f"n{n}_{threads}x{apb}"
            try:
                engine.set_launch(threads, 0, apb)
                ms = _timed(lambda: run(b), calls)
                engine.sync_status()
            except RuntimeError as exc:       # a shape that does not fit this basis
                timings[tag] = str(exc)
                continue
            timings[tag] = {"ms": ms}
            if best is None or ms < best["ms"]:
                best = {"n_pad": n, "threads": threads, "atoms_per_block": apb, "ms": ms, "batch": b}
    if best is None:
        raise RuntimeError("no launch shape fits this basis")
    engine.set_launch(best["threads"], 0, best["atoms_per_block"])
    return best, timings


def tune_batch(engine: MTPEngine, batch, candidates: Iterable[Tuple[int, int]] = DEFAULT_CANDIDATES,
               tiles: Optional[Iterable[int]] = None, calls: int = 3) -> dict:
    """Fastest (n_pad, threads, atoms per block) for the batched forward of `batch`
    (a train.DeviceBatch).  Returns {"n_pad", "threads", "atoms_per_block", "ms",
    "batch" (restrided), "timings"}; the engine is left configured with the winner."""
    longest = int(batch.counts.max()) if batch.natoms else 1
    tiles = tuple(tiles) if tiles is not None else tile_candidates(longest)

    def run(b):
        engine.batch_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig)

    best, timings = _search(engine, batch, tiles, tuple(candidates), run, calls)
    _store(cache_key(engine, best["n_pad"]) + "|batch",
           {"threads": best["threads"], "atoms_per_block": best["atoms_per_block"], "ms": best["ms"]})
    return dict(best, timings=timings)


ADJOINT_CANDIDATES = ((256, 1), (512, 1))


def tune_step(engine: MTPEngine, batch, step, candidates: Iterable[Tuple[int, int]] = DEFAULT_CANDIDATES,
              tiles: Optional[Iterable[int]] = None, calls: int = 2, tag: str = "step") -> dict:
    """Fastest (n_pad, threads, atoms per block) for a whole training step
    `step(b)` on the restrided batch b (for example forward, loss and the
    adjoint, which share the engine's launch settings); same return layout as
    tune_batch."""
    longest = int(batch.counts.max()) if batch.natoms else 1
    tiles = tuple(tiles) if tiles is not None else tile_candidates(longest)
    best, timings = _search(engine, batch, tiles, tuple(candidates), step, calls)
    _store(cache_key(engine, best["n_pad"]) + "|" + tag,
           {"threads": best["threads"], "atoms_per_block": best["atoms_per_block"], "ms": best["ms"]})
    return dict(best, timings=timings)


def tune_adjoint(engine: MTPEngine, batch, gE, gF, gS, candidates: Iterable[Tuple[int, int]] = ADJOINT_CANDIDATES,
                 tiles: Optional[Iterable[int]] = None, calls: int = 2) -> dict:
    """Fastest (n_pad, threads) for the training gradient of `batch` with upstream
    gradients (gE, gF, gS); same return layout as tune_batch."""
    longest = int(batch.counts.max()) if batch.natoms else 1
    tiles = tuple(tiles) if tiles is not None else tile_candidates(longest)

    def run(b):
        engine.adjoint_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig, gE, gF, gS)

    best, timings = _search(engine, batch, tiles, tuple(candidates), run, calls)
    _store(cache_key(engine, best["n_pad"]) + "|adjoint", {"threads": best["threads"], "ms": best["ms"]})
    return dict(best, timings=timings)
