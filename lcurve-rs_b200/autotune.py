"""Autotuner of a resident batch's launch shapes, with a JSON cache.

The planner picks three launch-shape choices by heuristic: elements per flux
work unit (in chunks of 256), threads per Roche-eclipsed element in the
phase scan, and persistent flux blocks per SM (lcb_batch_set_tuning in
lcurve_b200.h).  `autotune` times candidates for each choice on the batch
itself -- one warm-up evaluation, then the device time of `repeats`
evaluations from the library's per-stage CUDA events (Batch.profile) -- one
choice at a time, starting from the heuristic and keeping the fastest, and
records the winner under the batch's size class (models, element-evals and
Roche elements, in powers of two) and the device name.  `apply_cached` sets
a recorded choice on another batch of the same class.

Every candidate is a value the heuristic itself can produce, so the kernels
run as usual; results change only in the FP32 summation order of the flux
sum.  The reference has no counterpart (one fixed launch shape,
crates/lcurve-cuda/kernels/flux_kernel.cu:81, 543-545).
"""
from __future__ import annotations

import json
import math
import os
import pathlib

CHUNKS = (1, 2, 4, 8, 16)
SPLITS = (1, 2, 4, 8, 16)
KEYS = ("flux_chunks", "roche_split", "flux_blocks_per_sm")


def size_class(stats: dict) -> str:
    """Batches of the same class share a tuning: log2 of the model count,
    element-evals and Roche-eclipsed elements, rounded."""
    def lg(v):
        return int(round(math.log2(max(int(v), 1))))
    return f"m{lg(stats['models'])}-e{lg(stats['element_evals'])}-r{lg(stats['roche_elements'])}"


def _device_time(batch, scale: bool, repeats: int) -> float:
    batch.run(scale=scale)  # warm-up: graph capture and buffers for this shape
    best = math.inf
    for _ in range(repeats):
        best = min(best, sum(batch.profile(scale=scale).values()))
    return best


def autotune(batch, scale: bool = False, repeats: int = 2, cache: str | os.PathLike | None = None,
             device_name: str = "cuda") -> dict:
    """Tunes `batch` in place and returns {choice: value, 'ms': device time,
    'heuristic_ms': the heuristic's time, 'class': size class}.  With `cache`,
    the winner is recorded there (JSON: {device: {class: choice}})."""
    batch.set_tuning(0, 0, 0)
    current = batch.tuning()
    heuristic_ms = best_ms = _device_time(batch, scale, repeats)
    stats = batch.stats()
    max_bps = current["flux_blocks_per_sm"]
    axes = [("flux_chunks", CHUNKS)]
    if stats["roche_elements"] > 0:
        axes.append(("roche_split", SPLITS))
    axes.append(("flux_blocks_per_sm", tuple(range(1, max_bps + 1))))
    for key, values in axes:
        for v in values:
            if v == current[key]:
                continue
            trial = dict(current, **{key: v})
            batch.set_tuning(*(trial[k] for k in KEYS))
            ms = _device_time(batch, scale, repeats)
            if ms < best_ms:
                best_ms, current = ms, batch.tuning()
    # an axis that was not searched keeps the heuristic (0), so a cached choice applied to
    # a batch that does have, say, Roche-eclipsed elements does not pin that axis
    searched = {key for key, _ in axes}
    choice = {k: (current[k] if k in searched else 0) for k in KEYS}
    batch.set_tuning(*(choice[k] for k in KEYS))
    result = dict(current, ms=best_ms, heuristic_ms=heuristic_ms, **{"class": size_class(stats)})
    if cache is not None:
        path = pathlib.Path(cache)
        table = json.loads(path.read_text()) if path.exists() else {}
        table.setdefault(device_name, {})[result["class"]] = choice
        path.write_text(json.dumps(table, indent=1, sort_keys=True))
    return result


def apply_cached(batch, cache: str | os.PathLike, device_name: str = "cuda") -> bool:
    """Sets the recorded tuning of the batch's size class, if there is one."""
    path = pathlib.Path(cache)
    if not path.exists():
        return False
    choice = json.loads(path.read_text()).get(device_name, {}).get(size_class(batch.stats()))
    if choice is None:
        return False
    batch.set_tuning(*(int(choice[k]) for k in KEYS))
    return True
