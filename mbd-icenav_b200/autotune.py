"""Autotuner of the batched rollouts' work split.

How a substep's work is split over the persistent grid is a runtime choice of
the handle (``dem_set_work_split``): a thread or a warp per active element,
and a CTA or a warp per list rebuild / escaped element.  Every choice gives
bit-identical results (the GPU tests check each one against the others), so
the fastest can be picked by measurement alone.  ``tune`` times each choice on
the caller's own batch with CUDA events (median of a few runs) and sets the
fastest; choices are cached per workload bucket (systems, mean elements per
system, substeps), so a planner that builds many batches of the same shape
tunes once.  No counterpart in the reference (XLA picks its own schedule).
"""
from __future__ import annotations

import json
import math
import os
from typing import Callable, Dict, Optional, Tuple

from . import _abi

CHOICES = (
    ("auto", _abi.DEM_SPLIT_AUTO, _abi.DEM_SPLIT_AUTO),
    ("thread/cta", _abi.DEM_SPLIT_THREAD, _abi.DEM_SPLIT_CTA),
    ("thread/warp", _abi.DEM_SPLIT_THREAD, _abi.DEM_SPLIT_WARP),
    ("warp/cta", _abi.DEM_SPLIT_WARP, _abi.DEM_SPLIT_CTA),
    ("warp/warp", _abi.DEM_SPLIT_WARP, _abi.DEM_SPLIT_WARP),
)

_cache: Dict[str, str] = {}


def bucket(n_systems: int, n_elements: int, n_substeps: int) -> str:
    """Workload bucket: systems and mean elements per system in powers of two."""
    per = max(1, n_elements // max(1, n_systems))
    return f"q{int(math.log2(max(1, n_systems)))}-e{int(math.log2(per))}-k{n_substeps}"


def _cache_path() -> Optional[str]:
    return os.environ.get("MBD_ICENAV_AUTOTUNE")


def _load():
    p = _cache_path()
    if p and os.path.exists(p) and not _cache:
        try:
            with open(p) as fh:
                _cache.update(json.load(fh))
        except (OSError, ValueError):
            pass


def _save():
    p = _cache_path()
    if p:
        tmp = p + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(_cache, fh, indent=1, sort_keys=True)
        os.replace(tmp, p)


def apply(frame_step, name: str):
    for nm, fsplit, msplit in CHOICES:
        if nm == name:
            frame_step.set_work_split(fsplit, msplit)
            return
    raise ValueError(f"unknown work split {name!r}")


def tune(frame_step, run: Callable[[], object], repeats: int = 3, key: Optional[str] = None,
         force: bool = False) -> Tuple[str, Dict[str, float]]:
    """Time ``run()`` (one batch on ``frame_step``) under every work split, set
    the fastest and return (its name, {name: median ms}).  With a cached choice
    for ``key`` (default: the handle's workload bucket) it is set without timing."""
    import torch
    _load()
    if key is None:
        key = bucket(frame_step.n_systems, frame_step.n, frame_step.n_ice_steps)
    if key in _cache and not force:
        apply(frame_step, _cache[key])
        return _cache[key], {}
    stream = torch.cuda.current_stream(frame_step.device)
    times: Dict[str, float] = {}
    for nm, fsplit, msplit in CHOICES:
        frame_step.set_work_split(fsplit, msplit)
        run()  # warm: lists and buckets settle for this split
        ms = []
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        times[nm] = sorted(ms)[len(ms) // 2]
    best = min(times, key=times.get)
    apply(frame_step, best)
    _cache[key] = best
    _save()
    return best, times
