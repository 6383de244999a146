"""Autotuner for the launch configuration of a workload.

The settings change speed but not results (every kernel form sums the same terms in the same
order, and the neighbour list is always a superset of the overlapping pairs summed in
caller-index order, whatever its cutoff or the re-sort):

* ``contact_lanes``     threads per particle of the contact kernel: 0 automatic (one thread per
                        particle in dense steps, 8 in sparse ones), 1, 4 or 8 (the three-kernel
                        step with that cooperative width)
* ``dense_form``        dense steps as one kernel (1) or as the pair-parallel three kernels (2)
* ``stream_split``      streaming pass: 0 automatic (one persistent kernel over tiles staged in
                        shared memory) or 1 (one thread per particle, ``stream_block`` wide blocks)
* ``stream_block``      block size of the one-thread-per-particle streaming kernel (64, 128, 256)
* ``steps_per_launch``  0: the step loop as a graph while-loop; else fused steps per captured graph
* ``skin``              Verlet skin (0.5, 1, 2 or 4 times the scenario's), i.e. the rebuild cadence
                        against the listed neighbours a streaming pass checks

``tune`` times short runs of the caller's workload for each candidate, one setting at a time
(coordinate search from the defaults), and caches the winner per size bucket (log2 of the
particle count, precision, batched or single, and for a batch the scene-size bucket of its
scenes) in a JSON file (``$CABANADEM_B200_TUNE_CACHE``, default
``~/.cache/cabanadem_b200/autotune.json``).  Batches are tuned per scene-size bucket through
``scenarios.split_scenes`` and run by ``api.BatchRunner``.
"""
from __future__ import annotations

import json
import math
import os
import time

from . import api

DEFAULTS = dict(contact_lanes=0, dense_form=0, stream_split=0, stream_block=128, steps_per_launch=0,
                skin_factor=1.0)
CANDIDATES = dict(contact_lanes=(0, 1, 4, 8), dense_form=(1, 2), stream_split=(0, 1), stream_block=(64, 128, 256),
                  steps_per_launch=(0, 32), skin_factor=(0.5, 1.0, 2.0, 4.0))
ORDER = ("contact_lanes", "dense_form", "stream_split", "stream_block", "steps_per_launch", "skin_factor")


def cache_path():
    return os.environ.get("CABANADEM_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "cabanadem_b200", "autotune.json"))


def bucket(sc, precision):
    batched = sc.extra.get("scene") is not None
    key = "n2^%d|p%d|%s" % (int(math.log2(max(sc.state.n, 1))), int(precision), "batched" if batched else "single")
    if batched and sc.extra.get("counts") is not None:
        from .scenarios import scene_bucket_of
        sb = {scene_bucket_of(int(c)) for c in sc.extra["counts"]}
        key += "|scenes%s" % (str(sb.pop()) if len(sb) == 1 else "mixed")
    return key


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table):
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)


def time_config(sc, cfg, precision, warmup, steps, ctx=None):
    """Seconds per step of `steps` fused steps after `warmup` steps."""
    base_skin = sc.skin
    sc.skin = base_skin * cfg["skin_factor"]
    try:
        s = api.from_scenario(sc, ctx=ctx, precision=precision, **_solver_kwargs(cfg))
        s.run_steps(warmup)
        t0 = time.perf_counter()
        s.run_steps(steps)      # returns after the device finished (status read-back)
        dt = (time.perf_counter() - t0) / steps
        s.close()
        s.particles.close()
    finally:
        sc.skin = base_skin
    return dt


def tune(sc, precision=0, warmup=20, steps=200, use_cache=True, ctx=None):
    """Best setting of every knob of CANDIDATES for this workload's bucket."""
    key = bucket(sc, precision)
    table = _load() if use_cache else {}
    if use_cache and key in table:
        return dict(table[key]["config"])
    best = dict(DEFAULTS)
    best_t = time_config(sc, best, precision, warmup, steps, ctx)
    trials = [(dict(best), best_t)]
    tried = {tuple(sorted(best.items()))}
    for name in ORDER:
        for v in CANDIDATES[name]:
            cfg = dict(best)
            cfg[name] = v
            key_cfg = tuple(sorted(cfg.items()))
            if key_cfg in tried:      # the current best, or timed before the best moved
                continue
            tried.add(key_cfg)
            t = time_config(sc, cfg, precision, warmup, steps, ctx)
            trials.append((cfg, t))
            if t < best_t:
                best, best_t = cfg, t
    table[key] = {"config": best, "s_per_step": best_t, "trials": [[c, t] for c, t in trials]}
    if use_cache:
        _store(table)
    return dict(best)


def packaged(sc, precision):
    """The B200 settings shipped with the package for this workload's bucket
    (``data/autotune_b200.json``, found by ``tune`` on a B200), or None."""
    path = os.path.join(os.path.dirname(__file__), "data", "autotune_b200.json")
    try:
        with open(path) as f:
            table = json.load(f)
    except (OSError, ValueError):
        return None
    cfg = table.get(bucket(sc, precision))
    return dict(cfg) if isinstance(cfg, dict) else None


def _solver_kwargs(cfg):
    full = dict(DEFAULTS)
    full.update(cfg)
    return dict(stream_block=full["stream_block"], steps_per_launch=full["steps_per_launch"],
                contact_lanes=full["contact_lanes"], dense_form=full["dense_form"], stream_split=full["stream_split"])


def apply(sc, cfg):
    """Scenario settings for a tuned configuration (skin) and from_scenario keyword arguments."""
    sc.skin = sc.skin * dict(DEFAULTS, **cfg)["skin_factor"]
    return _solver_kwargs(cfg)
