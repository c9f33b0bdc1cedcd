"""Autotuner of the fused patch step.

Chooses the patch shape (elements per patch, node cap) and the schedule (one
CTA per patch, or a persistent grid striding over the patches) by timing a
few steps of each candidate with CUDA events on the model's stream, and
caches the winner in a JSON file keyed by GPU name, element type, precision
mode and problem size (log2 bucket of the element count).
"""
from __future__ import annotations

import json
import math
import os

from . import _abi

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "akantu_b200", "tuning.json")

# (elements per patch, node cap, persistent CTAs per SM or 0)
CANDIDATES = {
    _abi.TRIANGLE_3: [(1024, 640, 0), (512, 320, 0), (2048, 1100, 0), (1024, 640, 3), (768, 480, 0)],
    _abi.TETRAHEDRON_4: [(1024, 400, 0), (512, 220, 0), (1536, 500, 0), (1024, 400, 3)],
    _abi.HEXAHEDRON_8: [(512, 800, 0), (256, 448, 0), (384, 640, 0), (512, 800, 2)],
    _abi.SEGMENT_2: [(1024, 1100, 0), (512, 600, 0)],
}


def _gpu_key():
    try:
        import torch
        p = torch.cuda.get_device_properties(0)
        return p.name, p.multi_processor_count
    except Exception:
        return "unknown", 148


def cache_key(element_type, precision, nb_elements):
    name, _ = _gpu_key()
    bucket = int(math.log2(max(nb_elements, 1)))
    return "%s|%d|%d|%d" % (name, element_type, precision, bucket)


def load_cache(path=DEFAULT_CACHE):
    try:
        with open(path) as fh:
            return json.load(fh)
    except Exception:
        return {}


def save_cache(cache, path=DEFAULT_CACHE):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(cache, fh, indent=1)
    except OSError:
        pass


def tune(build, element_type, precision, nb_elements, steps=20, warmup=3,
         cache_path=DEFAULT_CACHE, use_cache=True, log=None):
    """build(patch_elements, patch_nodes, patch_grid) -> a ready model (time
    step set). Returns (best options dict, list of (options, ms/step))."""
    key = cache_key(element_type, precision, nb_elements)
    cache = load_cache(cache_path) if use_cache else {}
    if key in cache:
        return cache[key], []
    _, sms = _gpu_key()
    results = []
    for pe, pn, per_sm in CANDIDATES[element_type]:
        grid = per_sm * sms if per_sm else 0
        model = build(pe, pn, grid)
        model.solveSteps(warmup)
        ms = model.timeSolveSteps(steps) / steps
        model.close()
        opt = dict(patch_elements=pe, patch_nodes=pn, patch_grid=grid)
        results.append((opt, ms))
        if log:
            log("tune %s: %.4f ms/step" % (opt, ms))
    best = min(results, key=lambda r: r[1])[0]
    cache[key] = best
    if use_cache:
        save_cache(cache, cache_path)
    return best, results
