"""Autotuner of the fused patch step.

Chooses the patch shape (elements per patch, node cap) and the schedule (one
CTA per patch, or a persistent grid of k CTAs per SM striding over the
patches) by timing a few steps of each candidate with CUDA events on the
model's stream, in three stages per element type: the patch size at the
type's usual nodes-per-element ratio, then the node cap around the best
size, then the persistent schedules of the best shape. Candidates the
library refuses (a node cap too small for the mesh, shared memory over the
limit) are skipped. The winner is cached in a JSON file keyed by GPU name,
element type, precision mode and problem size (log2 bucket of the element
count).
"""
from __future__ import annotations

import json
import math
import os

from . import _abi

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "akantu_b200", "tuning.json")

# Search space per element type: patch sizes (elements), node caps as
# multiples of the patch size (the middle one is the usual ratio of a compact
# patch of that type), persistent CTAs per SM tried for the best shape.
SPACE = {
    _abi.SEGMENT_2: dict(elements=(256, 512, 1024, 2048), ratios=(1.02, 1.08, 1.15), persist=(2, 4)),
    _abi.TRIANGLE_3: dict(elements=(256, 384, 512, 768, 1024, 1536, 2048),
                          ratios=(0.56, 0.625, 0.70), persist=(2, 3)),
    _abi.TETRAHEDRON_4: dict(elements=(256, 384, 512, 768, 1024, 1536),
                             ratios=(0.33, 0.39, 0.47), persist=(2, 3)),
    _abi.HEXAHEDRON_8: dict(elements=(128, 192, 256, 384, 512),
                            ratios=(1.35, 1.56, 1.8), persist=(1, 2)),
}


def _node_cap(elements, ratio):
    return int(math.ceil(elements * ratio / 16.0)) * 16


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
    space = SPACE[element_type]
    results, seen = [], {}

    def trial(pe, pn, per_sm):
        opt = dict(patch_elements=int(pe), patch_nodes=int(pn),
                   patch_grid=int(per_sm * sms) if per_sm else 0)
        key = tuple(opt.values())
        if key in seen:
            return seen[key]
        try:
            model = build(opt["patch_elements"], opt["patch_nodes"], opt["patch_grid"])
        except Exception as exc:  # refused shape: skipped
            if log:
                log("tune %s: skipped (%s)" % (opt, exc))
            seen[key] = None
            return None
        try:
            model.solveSteps(warmup)
            ms = model.timeSolveSteps(steps) / steps
        finally:
            model.close()
        results.append((opt, ms))
        seen[key] = ms
        if log:
            log("tune %s: %.4f ms/step" % (opt, ms))
        return ms

    def best_of(cands):
        timed = [(c, trial(*c)) for c in cands]
        timed = [(c, t) for c, t in timed if t is not None]
        return min(timed, key=lambda ct: ct[1])[0] if timed else None

    mid = space["ratios"][len(space["ratios"]) // 2]
    shape = best_of([(pe, _node_cap(pe, mid), 0) for pe in space["elements"]])
    if shape is None:
        raise RuntimeError("autotune: no candidate could be built")
    pe = shape[0]
    shape = best_of([(pe, _node_cap(pe, r), 0) for r in space["ratios"]])
    best_of([shape] + [(shape[0], shape[1], k) for k in space["persist"]])
    best = min(results, key=lambda r: r[1])[0]
    cache[key] = best
    if use_cache:
        save_cache(cache, cache_path)
    return best, results
