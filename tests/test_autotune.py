"""The autotuner's staged search (akantu_b200/autotune.py) on a fake model
whose step time is a known function of the patch shape: it must find the
fastest shape among the candidates it builds, skip shapes the builder
refuses, try the persistent schedules of the best shape only, reuse its
cache, and build no candidate twice."""
import math

import pytest

from akantu_b200 import _abi, autotune


class FakeModel:
    def __init__(self, pe, pn, grid, cost):
        self.ms = cost(pe, pn, grid)

    def solveSteps(self, n):
        pass

    def timeSolveSteps(self, n):
        return self.ms * n

    def close(self):
        pass


def run(tmp_path, etype, cost, refuse=lambda pe, pn, g: False):
    built = []

    def build(pe, pn, grid):
        built.append((pe, pn, grid))
        if refuse(pe, pn, grid):
            raise RuntimeError("refused")
        return FakeModel(pe, pn, grid, cost)
    best, trials = autotune.tune(build, etype, _abi.MODE_FP64, 10 ** 6,
                                 cache_path=str(tmp_path / "tuning.json"))
    return best, trials, built


@pytest.mark.parametrize("etype", [_abi.TRIANGLE_3, _abi.TETRAHEDRON_4, _abi.HEXAHEDRON_8,
                                   _abi.SEGMENT_2])
def test_search_finds_the_fastest_candidate(tmp_path, etype):
    space = autotune.SPACE[etype]
    pe_best = space["elements"][len(space["elements"]) // 2]
    r_best = space["ratios"][-1]

    def cost(pe, pn, grid):  # best at (pe_best, r_best), one CTA per patch
        return (1.0 + abs(math.log2(pe / pe_best)) + 3 * abs(pn / pe - r_best)
                + (0.2 if grid else 0.0))
    best, trials, built = run(tmp_path, etype, cost)
    assert best["patch_elements"] == pe_best
    assert best["patch_nodes"] == autotune._node_cap(pe_best, r_best)
    assert best["patch_grid"] == 0
    assert min(t[1] for t in trials) == pytest.approx(cost(pe_best, best["patch_nodes"], 0))
    assert len(built) == len(set(built))  # no candidate built twice
    assert len(built) == len(space["elements"]) + len(space["ratios"]) - 1 + len(space["persist"])
    # persistent schedules are tried only for the best shape
    assert {(pe, pn) for pe, pn, g in built if g} == {(pe_best, best["patch_nodes"])}
    # the cache answers the second call without building
    best2, trials2, built2 = run(tmp_path, etype, cost)
    assert best2 == best and trials2 == [] and built2 == []


def test_refused_shapes_are_skipped(tmp_path):
    def cost(pe, pn, grid):
        return 1.0 / pe  # bigger is faster...
    big = autotune.SPACE[_abi.TRIANGLE_3]["elements"][-1]
    best, trials, built = run(tmp_path, _abi.TRIANGLE_3, cost,
                              refuse=lambda pe, pn, g: pe == big)  # ...but the biggest is refused
    assert best["patch_elements"] < big
    assert all(t[0]["patch_elements"] != big for t in trials)


def test_nothing_buildable_raises(tmp_path):
    with pytest.raises(RuntimeError):
        run(tmp_path, _abi.SEGMENT_2, lambda *a: 1.0, refuse=lambda *a: True)
