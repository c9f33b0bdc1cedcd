"""bench.py's reference arm (the oracle on this host's cores) on a small
cube, as the driver launches it: one JSON line with the contract's keys, the
GPU arm's metric, unit and workload string, the warm-up steps it was asked
for, and a positive rate; under torchrun only rank 0 prints, the other ranks
exit 0 without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "impl",
        "cpu_baseline", "e2e")


def run(world, rank, cells=6):
    env = dict(os.environ, WORLD_SIZE=str(world), RANK=str(rank))
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--cells", str(cells),
                          "--steps", "2", "--warmup", "4"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_single_gpu_line():
    import bench
    (d,) = run(1, 0)
    assert all(k in d for k in KEYS), [k for k in KEYS if k not in d]
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["dtype"] == "f64" and d["n_gpus"] == 1
    assert d["warmup"] == 4 and d["steps"] == 2
    # the GPU arm's workload string for the same --cells
    assert d["config"]["workload"] == ("cube_tet4: 6^3 cells x 6 tetrahedron_4 (1296 elements, "
                                       "343 nodes), linear elastic, FP64, dt = 0.8 x stable")
    assert d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_under_torchrun():
    (d,) = run(2, 0)
    assert d["n_gpus"] == 2
    assert d["config"]["workload"] == ("bar_tet4: 6 x 6 x 12 cells x 6 tetrahedron_4 (2592 "
                                       "elements, 637 nodes), linear elastic, FP64, "
                                       "dt = 0.8 x stable")
    assert run(2, 1) == []  # rank 1: no line, exit 0
