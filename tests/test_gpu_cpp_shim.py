"""The C++ shim (include/akantu_b200/solid_mechanics_model.hh) driving
libakb.so from a compiled program, checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from akantu_b200 import _abi, configs
from tests.golden_cases import OracleAdapter

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def build_program(tmp_path, name="shim_plate"):
    exe = str(tmp_path / name)
    lib = os.path.join(ROOT, "akantu_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", name + ".cc"), "-o", exe,
                    "-L", lib, "-lakb", "-Wl,-rpath," + lib], check=True)
    return exe


def test_shim_compiles(tmp_path):
    """The shim header compiles and links against libakb.so (no GPU needed)."""
    build_program(tmp_path)
    build_program(tmp_path, "shim_fe2")


@pytest.mark.gpu
def test_shim_fe2_user_material_with_rves(tmp_path):
    """A user material backed by homogeneous RVE solves equals the built-in
    neo-Hookean material, through the C++ shim."""
    exe = build_program(tmp_path, "shim_fe2")
    out = subprocess.run([exe, "40"], check=True, capture_output=True, text=True).stdout
    v = np.array([[float(x) for x in ln.split()] for ln in out.strip().splitlines()])
    a, b = v[:, 0], v[:, 1]
    assert np.abs(a).max() > 0
    assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [_abi.MODE_FP64_REFERENCE, _abi.MODE_FP64])
def test_shim_plate_matches_oracle(tmp_path, mode):
    exe = build_program(tmp_path)
    out = subprocess.run([exe, "100", str(mode)], check=True, capture_output=True, text=True).stdout
    vals = np.array([[float(x) for x in ln.split()] for ln in out.strip().splitlines()[1:]])
    ekin = float(out.splitlines()[0])
    w = configs.plate_tri3(nx=20, ny=4, lx=1.0, ly=0.2)
    cpu = OracleAdapter(w["mesh"], w["materials"])
    configs.setup_model(cpu, w)
    cpu.solve_steps(100)
    ref = cpu.get(_abi.FIELD_DISPLACEMENT)
    if mode == _abi.MODE_FP64_REFERENCE:
        assert np.array_equal(vals, ref)
    else:
        assert np.abs(vals - ref).max() <= 1e-10 * np.abs(ref).max()
    assert ekin == pytest.approx(cpu.energy(_abi.ENERGY_KINETIC), rel=1e-10)
