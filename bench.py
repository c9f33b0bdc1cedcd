#!/usr/bin/env python3
"""Explicit element-steps/s of the central-difference lumped-mass step.

Workload: the 3D linear-elastic cube of 100^3 cells x 6 tetrahedron_4
(6 000 000 elements, 1 030 301 nodes), E = 70 GPa, nu = 0.33, rho = 2700,
bottom face fixed, top face v_z = 1 m/s, dt = 0.8 x stable, FP64 (the
FP32-bulk form is measured beside it). One step = one solveStep() over the
whole mesh; the metric counts elements x steps per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1). With N > 1 ranks the workload is
one mesh cut over the GPUs: the cube stacked N times along z (bar_tet4), one
100^3 cube per GPU (weak scaling), the forces on the interface planes
exchanged with the neighbouring GPUs every step (grouped NCCL send/recv);
--replicas runs one independent cube per rank instead. Device time is
measured with CUDA events on the model's stream, max over ranks. Prints one
JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from akantu_b200 import _abi, configs  # noqa: E402

METRIC = "explicit element-steps/s"
UNIT = "element-steps/s"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def b_alg_bytes(w, fp32):
    """Compulsory bytes of one step: int32 connectivity, reference
    coordinates, FP64 u/v/a read + write, FP64 inverse mass per node, one
    mask byte per node (f_ext is zero in this workload)."""
    mesh = w["mesh"]
    E, N, n = mesh.getNbElement(), mesh.getNbNodes(), mesh.connectivity.shape[1]
    d = mesh.spatial_dimension
    return E * n * 4 + N * d * (4 if fp32 else 8) + N * d * 8 * 6 + N * 8 + N * 1


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.6)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        # samples under load: the top half of the SM clocks seen
        load = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# --------------------------------------------------------------------------
class Dist:
    def __init__(self, want_gpus):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if os.environ.get("AKB_DIST_BACKEND", "nccl") == "gloo":  # CPU tests of the plumbing
                dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
            else:
                torch.cuda.set_device(self.local_rank)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                        device_id=torch.device("cuda", self.local_rank))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        dev = "cpu" if self.pg.get_backend() == "gloo" else "cuda"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.pg:
            return x
        import torch
        dev = "cpu" if self.pg.get_backend() == "gloo" else "cuda"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def make_model(w, mode, device):
    from akantu_b200.model import SolidMechanicsModel, material_from_dict
    m = SolidMechanicsModel(w["mesh"], [material_from_dict(mm) for mm in w["materials"]],
                            precision=mode, device=device)
    m.initFull()
    return m


class Facade:
    def __init__(self, m):
        self.m = m

    def set(self, f, v):
        self.m.setField(f, v)

    def set_blocked(self, b):
        self.m.setBlockedDOFs(b)

    def stable_time_step(self):
        return self.m.getStableTimeStep()

    def set_time_step(self, dt):
        self.m.setTimeStep(dt)


def reset_state(m, w):
    m.setField(_abi.FIELD_DISPLACEMENT, w["u0"])
    m.setField(_abi.FIELD_VELOCITY, w["v0"])
    m.setField(_abi.FIELD_ACCELERATION, np.zeros_like(w["u0"]))


def time_device(m, w, steps, warmup, dist, sampler=None):
    reset_state(m, w)
    m.solveSteps(warmup)
    reset_state(m, w)
    m.synchronize()
    dist.barrier()
    if sampler:
        sampler.start()
    ms = m.timeSolveSteps(steps)
    clocks = sampler.stop() if sampler else None
    dist.barrier()
    return dist.max(ms), clocks


def time_e2e(m, w, steps, dist):
    """The reference-facing loop through the C ABI with host buffers
    (examples/explicit/explicit_dynamic.cc:87-99): per step applyBC(FixedValue)
    of the fixed face, every component in one call, from pinned host memory,
    solveStep, and the kinetic energy of the step copied to its own pinned
    host slot (queued without a host round trip; every step's value is read
    after the final synchronisation, inside the timed region)."""
    import torch
    from akantu_b200._lib import check, lib
    L = lib()
    d = w["mesh"].spatial_dimension
    fixed = np.nonzero(w["blocked"][:, 0])[0].astype(np.uint32)
    nodes_h = torch.from_numpy(fixed).pin_memory()
    vals_h = torch.zeros(fixed.size * d, dtype=torch.float64).pin_memory()
    energies = torch.zeros(steps, dtype=torch.float64).pin_memory()
    pn = C.cast(nodes_h.data_ptr(), C.POINTER(C.c_uint32))
    pv = C.cast(vals_h.data_ptr(), C.POINTER(C.c_double))
    h = m.handle
    reset_state(m, w)
    m.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for s in range(steps):
        check(L.akb_apply_dirichlet(h, pn, fixed.size, _abi.ALL_COMPONENTS, pv))
        check(L.akb_solve_step(h))
        check(L.akb_get_energy_async(h, _abi.ENERGY_KINETIC,
                                     C.c_void_p(energies.data_ptr() + 8 * s)))
    check(L.akb_synchronize(h))
    ek = energies.numpy().copy()  # every step's kinetic energy on the host
    t1 = time.perf_counter()
    dist.barrier()
    assert np.all(np.isfinite(ek)) and ek[-1] > 0
    h2d = fixed.size * (4 + 8 * d)
    return dist.max(t1 - t0), h2d, 8


def kernel_times(m, steps):
    from akantu_b200._lib import check, lib
    L = lib()
    out = (C.c_double * _abi_max_slots())()
    check(L.akb_time_kernels(m.handle, steps, out, _abi_max_slots()))
    names = [L.akb_kernel_name(m.handle, k).decode() for k in range(_abi_max_slots())]
    return [(n, out[k]) for k, n in enumerate(names) if n]


def _abi_max_slots():
    return 8


def cpu_baseline(w, seconds_target=15.0):
    """The oracle (FP64 CPU restatement, OpenMP, bitwise equal to the serial
    reference order) on this host's cores, bounded sample of the workload."""
    from oracle.oracle import OracleModel, material_desc
    threads = os.cpu_count() or 1
    m = OracleModel(w["mesh"], [material_desc(**mm) for mm in w["materials"]], fast=True)
    m.set_threads(threads)
    m.blocked[...] = w["blocked"]
    m.displacement[...] = w["u0"]
    m.velocity[...] = w["v0"]
    m.set_time_step(w["dt_factor"] * m.stable_time_step())
    t1 = m.time_steps(1)
    steps = int(max(1, min(50, seconds_target / max(t1, 1e-6))))
    t = m.time_steps(steps)
    E = w["mesh"].getNbElement()
    return dict(value=E * steps / t, unit=UNIT, cores=threads, kind="port",
                sample="%d steps of the full %d-element mesh after 1 warm-up step "
                       "(FP64 CPU restatement, OpenMP)" % (steps, E))


def run_ours(args, dist):
    import torch
    device = dist.local_rank
    torch.cuda.set_device(device)
    w = configs.cube_tet4(args.cells)
    E = w["mesh"].getNbElement()
    peak, peak_kind = load_peaks()
    m = make_model(w, _abi.MODE_FP64, device)
    dt = configs.setup_model(Facade(m), w)
    sampler = ClockSampler(device)
    ms, clocks = time_device(m, w, args.steps, args.warmup, dist, sampler)
    value = dist.world * E * args.steps / (ms / 1e3)
    ktimes = kernel_times(m, min(args.steps, 50))
    step_ms = sum(t for _, t in ktimes)
    top = max(ktimes, key=lambda kv: kv[1])
    balg = b_alg_bytes(w, False)
    e2e_steps = min(args.steps, 200)
    e2e_s, h2d, d2h = time_e2e(m, w, e2e_steps, dist)
    e2e_value = dist.world * E * e2e_steps / e2e_s
    u64 = m.getDisplacement().copy() if dist.rank == 0 else None
    # FP32-bulk beside it, error vs the FP64 GPU run after the same steps
    m32 = make_model(w, _abi.MODE_FP32_BULK, device)
    configs.setup_model(Facade(m32), w)
    m32.setTimeStep(dt)
    ms32, _ = time_device(m32, w, args.steps, args.warmup, dist)
    fp32 = dict(value=dist.world * E * args.steps / (ms32 / 1e3),
                ms_per_step=ms32 / args.steps,
                roofline_frac=(b_alg_bytes(w, True) / (ms32 / args.steps / 1e3) / 1e9) / peak)
    if dist.rank == 0:
        # same K steps from the same state in both precisions
        reset_state(m, w)
        m.solveSteps(args.steps)
        reset_state(m32, w)
        m32.solveSteps(args.steps)
        u64 = m.getDisplacement().copy()
        u32 = m32.getDisplacement()
        fp32["rel_err_displacement_vs_fp64"] = float(np.abs(u32 - u64).max() / np.abs(u64).max())
    m32.close()
    parity = None
    if dist.rank == 0:
        # full-size parity: the same K steps in the reference-order GPU mode
        # (the reference's operation order, bitwise equal to the oracle on
        # the sizes the oracle runs) against the fused FP64 step
        mref = make_model(w, _abi.MODE_FP64_REFERENCE, device)
        configs.setup_model(Facade(mref), w)
        mref.setTimeStep(dt)
        reset_state(mref, w)
        mref.solveSteps(args.steps)
        uref = mref.getDisplacement()
        vref = mref.getVelocity()
        mref.close()
        v64 = m.getVelocity()
        parity = {"steps": args.steps, "reference": "AKB_MODE_FP64_REFERENCE on the GPU",
                  "rel_err_displacement": float(np.abs(u64 - uref).max() / np.abs(uref).max()),
                  "rel_err_velocity": float(np.abs(v64 - vref).max() / np.abs(vref).max())}
    launches = args.steps * len(ktimes)
    result = None
    if dist.rank == 0:
        achieved = balg / (step_ms / 1e3) / 1e9
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "cube_tet4: %d^3 cells x 6 tetrahedron_4 (%d elements, "
                                   "%d nodes), linear elastic, FP64, dt = 0.8 x stable"
                                   % (args.cells, E, w["mesh"].getNbNodes()), "elements": E,
                       "nodes": w["mesh"].getNbNodes(), "time_step": dt,
                       "parallelism": "replicas" if dist.world > 1 else "single GPU",
                       "l2": "no flush: per-step working set %.0f MB > 126 MB L2" % (balg / 1e6)},
            "roofline": {"bound": "hbm", "kernel": "whole step (%s)" % ", ".join(n for n, _ in ktimes),
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_step": balg,
                         # DRAM bytes of one k_patch_step launch from an ncu capture
                         # (dram__bytes_read.sum + dram__bytes_write.sum) of the
                         # 90^3-cell cube (4.374 M elements, 232.7 MB), scaled by
                         # elements; the capture is not taken inside this run
                         "traffic": 232.7e6 * E / 4.374e6,
                         "traffic_kernel": "k_patch_step (ncu, 90^3 cells, scaled by elements)",
                         "kernels_ms": {n: t for n, t in ktimes},
                         "dominant": top[0]},
            "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "gpu_launches": launches,
            "fp32_bulk": fp32,
            "fp64_vs_reference_order": parity,
        }
    m.close()
    return result


def run_decomposed(args, dist):
    """bar_tet4: the headline cube stacked N times along z as ONE mesh (N =
    ranks x --parts-per-rank), cut into its cubes, parts_per_rank slabs per
    GPU, each slab the 100^3 x 6 cube (weak scaling: the work per GPU is the
    headline's). Per step each part runs the fused step, packs the forces on
    its interface planes, exchanges them with its neighbours only (grouped
    NCCL send/recv on the step's stream, a copy between parts of one GPU),
    and finishes the planes with the sums in part order."""
    import torch
    from akantu_b200._lib import check, lib
    from akantu_b200.decompose import DistributedModel
    device = dist.local_rank
    torch.cuda.set_device(device)
    ppr = max(1, args.parts_per_rank)
    nslabs = dist.world * ppr
    here = list(range(dist.rank * ppr, (dist.rank + 1) * ppr))
    s = configs.bar_tet4_slabs(args.cells, nslabs, here)
    peak, peak_kind = load_peaks()
    dm = DistributedModel(None, s["materials"], nslabs, precision=_abi.MODE_FP64, device=device,
                          parts=s["parts"], nb_nodes=s["nb_nodes"], group=None)
    E_part = s["parts"][0].mesh.getNbElement()
    E = E_part * nslabs

    def reset():
        dm.set_blocked(s["blocked"])
        dm.set_field(_abi.FIELD_DISPLACEMENT, s["u0"])
        dm.set_field(_abi.FIELD_VELOCITY, s["v0"])
        dm.set_field(_abi.FIELD_ACCELERATION, np.zeros_like(s["u0"]))

    reset()
    dt = s["dt_factor"] * dm.stable_time_step()
    dm.set_time_step(dt)
    dm.solve_steps(args.warmup)
    reset()
    sampler = ClockSampler(device)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler.start()
    e0.record()
    dm.solve_steps(args.steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    dist.barrier()
    ms = dist.max(e0.elapsed_time(e1))
    # e2e through the C ABI with host buffers: per step the bottom face's
    # Dirichlet values (all components, one call, on the part holding it)
    # from pinned memory, the step, and each part's kinetic energy queued
    # into its own pinned slot; read after the final synchronisation
    L = lib()
    e2e_steps = min(args.steps, 200)
    fixed_g = np.nonzero(s["blocked"][:, 0])[0]
    bcs = []
    for p, b in zip(dm.parts, dm.backends):
        loc = np.searchsorted(p.nodes, fixed_g)
        loc = loc[(loc < len(p.nodes)) & (p.nodes[np.minimum(loc, len(p.nodes) - 1)] == fixed_g)]
        if len(loc):
            nh = torch.from_numpy(loc.astype(np.uint32)).pin_memory()
            vh = torch.zeros(len(loc) * 3, dtype=torch.float64).pin_memory()
            bcs.append((b.m.handle, nh, vh, len(loc)))
    energies = torch.zeros((e2e_steps, len(dm.backends)), dtype=torch.float64).pin_memory()
    reset()
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        for h, nh, vh, n in bcs:
            check(L.akb_apply_dirichlet(h, C.cast(nh.data_ptr(), C.POINTER(C.c_uint32)), n,
                                        _abi.ALL_COMPONENTS,
                                        C.cast(vh.data_ptr(), C.POINTER(C.c_double))))
        dm.solve_step()
        for j, b in enumerate(dm.backends):
            check(L.akb_get_energy_async(b.m.handle, _abi.ENERGY_KINETIC,
                                         C.c_void_p(energies.data_ptr() + 8 * (k * len(dm.backends) + j))))
    for b in dm.backends:
        check(L.akb_synchronize(b.m.handle))
    ek = energies.numpy().sum(axis=1)
    t1 = time.perf_counter()
    dist.barrier()
    assert np.all(np.isfinite(ek))
    e2e_s = dist.max(t1 - t0)
    h2d = int(dist.sum(float(sum(n * (4 + 24) for _, _, _, n in bcs))))
    d2h = 8 * nslabs
    nbytes = dist.sum(float(dm.bytes_per_step))
    balg = b_alg_bytes({"mesh": s["parts"][0].mesh}, False) * ppr
    # per step and part: the fused step, the pack (rows to send), the ordered
    # sums (interface rows), the shared-node pass
    launches = int(dist.sum(float(sum(2 + (x.n_send > 0) + (x.sum_ptr.size > 1)
                                      for x in dm.plans))))
    dm.close()
    if dist.rank != 0:
        return None
    achieved = balg / (ms / args.steps / 1e3) / 1e9
    n = args.cells
    return {"metric": METRIC, "value": E * args.steps / (ms / 1e3), "unit": UNIT,
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "bar_tet4: %d x %d x %d cells x 6 tetrahedron_4 (%d elements, "
                                   "%d nodes), linear elastic, FP64, dt = 0.8 x stable"
                                   % (n, n, n * nslabs, E, s["nb_nodes"]),
                       "elements": E, "time_step": dt,
                       "parallelism": "one mesh cut into %d cubes along z, %d per GPU; "
                                      "neighbour exchange of the interface planes" % (nslabs, ppr),
                       "exchange_bytes_per_step": nbytes,
                       "l2": "no flush: per-GPU working set %.0f MB > 126 MB L2" % (balg / 1e6)},
            "roofline": {"bound": "hbm", "kernel": "whole step per GPU (fused step, pack, "
                                                   "exchange, interface sums, k_finish_list)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_step": balg, "traffic": None},
            "clocks": clocks,
            "e2e": {"value": E * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "gpu_launches": args.steps * launches}


def run_plate(args, device):
    """The reference's CPU-runnable configuration: the 200 x 20 triangle_3
    plate (8000 elements), 1000 steps, FP64, in all three modes, against the
    single-thread FP64 oracle on the same steps (a launch-bound size on the
    GPU: CUDA-graph replays of 32-step chunks)."""
    from akantu_b200.model import material_from_dict
    from oracle.oracle import OracleModel, material_desc
    w = configs.plate_tri3()
    E = w["mesh"].getNbElement()
    out = {"workload": "plate_tri3: 200 x 20 squares x 2 triangle_3 (%d elements), 1000 steps" % E}
    cpu = OracleModel(w["mesh"], [material_desc(**mm) for mm in w["materials"]])
    cpu.blocked[...] = w["blocked"]
    cpu.displacement[...] = w["u0"]
    dt = w["dt_factor"] * cpu.stable_time_step()
    cpu.set_time_step(dt)
    t = cpu.time_steps(w["steps"])
    out["cpu_oracle_1_thread"] = {"value": E * w["steps"] / t, "unit": UNIT, "s": t}
    ref = cpu.displacement.copy()
    from akantu_b200.model import SolidMechanicsModel
    for mode, name in ((_abi.MODE_FP64_REFERENCE, "fp64_reference"), (_abi.MODE_FP64, "fp64"),
                       (_abi.MODE_FP32_BULK, "fp32_bulk")):
        m = SolidMechanicsModel(w["mesh"], [material_from_dict(mm) for mm in w["materials"]],
                                precision=mode, device=device)
        m.initFull()
        m.setBlockedDOFs(w["blocked"])
        m.setField(_abi.FIELD_DISPLACEMENT, w["u0"])
        m.setTimeStep(dt)
        ms = m.timeSolveSteps(w["steps"])
        u = m.getDisplacement()
        out[name] = {"value": E * w["steps"] / (ms / 1e3), "unit": UNIT, "ms": ms,
                     "rel_err_displacement_vs_oracle":
                         float(np.abs(u - ref).max() / np.abs(ref).max())}
        m.close()
    return out


def run_hex8(args, device, peak):
    """3D finite-strain neo-Hookean block, 128^3 hexahedron_8 (2 097 152
    elements), FP32 element arithmetic with FP64 nodal state, against the
    FP64 GPU run of the same steps (the FP64 CPU oracle at this size would
    take hours; the small-size parity tests compare both to the oracle)."""
    w = configs.block_hex8(args.hex_cells, 0.01 * args.hex_cells)
    E = w["mesh"].getNbElement()
    steps = w["steps"] if args.hex_steps <= 0 else args.hex_steps
    out = {"workload": "block_hex8: %d^3 hexahedron_8, 2x2x2 Gauss, neo-Hookean lambda = 1 MPa, "
                       "mu = 0.4 MPa, rho = 1100, face x = 0 fixed, v ~ N(0, 0.05)" % args.hex_cells,
           "elements": E, "steps": steps}
    states = {}
    modes = [(n, md) for n, md in (("fp32_bulk", _abi.MODE_FP32_BULK), ("fp64", _abi.MODE_FP64))
             if n in args.hex_modes.split(",")]
    for name, mode in modes:
        m = make_model(w, mode, device)
        dt = configs.setup_model(Facade(m), w)
        m.solveSteps(3)
        reset_state(m, w)
        ms = m.timeSolveSteps(steps)
        fb = b_alg_bytes(w, mode == _abi.MODE_FP32_BULK)
        states[name] = (m.getDisplacement().copy(), m.getInternalForce().copy())
        out[name] = {"value": E * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
                     "hbm_roofline_frac": fb / (ms / steps / 1e3) / 1e9 / peak,
                     "kernels_ms": dict(kernel_times(m, 10))}
        m.close()
    if len(states) == 2:
        (u32, f32), (u64, f64) = states["fp32_bulk"], states["fp64"]
        out["fp32_vs_fp64"] = {
            "rel_err_displacement": float(np.abs(u32 - u64).max() / np.abs(u64).max()),
            "rel_err_internal_force": float(np.abs(f32 - f64).max() / np.abs(f64).max())}
    out["time_step"] = dt
    # compute roofline of the FP64 launch, from an ncu capture of this
    # workload (sm__inst_executed_pipe_fp64, % of peak; not taken in this run)
    out["compute_roofline"] = {"bound": "fp64 pipe (FP64) / fma pipe (FP32-bulk)",
                               "fp64_pipe_active": 0.445, "fp32_bulk_fma_pipe_active": 0.413,
                               "kernel": "k_patch_step<hex8, double> / <hex8, float>",
                               "source": "ncu captures of the 96^3 block "
                                         "(profiles/k_patch_step_block_hex8_96.md)"}
    return out


def batch_alg_bytes(meshes):
    """b_alg_bytes over the instances of a batch (their union)."""
    E = sum(m.getNbElement() for m in meshes)
    N = sum(m.getNbNodes() for m in meshes)
    n, d = meshes[0].connectivity.shape[1], meshes[0].spatial_dimension
    return E * n * 4 + N * d * 8 + N * d * 8 * 6 + N * 8 + N * 1


def run_batch(args, device, log=None):
    """4096 triangle_3 plates of uneven size in one batch (one fused launch
    per step, CUDA-graph replay, autotuned patch shape and schedule), and the
    same plates as separate models on a sample of instances."""
    from akantu_b200 import autotune
    from akantu_b200.batch import BatchModel
    w = configs.plates_batch(args.batch_instances)
    E = sum(m.getNbElement() for m in w["meshes"])
    steps = w["steps"] if args.batch_steps <= 0 else args.batch_steps
    # tune on a sample of the instances, then build the whole batch
    rng = np.random.default_rng(1)
    sample = sorted(rng.choice(len(w["meshes"]), size=min(256, len(w["meshes"])), replace=False))
    ws = {k: ([w[k][i] for i in sample] if isinstance(w[k], list) else w[k]) for k in w}

    def build(pe, pn, grid, ww=ws):
        b = BatchModel(ww["meshes"], ww["materials"], precision=_abi.MODE_FP64, device=device,
                       patch_elements=pe, patch_nodes=pn, patch_grid=grid)
        b.initFull()
        configs.setup_batch(b, ww)
        return b
    best, trials = autotune.tune(build, _abi.TRIANGLE_3, _abi.MODE_FP64,
                                 sum(m.getNbElement() for m in ws["meshes"]) * len(w["meshes"]) // len(sample),
                                 log=log)
    b = build(best["patch_elements"], best["patch_nodes"], best["patch_grid"], w)
    b.solveSteps(3)
    configs.setup_batch(b, w)
    ms = b.timeSolveSteps(steps)
    balg = batch_alg_bytes(w["meshes"])
    peak, peak_kind = load_peaks()
    achieved = balg / (ms / steps / 1e3) / 1e9
    out = {"workload": "%d triangle_3 plates, %d elements, %d nodes, per-plate E, nu, rho, dt"
                       % (len(w["meshes"]), E, int(b.node_offsets[-1])),
           "elements": E, "steps": steps,
           "batched": {"value": E * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
                       "launches_per_step": len(kernel_times(b, 5)), "tuned": best,
                       "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                                    "unit": "GB/s", "frac": achieved / peak,
                                    "peak_source": peak_kind,
                                    "algorithmic_bytes_per_step": balg},
                       "trials_ms_per_step": [[t[0], t[1]] for t in trials]}}
    b.close()
    # the same sample as separate models (one model per plate, graph replays)
    sub_steps = 20
    models = []
    for i in sample:
        m = SolidMechanicsModel_for(w, i, device, best)
        models.append(m)
    import torch
    for m in models:  # instantiates each model's graph outside the timed loop
        m.solveSteps(sub_steps)
    for m in models:
        m.synchronize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for m in models:
        m.solveSteps(sub_steps)
    for m in models:
        m.synchronize()
    t1 = time.perf_counter()
    Es = sum(w["meshes"][i].getNbElement() for i in sample)
    bs = build(best["patch_elements"], best["patch_nodes"], best["patch_grid"], ws)
    bs.solveSteps(2 * sub_steps)
    ub = bs.getField(_abi.FIELD_DISPLACEMENT)
    same = all(np.array_equal(ub[bs.instance_rows(j)], m.getDisplacement())
               for j, m in enumerate(models))
    msb = bs.timeSolveSteps(sub_steps)
    out["per_mesh_sample"] = {"instances": len(sample), "elements": Es, "steps": sub_steps,
                              "per_mesh_value": Es * sub_steps / (t1 - t0),
                              "batched_value": Es * sub_steps / (msb / 1e3),
                              "bitwise_equal_to_batched": bool(same), "unit": UNIT}
    for m in models:
        m.close()
    bs.close()
    return out


def mlp_inference(net, nq, reps=20):
    """Surrogate inference on nq Gauss points (seeded gradients of the FE^2
    envelope): the network kernel on ready features, the torch feature path
    around it, and the macro step's fused form (features, network, |H|
    rescale and envelope list in one launch, akb_mlp_stress); CUDA events,
    best of three runs of `reps` calls."""
    import torch
    from akantu_b200 import fe2
    from akantu_b200.surrogate import scaled_features
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn):
        a, b = ev(), ev()
        torch.cuda.synchronize()
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    Hq = torch.as_tensor(fe2.sample_gradients(nq, seed=9), device="cuda")
    Xq = Hq.transpose(1, 2).reshape(-1, 9).contiguous()
    xq, _ = scaled_features(Xq)
    Pq = torch.empty_like(Xq)
    fb = (torch.empty(nq, dtype=torch.int32, device="cuda"),
          torch.zeros(1, dtype=torch.int32, device="cuda"))
    for _ in range(5):  # warm every path (allocator, clocks)
        net.forward_features(xq)
        net.predict_flat(Xq)
        net.stress_into(Xq, Pq, envelope=(0.3, 0.5), fallback=fb)
    ms_k = min(timed(lambda: [net.forward_features(xq) for _ in range(reps)]) for _ in range(3))
    ms_e = min(timed(lambda: [net.predict_flat(Xq) for _ in range(reps)]) for _ in range(3))
    ms_f = min(timed(lambda: [net.stress_into(Xq, Pq, envelope=(0.3, 0.5), fallback=fb)
                              for _ in range(reps)]) for _ in range(3))
    flop = 2 * sum(max(k, 16) * max(n, 16) for k, n in net.layer_shapes())
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak = float(json.load(fh)["bf16_tflops"])
    except Exception:
        peak = 1590.0
    tf = flop * nq / (ms_k / reps * 1e-3) / 1e12
    return {"samples": nq, "kernel_ms": ms_k / reps, "with_features_ms": ms_e / reps,
            "fused_stress_ms": ms_f / reps, "tflops": tf, "flop_per_sample": flop,
            "tensor_roofline_frac": tf / peak, "peak_tflops": peak}


def run_mlp(args, device):
    """The surrogate's inference alone (akantu_b200/data/rve_surrogate.npz) on one macro
    step's 262 144 Gauss points."""
    from akantu_b200.surrogate import MLPSurrogate
    net = MLPSurrogate.load(os.path.join(ROOT, "akantu_b200", "data", "rve_surrogate.npz"),
                            device=device)
    return mlp_inference(net, 8 * args.fe2_cells ** 3)


def run_fe2(args, device, log=None):
    """FE^2 of a 32^3 hexahedron_8 block with a 16^3 periodic RVE at each of its
    262 144 Gauss points: the learned surrogate against held-out RVE solves,
    the learned and the plain (RVE) macro step times, and the macro
    displacement of a learned run against a plain run on a coarser block."""
    import torch
    from akantu_b200 import fe2
    from akantu_b200.surrogate import MLPSurrogate
    rve, mats, vf = fe2.spec_rve(16)
    frac = [1 - vf, vf]
    out = {"workload": "macro %d^3 hexahedron_8 (%d Gauss points), RVE 16^3 voxels, sphere "
                       "voxel fraction %.4f, neo-Hookean matrix lambda 1 MPa mu 0.4 MPa, "
                       "inclusion x10; stretch 5%% over %d steps"
                       % (args.fe2_cells, 8 * args.fe2_cells ** 3, vf, args.fe2_ramp)}
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn):
        a, b = ev(), ev()
        torch.cuda.synchronize()
        a.record()
        r = fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b), r

    # RVE solves: held-out samples (another seed than the training set's)
    ms, (Xh, Yh, it, _) = timed(lambda: fe2.generate_dataset(rve, args.fe2_heldout, seed=7))
    out["rve"] = {"solves": args.fe2_heldout, "ms": ms,
                  "solves_per_s": args.fe2_heldout / ms * 1e3,
                  "mean_iterations": float(it.float().mean()),
                  "shared_bytes_per_solve": rve.shared_bytes}
    path = os.path.join(ROOT, "akantu_b200", "data", "rve_surrogate.npz")
    if not os.path.exists(path):
        out["surrogate"] = "no trained weights (run python -m akantu_b200.train_surrogate)"
        return out
    net = MLPSurrogate.load(path, device=device)
    Xs, Ys, _, rs = fe2.generate_dataset(rve, args.fe2_heldout, seed=8, small=True)
    ok = torch.isfinite(rs) & (rs <= 1e-3)
    out["surrogate"] = {"heldout_error": fe2.surrogate_error(net, Xh, Yh),
                        "heldout_error_small_strain": fe2.surrogate_error(net, Xs[ok], Ys[ok])}
    # inference throughput over one macro step's Gauss points
    nq = 8 * args.fe2_cells ** 3
    out["surrogate"]["inference"] = mlp_inference(net, nq)

    # learned FE^2: the whole ramp on the full block
    learned = fe2.MaterialFE2(rve, surrogate=net)
    m = fe2.macro_block(learned.material(mats, frac), cells=args.fe2_cells)
    dt = 0.8 * m.getStableTimeStep()
    m.setTimeStep(dt)
    step_ms = []
    for s in range(1, args.fe2_ramp + 1):
        ms, _ = timed(lambda: fe2.macro_step(m, s, ramp_steps=args.fe2_ramp))
        step_ms.append(ms)
    learned_ms = float(np.median(step_ms[5:]))
    u_learned = m.getDisplacement().copy()
    out["learned_step"] = {"ms_median": learned_ms, "steps": args.fe2_ramp,
                           "fallback_points": learned.stats["fallback"], "time_step": dt}
    # plain FE^2 step at the end state: every Gauss point relaxes its RVE,
    # first from zero fluctuations, then warm-started from the previous step
    learned.surrogate = None
    ms_cold, _ = timed(lambda: fe2.macro_step(m, args.fe2_ramp + 1, ramp_steps=args.fe2_ramp))
    it_cold = learned.stats["iterations"]
    ms_warm, _ = timed(lambda: fe2.macro_step(m, args.fe2_ramp + 2, ramp_steps=args.fe2_ramp))
    out["plain_step"] = {"ms_cold_start": ms_cold, "ms_warm_start": ms_warm,
                         "rve_solves_per_step": nq,
                         "mean_iterations_cold": it_cold / nq,
                         "mean_iterations_warm": (learned.stats["iterations"] - it_cold) / nq}
    out["speedup_learned_vs_plain"] = {"cold": ms_cold / learned_ms, "warm": ms_warm / learned_ms}
    m.close()
    if log:
        log("fe2: learned %.3f ms/step, plain %.1f / %.1f ms" % (learned_ms, ms_cold, ms_warm))
    # macro displacement error: learned vs plain FE^2 over the whole ramp on a
    # coarser block (a plain run of the full block is 200 x the plain step)
    us = {}
    for name, sur in (("plain", None), ("learned", net)):
        prov = fe2.MaterialFE2(rve, surrogate=sur)
        mm = fe2.macro_block(prov.material(mats, frac), cells=args.fe2_check_cells)
        mm.setTimeStep(0.8 * mm.getStableTimeStep())
        ms, _ = timed(lambda: [fe2.macro_step(mm, s, ramp_steps=args.fe2_ramp)
                               for s in range(1, args.fe2_ramp + 1)])
        us[name] = (mm.getDisplacement().copy(), ms)
        mm.close()
    (up, msp), (ul, msl) = us["plain"], us["learned"]
    out["displacement_check"] = {
        "cells": args.fe2_check_cells, "steps": args.fe2_ramp,
        "rel_err_displacement": float(np.abs(ul - up).max() / np.abs(up).max()),
        "plain_run_s": msp / 1e3, "learned_run_s": msl / 1e3}
    out["learned_full_run_max_ux"] = float(np.abs(u_learned[:, 0]).max())
    return out


def run_batch_sharded(args, dist):
    """The 4096-plate batch split over the ranks by element count (no
    collective in the step; device time max over ranks). Every rank calls
    this; rank 0 returns the result."""
    from akantu_b200.batch import BatchModel, partition_instances
    w = configs.plates_batch(args.batch_instances)
    sizes = [m.getNbElement() for m in w["meshes"]]
    mine = partition_instances(sizes, dist.world)[dist.rank]
    ws = {k: ([w[k][i] for i in mine] if isinstance(w[k], list) else w[k]) for k in w}
    steps = w["steps"] if args.batch_steps <= 0 else args.batch_steps
    b = BatchModel(ws["meshes"], ws["materials"], precision=_abi.MODE_FP64,
                   device=dist.local_rank, patch_elements=768, patch_nodes=480)
    b.initFull()
    configs.setup_batch(b, ws)
    b.solveSteps(3)
    configs.setup_batch(b, ws)
    b.synchronize()
    dist.barrier()
    ms = dist.max(b.timeSolveSteps(steps))
    dist.barrier()
    b.close()
    E = float(sum(sizes))
    return {"workload": "%d triangle_3 plates over %d ranks (elements per rank balanced)"
                        % (len(sizes), dist.world),
            "elements": E, "steps": steps, "value": E * steps / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / steps, "scaling": "strong",
            "elements_rank0": float(sum(sizes[i] for i in mine))}


def SolidMechanicsModel_for(w, i, device, opts):
    from akantu_b200.model import SolidMechanicsModel, material_from_dict
    m = SolidMechanicsModel(w["meshes"][i], [material_from_dict(w["materials"][i])],
                            precision=_abi.MODE_FP64, device=device,
                            patch_elements=opts["patch_elements"], patch_nodes=opts["patch_nodes"])
    m.initFull()
    m.setBlockedDOFs(w["blocked"][i])
    m.setField(_abi.FIELD_DISPLACEMENT, w["u0"][i])
    m.setTimeStep(w["dt_factor"] * m.getStableTimeStep())
    return m


def run_reference(args, dist):
    if dist.rank != 0:
        return None
    w = configs.cube_tet4(args.cells)
    from oracle.oracle import OracleModel, material_desc
    threads = os.cpu_count() or 1
    m = OracleModel(w["mesh"], [material_desc(**mm) for mm in w["materials"]], fast=True)
    m.set_threads(threads)
    m.blocked[...] = w["blocked"]
    m.velocity[...] = w["v0"]
    dt = w["dt_factor"] * m.stable_time_step()
    m.set_time_step(dt)
    warm = args.warmup  # at least 3 (main raises W to 3)
    m.time_steps(warm)
    steps = min(args.steps, 40)
    t = m.time_steps(steps)
    E = w["mesh"].getNbElement()
    N = w["mesh"].getNbNodes()
    c = args.cells
    value = E * steps / t
    if dist.world > 1:  # our arm: the cube stacked once per GPU as one mesh
        workload = ("bar_tet4: %d x %d x %d cells x 6 tetrahedron_4 (%d elements, %d nodes), "
                    "linear elastic, FP64, dt = 0.8 x stable"
                    % (c, c, c * dist.world, E * dist.world, (c + 1) ** 2 * (c * dist.world + 1)))
        sample = ("%d of the requested %d steps on one of the bar's %d cubes (%d "
                  "elements; every cube has the same CPU rate per element-step; the "
                  "reference cannot be built: Boost is absent)"
                  % (steps, args.steps, dist.world, E))
    else:
        workload = ("cube_tet4: %d^3 cells x 6 tetrahedron_4 (%d elements, %d nodes), "
                    "linear elastic, FP64, dt = 0.8 x stable" % (c, E, N))
        sample = ("%d of the requested %d steps on the full mesh (the reference cannot be "
                  "built: Boost is absent)" % (steps, args.steps))
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": steps, "warmup": warm, "ms_per_step": t / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": workload, "elements": E, "time_step": dt},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cells", type=int, default=100,
                    help="cells per cube side (100 = the benchmark; smaller for profiling)")
    ap.add_argument("--only-headline", action="store_true",
                    help="skip the hexahedron and batch workloads")
    ap.add_argument("--hex-cells", type=int, default=128)
    ap.add_argument("--hex-steps", type=int, default=0, help="0 = the workload's 2000 steps")
    ap.add_argument("--hex-modes", default="fp32_bulk,fp64",
                    help="precisions of the hexahedron workload (profiling one alone)")
    ap.add_argument("--batch-instances", type=int, default=4096)
    ap.add_argument("--batch-steps", type=int, default=0, help="0 = the workload's 500 steps")
    ap.add_argument("--fe2-cells", type=int, default=32)
    ap.add_argument("--fe2-ramp", type=int, default=200)
    ap.add_argument("--fe2-heldout", type=int, default=4096)
    ap.add_argument("--fe2-check-cells", type=int, default=8)
    ap.add_argument("--no-fe2", action="store_true")
    ap.add_argument("--decompose", action="store_true",
                    help="one mesh cut over the ranks (the default with several ranks): the "
                         "headline cube stacked once per part along z, one part per GPU")
    ap.add_argument("--replicas", action="store_true",
                    help="with several ranks, one independent headline cube per rank instead")
    ap.add_argument("--parts-per-rank", type=int, default=1)
    ap.add_argument("--workload", default="",
                    choices=["", "plate_tri3", "block_hex8", "plates_batch", "fe2", "mlp"],
                    help="run only this secondary workload (1 GPU) and print its result")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return

        class _D:
            pass
        d = _D()
        d.rank, d.world = rank, world
        res = run_reference(args, d)
        print(json.dumps(res), flush=True)
        return
    if args.workload:  # one secondary workload alone, for profiling
        import torch
        torch.cuda.set_device(0)
        peak, _ = load_peaks()
        fn = {"plate_tri3": lambda: run_plate(args, 0), "block_hex8": lambda: run_hex8(args, 0, peak),
              "plates_batch": lambda: run_batch(args, 0),
              "fe2": lambda: run_fe2(args, 0, log=lambda s: print(s, file=sys.stderr, flush=True)),
              "mlp": lambda: run_mlp(args, 0)}[args.workload]
        print(json.dumps({"workloads": {args.workload: fn()}}), flush=True)
        return
    dist = Dist(args.gpus)
    if args.decompose or (dist.world > 1 and not args.replicas):
        try:
            res = run_decomposed(args, dist)
            if dist.world > 1 and not args.only_headline:
                sharded = run_batch_sharded(args, dist)  # every rank takes part
                if dist.rank == 0:
                    res["workloads"] = {"plates_batch_sharded": sharded}
            if dist.rank == 0:
                print(json.dumps(res), flush=True)
        finally:
            dist.close()
        return
    try:
        res = run_ours(args, dist)
        if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(configs.cube_tet4(args.cells))
        if dist.world > 1 and not args.only_headline:
            sharded = run_batch_sharded(args, dist)  # every rank takes part
            if dist.rank == 0:
                res["workloads"] = {"plates_batch_sharded": sharded}
        elif dist.rank == 0 and not args.only_headline:
            peak, _ = load_peaks()
            res["workloads"] = {
                "plate_tri3": run_plate(args, dist.local_rank),
                "block_hex8": run_hex8(args, dist.local_rank, peak),
                "plates_batch": run_batch(args, dist.local_rank,
                                          log=lambda s: print(s, file=sys.stderr, flush=True)),
            }
            if not args.no_fe2:
                res["workloads"]["fe2"] = run_fe2(
                    args, dist.local_rank, log=lambda s: print(s, file=sys.stderr, flush=True))
        if dist.rank == 0:
            print(json.dumps(res), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
