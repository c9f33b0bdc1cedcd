"""The partitioned-mesh path on CPU: the partition and the parts it builds,
and the interface exchange (mass once, forces every step) driven by
akantu_b200.decompose.DistributedModel, with the FP64 CPU oracle standing in
for each part's GPU model. A mesh cut into 2 or 3 parts, in one process and
over two gloo ranks, must step like the whole mesh in one oracle model
(<= 1e-11 relative after 60 steps: the interface sums are added in another
order)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from akantu_b200 import _abi, configs
from akantu_b200.decompose import DistributedModel, build_parts, partition_elements

STEPS = 60


def _workload(n=6):
    w = configs.cube_tet4(n=n)
    rng = np.random.default_rng(7)
    v0 = w["v0"] + rng.normal(0.0, 0.1, w["v0"].shape)
    v0[w["blocked"].astype(bool)] = 0.0
    w["v0"] = v0
    return w


class OraclePart:
    """One part stepped by the CPU oracle with the split step of a GPU part:
    predictor and internal forces (begin), the interface forces out, the
    summed forces in, lumped solve and corrector (end)."""
    device = torch.device("cpu")

    def __init__(self, part, materials):
        from oracle.oracle import OracleModel, material_desc
        self.o = OracleModel(part.mesh, [material_desc(**mm) for mm in materials])
        self.o.assemble_mass_lumped()
        self.iface = part.iface_local.astype(np.int64)
        self.dt = None

    def begin(self):
        o, dt = self.o, self.dt
        free = o.blocked == 0
        u, v, a = o.displacement, o.velocity, o.acceleration
        dta = dt * a
        u[free] = (u + (dt * v + (0.5 * dt) * dta))[free]
        v[free] = (v + dta)[free]
        o.assemble_internal_forces()
        self.f = o.internal_force.copy()

    def export_forces(self, out):
        out.copy_(torch.from_numpy(self.f[self.iface]))

    def end(self, total):
        o, dt = self.o, self.dt
        self.f[self.iface] = total.numpy()
        free = o.blocked == 0
        r = (o.external_force + self.f) + o.mass * (-o.acceleration)
        x = r / o.mass
        o.velocity[free] = (o.velocity + (0.5 * dt) * x)[free]
        o.acceleration[free] = (o.acceleration + x)[free]

    def export_mass(self, out):
        out.copy_(torch.from_numpy(self.o.mass[self.iface, 0].copy()))

    def import_mass(self, total):
        self.o.mass[self.iface, :] = total.numpy()[:, None]

    def stable_time_step(self):
        return self.o.stable_time_step()

    def set_time_step(self, dt):
        self.dt = dt
        self.o.set_time_step(dt)

    def set_field(self, field, values):
        self.o.field(field)[...] = values

    def get_field(self, field):
        return self.o.field(field).copy()

    def set_blocked(self, blocked):
        self.o.blocked[...] = blocked


def _run_distributed(w, nparts, here=None, group=None):
    dm = DistributedModel(w["mesh"], w["materials"], nparts, here=here, group=group,
                          backend=lambda p: OraclePart(p, w["materials"]))
    dm.set_blocked(w["blocked"])
    dm.set_field(_abi.FIELD_DISPLACEMENT, w["u0"])
    dm.set_field(_abi.FIELD_VELOCITY, w["v0"])
    dt = w["dt_factor"] * dm.stable_time_step()
    dm.set_time_step(dt)
    dm.solve_steps(STEPS)
    return dt, dm.get_field(_abi.FIELD_DISPLACEMENT), dm.get_field(_abi.FIELD_VELOCITY)


def _run_whole(w):
    from tests.golden_cases import OracleAdapter
    cpu = OracleAdapter(w["mesh"], w["materials"])
    dt = configs.setup_model(cpu, w)
    cpu.solve_steps(STEPS)
    return dt, cpu.get(_abi.FIELD_DISPLACEMENT), cpu.get(_abi.FIELD_VELOCITY)


def _rel(x, ref):
    return np.abs(x - ref).max() / np.abs(ref).max()


@pytest.mark.parametrize("nparts", [2, 3, 5])
def test_partition_and_parts(nparts):
    mesh = configs.cube_tet4(n=6)["mesh"]
    part_of = partition_elements(mesh, nparts)
    counts = np.bincount(part_of, minlength=nparts)
    assert counts.sum() == len(mesh.connectivity)
    assert counts.max() - counts.min() <= 1
    parts, n_iface = build_parts(mesh, part_of, nparts)
    owners = np.zeros(len(mesh.nodes), dtype=int)
    seen = np.zeros(len(mesh.nodes), dtype=int)
    for p in parts:
        # local connectivity maps back to the global one
        assert np.array_equal(p.nodes[p.mesh.connectivity.astype(np.int64)],
                              mesh.connectivity[p.elements])
        owners[p.nodes[p.owned]] += 1
        seen[p.nodes] += 1
        assert np.array_equal(seen[p.nodes[p.iface_local]] >= 1, np.ones(len(p.iface_local), bool))
    assert (owners == 1).all()  # every node reported by exactly one part
    assert n_iface == int((seen >= 2).sum())
    rows = np.concatenate([p.iface_rows for p in parts])
    assert rows.min() == 0 and rows.max() == n_iface - 1


@pytest.mark.parametrize("nparts", [2, 3])
def test_parts_in_one_process_match_whole_mesh(nparts):
    w = _workload()
    dt_w, u_w, v_w = _run_whole(w)
    dt_d, u_d, v_d = _run_distributed(w, nparts)
    assert dt_d == dt_w
    assert _rel(u_d, u_w) <= 1e-11 and _rel(v_d, v_w) <= 1e-11


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import sys
    from datetime import timedelta
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        w = _workload()
        dt, u, v = _run_distributed(w, world)
        out[rank] = dict(dt=dt, u=u, v=v)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_match_whole_mesh():
    world, port = 2, _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    w = _workload()
    dt_w, u_w, v_w = _run_whole(w)
    for r in range(world):
        assert res[r]["dt"] == dt_w
        assert _rel(res[r]["u"], u_w) <= 1e-11 and _rel(res[r]["v"], v_w) <= 1e-11
