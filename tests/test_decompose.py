"""The partitioned-mesh path on CPU: the partition and the parts it builds,
the neighbour exchange plans (what each part sends to and receives from each
neighbour, and the order of every interface node's sum), and the exchange
(mass once, forces every step) driven by
akantu_b200.decompose.DistributedModel, with the FP64 CPU oracle standing in
for each part's GPU model and the plan's sums restated in numpy. A mesh cut
into 2, 3 or 4 parts, in one process, over two gloo ranks and over three
gloo ranks holding several parts each, must step like the whole mesh in one
oracle model (<= 1e-11 relative after 60 steps: the interface sums are added
in another order), and every copy of an interface node must stay equal."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from akantu_b200 import _abi, configs
from akantu_b200.decompose import DistributedModel, ExchangePlan, build_parts, partition_elements

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

    def set_exchange(self, plan):
        self.plan = plan

    def _ordered_sums(self, own, recv):
        """Per interface row, 0 + its terms in the plan's order (own value
        for -1, else the received row), as akb_part_step_end_exchange adds."""
        x = self.plan
        cnt = np.diff(x.sum_ptr)
        total = np.zeros_like(own)
        for j in range(int(cnt.max()) if len(cnt) else 0):
            rows = np.nonzero(cnt > j)[0]
            src = x.sum_src[x.sum_ptr[rows] + j]
            val = np.where((src < 0).reshape((-1,) + (1,) * (own.ndim - 1)),
                           own[rows], recv[np.maximum(src, 0)] if len(recv) else 0.0)
            total[rows] += val
        return total

    def pack_forces(self, send):
        send.copy_(torch.from_numpy(self.f[self.iface][self.plan.send_rows.astype(np.int64)]))

    def end_exchange(self, recv):
        self.f[self.iface] = self._ordered_sums(self.f[self.iface], recv.numpy())
        self._finish()

    def _finish(self):
        o, dt = self.o, self.dt
        free = o.blocked == 0
        r = (o.external_force + self.f) + o.mass * (-o.acceleration)
        x = r / o.mass
        o.velocity[free] = (o.velocity + (0.5 * dt) * x)[free]
        o.acceleration[free] = (o.acceleration + x)[free]

    def pack_mass(self, send):
        send.copy_(torch.from_numpy(self.o.mass[self.iface, 0][self.plan.send_rows.astype(np.int64)]))

    def import_mass_exchange(self, recv):
        total = self._ordered_sums(self.o.mass[self.iface, 0].copy(), recv.numpy())
        self.o.mass[self.iface, :] = total[:, None]

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


def _run_distributed(w, nparts, here=None, group=None, copies=False, **kw):
    dm = DistributedModel(w["mesh"], w["materials"], nparts, here=here, group=group,
                          backend=lambda p: OraclePart(p, w["materials"]), **kw)
    dm.set_blocked(w["blocked"])
    dm.set_field(_abi.FIELD_DISPLACEMENT, w["u0"])
    dm.set_field(_abi.FIELD_VELOCITY, w["v0"])
    dt = w["dt_factor"] * dm.stable_time_step()
    dm.set_time_step(dt)
    dm.solve_steps(STEPS)
    out = (dt, dm.get_field(_abi.FIELD_DISPLACEMENT), dm.get_field(_abi.FIELD_VELOCITY))
    if copies:  # every local copy of every node, by global id
        return out + ([(p.nodes, b.get_field(_abi.FIELD_VELOCITY))
                       for p, b in zip(dm.parts, dm.backends)], dm.bytes_per_step)
    return out


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


@pytest.mark.parametrize("nparts", [2, 3, 5, 8])
def test_exchange_plans(nparts):
    """Each pair of neighbours sends each other the nodes they share, in the
    same order; every interface row sums each of its holders once, in
    ascending part order, its own value included."""
    mesh = configs.cube_tet4(n=6)["mesh"]
    parts, _ = build_parts(mesh, partition_elements(mesh, nparts), nparts)
    plans = [ExchangePlan(p) for p in parts]
    for p, x in zip(parts, plans):
        gid = p.nodes[p.iface_local.astype(np.int64)]
        assert x.n_send == x.n_recv
        for k, q in enumerate(x.neighbours):
            mine = gid[x.send_rows[x.send_ptr[k]:x.send_ptr[k + 1]].astype(np.int64)]
            xq = plans[q]
            kq = xq.neighbours.index(p.index)
            theirs = parts[q].nodes[parts[q].iface_local.astype(np.int64)][
                xq.send_rows[xq.send_ptr[kq]:xq.send_ptr[kq + 1]].astype(np.int64)]
            assert np.array_equal(mine, theirs)  # q's block lands in p's receive slot k
            assert np.all(np.diff(mine) > 0)
            assert np.array_equal(np.sort(mine), np.intersect1d(gid, parts[q].nodes))
        for i in range(len(gid)):
            hs = p.holders[p.holder_ptr[i]:p.holder_ptr[i + 1]]
            assert np.all(np.diff(hs) > 0) and p.index in hs
            src = x.sum_src[x.sum_ptr[i]:x.sum_ptr[i + 1]]
            for h, t in zip(hs, src):
                if h == p.index:
                    assert t == -1
                else:
                    k = x.neighbours.index(int(h))
                    assert x.recv_ptr[k] <= t < x.recv_ptr[k + 1]
                    assert x.send_rows[t] == i  # the same node, at the same place
    # a pair's blocks are equal in size; bytes = 2 x 8 x d per shared row
    total = sum(x.bytes_per_step(3, set(range(nparts)) - {p.index}) for p, x in zip(parts, plans))
    assert total == 2 * 8 * 3 * sum(x.n_send for x in plans)


def _plate():
    w = configs.plate_tri3(nx=40, ny=8, lx=4.0, ly=0.8)
    rng = np.random.default_rng(9)
    v0 = rng.normal(0.0, 0.1, w["u0"].shape)
    v0[w["blocked"].astype(bool)] = 0.0
    w["v0"] = v0
    return w


@pytest.mark.parametrize("nparts,work", [(2, _workload), (3, _workload), (4, _workload),
                                         (3, _plate), (5, _plate)])
def test_parts_in_one_process_match_whole_mesh(nparts, work):
    w = work()
    dt_w, u_w, v_w = _run_whole(w)
    dt_d, u_d, v_d, copies, nbytes = _run_distributed(w, nparts, copies=True)
    assert dt_d == dt_w
    assert _rel(u_d, u_w) <= 1e-11 and _rel(v_d, v_w) <= 1e-11
    assert nbytes == 0  # every neighbour in this process: copies only
    # every copy of an interface node equals its owner's value, bit for bit
    for nodes, v in copies:
        assert np.array_equal(v, v_d[nodes])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, per_rank, out):
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
        # parts dealt round-robin, so that a rank's neighbours are both local
        # and remote
        here = list(range(rank, world * per_rank, world))
        dt, u, v, copies, nbytes = _run_distributed(w, world * per_rank, here=here, copies=True)
        out[rank] = dict(dt=dt, u=u, v=v, copies=copies, nbytes=nbytes)
    finally:
        dist.destroy_process_group()


def _check_ranks(res, world):
    w = _workload()
    dt_w, u_w, v_w = _run_whole(w)
    for r in range(world):
        assert res[r]["dt"] == dt_w
        assert _rel(res[r]["u"], u_w) <= 1e-11 and _rel(res[r]["v"], v_w) <= 1e-11
        assert np.array_equal(res[r]["u"], res[0]["u"])
        assert res[r]["nbytes"] > 0
        for nodes, v in res[r]["copies"]:
            assert np.array_equal(v, res[0]["v"][nodes])  # copies on all ranks equal


@pytest.mark.timeout(300)
@pytest.mark.parametrize("world,per_rank", [(2, 1), (3, 2)])
def test_gloo_ranks_match_whole_mesh(world, per_rank):
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(world, port, per_rank, out), nprocs=world, join=True)
        res = dict(out)
    _check_ranks(res, world)


def test_bar_slabs_are_the_cut_of_the_whole_bar():
    """configs.bar_tet4_slabs builds each slab without the whole mesh; it must
    equal build_parts of the whole bar cut into its cubes along z."""
    n, nslabs = 4, 3
    w = configs.bar_tet4(n, nslabs)
    part_of = np.arange(len(w["mesh"].connectivity)) // (6 * n ** 3)
    parts, _ = build_parts(w["mesh"], part_of, nslabs)
    s = configs.bar_tet4_slabs(n, nslabs, range(nslabs))
    for a, b in zip(parts, s["parts"]):
        for f in ("nodes", "elements", "iface_local", "owned", "holder_ptr", "holders"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
        assert np.array_equal(a.mesh.nodes, b.mesh.nodes)
        assert np.array_equal(a.mesh.connectivity, b.mesh.connectivity)
    assert s["nb_nodes"] == len(w["mesh"].nodes)
    assert np.array_equal(s["blocked"], w["blocked"]) and np.array_equal(s["v0"], w["v0"])


def _slab_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import sys
    from datetime import timedelta
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        s = configs.bar_tet4_slabs(4, world, [rank])
        dm = DistributedModel(None, s["materials"], world, parts=s["parts"],
                              nb_nodes=s["nb_nodes"],
                              backend=lambda p: OraclePart(p, s["materials"]))
        dm.set_blocked(s["blocked"])
        dm.set_field(_abi.FIELD_VELOCITY, s["v0"])
        dt = s["dt_factor"] * dm.stable_time_step()
        dm.set_time_step(dt)
        dm.solve_steps(STEPS)
        out[rank] = dict(dt=dt, u=dm.get_field(_abi.FIELD_DISPLACEMENT), nbytes=dm.bytes_per_step)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_bar_slabs_over_gloo_ranks_match_whole_bar():
    """Three ranks, one slab each (the bench's weak-scaled layout): the
    middle rank exchanges with two neighbours, the end ranks with one."""
    world, port = 3, _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_slab_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    w = configs.bar_tet4(4, world)
    dt_w, u_w, _ = _run_whole(w)
    plane_bytes = 2 * 8 * 3 * 25  # a 5 x 5 node plane, sent and received
    for r in range(world):
        assert res[r]["dt"] == dt_w
        assert _rel(res[r]["u"], u_w) <= 1e-11
        assert res[r]["nbytes"] == plane_bytes * (2 if r == 1 else 1)
