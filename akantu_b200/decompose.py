"""A mesh partitioned over processes, one part (and one GPU) per process.

The reference distributes a SolidMechanicsModel over MPI ranks: each rank
holds its elements plus ghost elements, and the residual contributions of
nodes on the interface between ranks are summed by the synchronizers
(solid_mechanics_model.cc:94-100, 395-411; ElementSynchronizer,
element_synchronizer.hh:52, with its per-neighbour send and receive schemes).
Here a part is a model of its own elements and the nodes they touch
(`akb_model_create_part`); a node touched by elements of several parts (an
interface node) exists in each of them, and its holders are those parts.

Neighbour exchange. Two parts are neighbours when they share interface nodes.
Once per step every part packs, for each neighbour, its own internal force
on the nodes the two share (ascending global node id) into a send buffer
(`akb_part_pack_forces`), the blocks go to the neighbours by grouped
point-to-point transfers (NCCL send/recv on the models' stream over NVLink,
gloo on CPU tensors; a copy when both parts live in this process), and every
part finishes each interface node with the sum of its holders' values added
in ascending part order (`akb_part_step_end_exchange`), so every copy of a
node gets the same total, bit for bit. The lumped masses of the interface
nodes are summed the same way once, and all parts step with one time step,
the minimum of the parts' stable steps.

Bytes per part and step: 8 x d per node it shares with each neighbour, sent,
and as many received; nothing else crosses between processes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .mesh import Mesh


# ---------------------------------------------------------------------------
# partition
# ---------------------------------------------------------------------------
def partition_elements(mesh, nparts):
    """Part of every element: recursive coordinate bisection of the element
    centroids, each cut across the longest extent at the element count that
    gives the two sides whole numbers of equal parts."""
    conn = np.asarray(mesh.connectivity, dtype=np.int64)
    x = np.asarray(mesh.nodes, dtype=np.float64)
    ne = len(conn)
    part = np.zeros(ne, dtype=np.int32)
    if ne == 0 or nparts <= 1:
        return part
    cen = x[conn].mean(axis=1)

    def split(idx, first, count):
        if count == 1 or len(idx) == 0:
            part[idx] = first
            return
        left = count // 2
        k = len(idx) * left // count
        c = cen[idx]
        ax = int(np.argmax(c.max(axis=0) - c.min(axis=0)))
        order = np.lexsort((idx, c[:, ax]))  # by coordinate, ties by element id
        split(idx[order[:k]], first, left)
        split(idx[order[k:]], first + left, count - left)

    split(np.arange(ne), 0, int(nparts))
    return part


class MeshPart:
    """One part: its elements, the global ids of the nodes they touch
    (local node i is global node nodes[i]), its local mesh, its interface
    nodes (local ids; their rows in a numbering of all interface nodes of
    the mesh, or None) and the parts holding each of them (ascending, this
    one included: holders[holder_ptr[i]:holder_ptr[i+1]] for interface node
    i). owned[i]: this part reports node i (the lowest part holding a node
    owns it)."""

    def __init__(self, index, elements, nodes, mesh, iface_local, iface_rows, owned,
                 holder_ptr, holders):
        self.index = index
        self.elements = elements
        self.nodes = nodes
        self.mesh = mesh
        self.iface_local = iface_local
        self.iface_rows = iface_rows
        self.owned = owned
        self.holder_ptr = holder_ptr
        self.holders = holders


def build_parts(mesh, part_of, nparts):
    """The parts of a partitioned mesh and the number of interface nodes."""
    conn = np.asarray(mesh.connectivity, dtype=np.int64)
    x = np.asarray(mesh.nodes, dtype=np.float64)
    nn = len(x)
    part_of = np.asarray(part_of)
    node_sets = [np.unique(conn[part_of == p].ravel()) for p in range(nparts)]
    count = np.zeros(nn, dtype=np.int64)
    owner = np.full(nn, nparts, dtype=np.int64)
    for p, nodes in enumerate(node_sets):
        count[nodes] += 1
        owner[nodes] = np.minimum(owner[nodes], p)
    iface = np.nonzero(count >= 2)[0]
    row = np.full(nn, -1, dtype=np.int64)
    row[iface] = np.arange(len(iface))
    # holders of every interface node, ascending (CSR over the interface rows)
    pairs = np.concatenate([np.stack([row[nodes[count[nodes] >= 2]],
                                      np.full(int((count[nodes] >= 2).sum()), p)], 1)
                            for p, nodes in enumerate(node_sets)] or [np.zeros((0, 2), np.int64)])
    pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
    gptr = np.zeros(len(iface) + 1, dtype=np.int64)
    np.cumsum(np.bincount(pairs[:, 0], minlength=len(iface)), out=gptr[1:])
    ghold = pairs[:, 1]
    parts = []
    for p, nodes in enumerate(node_sets):
        elements = np.nonzero(part_of == p)[0]
        local_conn = np.searchsorted(nodes, conn[elements]).astype(np.uint32)
        pm = Mesh(mesh.spatial_dimension, mesh.element_type, x[nodes], local_conn)
        iface_local = np.nonzero(count[nodes] >= 2)[0]
        r = row[nodes[iface_local]]
        cnt = gptr[r + 1] - gptr[r]
        hptr = np.zeros(len(r) + 1, dtype=np.int64)
        np.cumsum(cnt, out=hptr[1:])
        take = np.repeat(gptr[r], cnt) + (np.arange(hptr[-1]) - np.repeat(hptr[:-1], cnt))
        parts.append(MeshPart(p, elements, nodes, pm, iface_local.astype(np.uint32), r,
                              owner[nodes] == p, hptr, ghold[take]))
    return parts, len(iface)


class ExchangePlan:
    """The neighbour exchange of one part (akb_part_set_exchange).

    neighbours: the parts sharing interface nodes with this one, ascending;
    send_rows[send_ptr[k]:send_ptr[k+1]]: the interface rows (indices into
    part.iface_local) packed for neighbours[k], ascending global node id;
    recv_ptr[k]: where neighbours[k]'s block starts in the received buffer
    (the same nodes in the same order, as that neighbour packs them);
    sum_ptr / sum_src: per interface row, its holders' values in ascending
    part order, -1 for this part's own, else a received row."""

    def __init__(self, part):
        p = part.index
        gid = np.asarray(part.nodes, dtype=np.int64)[part.iface_local.astype(np.int64)]
        n = len(gid)
        hptr, hold = part.holder_ptr, part.holders
        cnt = np.diff(hptr)
        row_of = np.repeat(np.arange(n), cnt)
        self.neighbours = [int(q) for q in np.unique(hold) if q != p]
        send_rows, send_ptr, pos = [], [0], {}
        for q in self.neighbours:
            rows = row_of[hold == q]
            rows = rows[np.argsort(gid[rows], kind="stable")]
            pos[q] = np.full(n, -1, dtype=np.int64)
            pos[q][rows] = send_ptr[-1] + np.arange(len(rows))
            send_rows.append(rows)
            send_ptr.append(send_ptr[-1] + len(rows))
        self.send_rows = (np.concatenate(send_rows) if send_rows
                          else np.zeros(0, np.int64)).astype(np.uint32)
        self.send_ptr = np.asarray(send_ptr, dtype=np.int64)
        self.recv_ptr = self.send_ptr.copy()  # the blocks received mirror the blocks sent
        src = np.full(len(hold), -1, dtype=np.int64)
        for q in self.neighbours:
            sel = hold == q
            src[sel] = pos[q][row_of[sel]]
        self.sum_ptr = np.asarray(hptr, dtype=np.int64)
        self.sum_src = src
        self.n_send = int(self.send_ptr[-1])
        self.n_recv = int(self.recv_ptr[-1])

    def bytes_per_step(self, dim, remote):
        """Bytes sent plus received per step with the neighbours in `remote`."""
        k = [i for i, q in enumerate(self.neighbours) if q in remote]
        rows = sum(int(self.send_ptr[i + 1] - self.send_ptr[i]) for i in k)
        return 2 * 8 * dim * rows


# ---------------------------------------------------------------------------
# the sum over processes
# ---------------------------------------------------------------------------
class Exchange:
    """Transfers between the parts of a torch.distributed group: the
    neighbour blocks of a step, and the minimum (time step) and whole-mesh
    sums (fields read back) outside the step; a process alone (holding all
    parts itself) only copies."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1

    def neighbours(self, plans, here, rank_of):
        """Prepares transfer(): plans[i] is the plan of local part here[i];
        rank_of[q] the rank (in the group) holding part q."""
        self.here = list(here)
        self.local = {q: i for i, q in enumerate(self.here)}
        self.plans = plans
        self.rank_of = rank_of
        self.me = self.dist.get_rank(self.group) if self.world > 1 else 0
        self.copies, self.remote = [], []
        for i, (p, x) in enumerate(zip(self.here, plans)):
            for k, q in enumerate(x.neighbours):
                recv = (i, int(x.recv_ptr[k]), int(x.recv_ptr[k + 1]))
                if q in self.local:  # q packed its block for p: copy it over
                    j = self.local[q]
                    kq = plans[j].neighbours.index(p)
                    self.copies.append((recv, (j, int(plans[j].send_ptr[kq]),
                                               int(plans[j].send_ptr[kq + 1]))))
                else:
                    send = (i, int(x.send_ptr[k]), int(x.send_ptr[k + 1]))
                    self.remote.append(((p, q), "send", send, rank_of[q]))
                    self.remote.append(((q, p), "recv", recv, rank_of[q]))
        # both ends of a pair of ranks post their messages in one order: by
        # (source part, destination part)
        self.remote.sort(key=lambda m: m[0])

    def transfer(self, sends, recvs):
        """recvs[i] <- the blocks the neighbours of local part i packed for
        it (rows of sends / recvs are values or d-vectors)."""
        for (i, a, b), (j, c, d) in self.copies:
            recvs[i][a:b].copy_(sends[j][c:d])
        if not self.remote:
            return
        dist = self.dist
        ops = []
        for (src, dst), kind, (i, a, b), peer in self.remote:
            g = peer if self.group is None else dist.get_global_rank(self.group, peer)
            tag = src * len(self.rank_of) + dst
            if kind == "send":
                ops.append(dist.P2POp(dist.isend, sends[i][a:b], g, self.group, tag))
            else:
                ops.append(dist.P2POp(dist.irecv, recvs[i][a:b], g, self.group, tag))
        for work in dist.batch_isend_irecv(ops):
            work.wait()

    def sum_(self, t):
        if self.world > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t

    def min(self, x, device="cpu"):
        if self.world == 1:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return float(t.item())


# ---------------------------------------------------------------------------
# a part on the GPU
# ---------------------------------------------------------------------------
class GpuPart:
    """A part as a libakb.so model (akb_model_create_part) on torch's current
    stream of its device, so that the torch operations and collectives of
    the exchange are ordered with its kernels."""

    def __init__(self, part, materials, precision, device=0, **patch):
        import torch
        from .model import SolidMechanicsModel, material_from_dict, torch_stream
        self.device = torch.device("cuda", device)
        self.m = SolidMechanicsModel(part.mesh, [material_from_dict(mm) for mm in materials],
                                     precision=precision, device=device,
                                     stream=torch_stream(device),
                                     interface_nodes=part.iface_local, **patch)
        self.m.initFull()
        self.dim = self.m.dim

    def _call(self, name, *args):
        from ._lib import check, lib
        check(getattr(lib(), name)(self.m.handle, *args))

    def set_exchange(self, plan):
        i64 = C.POINTER(C.c_int64)
        rows = np.ascontiguousarray(plan.send_rows, dtype=np.uint32)
        ptr = np.ascontiguousarray(plan.sum_ptr, dtype=np.int64)
        src = np.ascontiguousarray(plan.sum_src, dtype=np.int64)
        self._call("akb_part_set_exchange", plan.n_send,
                   rows.ctypes.data_as(C.POINTER(C.c_uint32)), plan.n_recv,
                   ptr.ctypes.data_as(i64), src.ctypes.data_as(i64))

    def begin(self):
        self._call("akb_part_step_begin")

    def pack_forces(self, send):
        self._call("akb_part_pack_forces", C.c_void_p(send.data_ptr()))

    def end_exchange(self, recv):
        self._call("akb_part_step_end_exchange", C.c_void_p(recv.data_ptr()))

    def pack_mass(self, send):
        self._call("akb_part_pack_mass", C.c_void_p(send.data_ptr()))

    def import_mass_exchange(self, recv):
        self._call("akb_part_import_mass_exchange", C.c_void_p(recv.data_ptr()))

    def stable_time_step(self):
        return self.m.getStableTimeStep()

    def set_time_step(self, dt):
        self.m.setTimeStep(dt)

    def set_field(self, field, values):
        self.m.setField(field, values)

    def get_field(self, field):
        return np.array(self.m.getField(field))

    def set_blocked(self, blocked):
        self.m.setBlockedDOFs(blocked)

    def close(self):
        self.m.close()


class DistributedModel:
    """The parts `here` (default: the part of this process's rank) of a mesh
    cut into nparts, stepped together with the other processes' parts.

    The parts come from cutting `mesh` (coordinate bisection, or part_of),
    or are given ready-made (`parts`: this process's MeshPart objects, with
    global node ids and holders; nb_nodes: the whole mesh's node count).
    Every process of the group calls the same methods in the same order
    (each is a collective when the group has several processes). Fields are
    exchanged as whole-mesh arrays: set_field takes the global array,
    get_field returns it (each node from its owning part)."""

    def __init__(self, mesh, materials, nparts, precision=_abi.MODE_FP64, device=0, here=None,
                 group=None, part_of=None, backend=None, parts=None, nb_nodes=None, **patch):
        import torch
        self.exchange = Exchange(group)
        world = self.exchange.world
        rank = self.exchange.dist.get_rank(group) if world > 1 else 0
        self.nparts = int(nparts)
        if parts is None:
            if here is None:
                here = [rank] if world > 1 else list(range(nparts))
            self.dim = mesh.spatial_dimension
            self.nb_nodes = len(mesh.nodes)
            self.part_of = partition_elements(mesh, nparts) if part_of is None else np.asarray(part_of)
            all_parts, self.n_interface = build_parts(mesh, self.part_of, nparts)
            self.parts = [all_parts[p] for p in here]
        else:
            self.parts = list(parts)
            here = [p.index for p in self.parts]
            self.dim = self.parts[0].mesh.spatial_dimension
            self.nb_nodes = int(nb_nodes)
            self.n_interface = None
        self.mesh = mesh
        # which rank holds each part
        if world > 1:
            gathered = [None] * world
            self.exchange.dist.all_gather_object(gathered, list(here), group=group)
        else:
            gathered = [list(here)]
        rank_of = [-1] * self.nparts
        for r, hs in enumerate(gathered):
            for q in hs:
                rank_of[q] = r
        if min(rank_of) < 0:
            raise ValueError("every part must be held by one process of the group")
        if backend is None:
            def backend(part):
                return GpuPart(part, materials, precision, device, **patch)
        self.backends = [backend(p) for p in self.parts]
        self.device = getattr(self.backends[0], "device", torch.device("cpu"))
        self.plans = [ExchangePlan(p) for p in self.parts]
        self.exchange.neighbours(self.plans, here, rank_of)
        for b, x in zip(self.backends, self.plans):
            b.set_exchange(x)
        f64 = dict(dtype=torch.float64, device=self.device)
        self._send = [torch.zeros((x.n_send, self.dim), **f64) for x in self.plans]
        self._recv = [torch.zeros((x.n_recv, self.dim), **f64) for x in self.plans]
        remote = {q for q in range(self.nparts) if q not in set(here)}
        self.bytes_per_step = sum(x.bytes_per_step(self.dim, remote) for x in self.plans)
        # lumped mass of the interface nodes: the sum over the parts holding them
        send = [torch.zeros(x.n_send, **f64) for x in self.plans]
        recv = [torch.zeros(x.n_recv, **f64) for x in self.plans]
        for b, t in zip(self.backends, send):
            b.pack_mass(t)
        self.exchange.transfer(send, recv)
        for b, t in zip(self.backends, recv):
            b.import_mass_exchange(t)
        self.dt = None

    # -- state ------------------------------------------------------------
    def set_field(self, field, values):
        values = np.asarray(values, dtype=np.float64).reshape(-1, self.dim)
        for p, b in zip(self.parts, self.backends):
            b.set_field(field, values[p.nodes])

    def set_blocked(self, blocked):
        blocked = np.asarray(blocked, dtype=np.uint8).reshape(-1, self.dim)
        for p, b in zip(self.parts, self.backends):
            b.set_blocked(blocked[p.nodes])

    def get_field(self, field):
        """The whole-mesh array, each node from the part that owns it."""
        import torch
        out = np.zeros((self.nb_nodes, self.dim))
        for p, b in zip(self.parts, self.backends):
            out[p.nodes[p.owned]] = b.get_field(field)[p.owned]
        if self.exchange.world > 1:
            t = torch.as_tensor(out, device=self.device)
            self.exchange.sum_(t)
            out = t.cpu().numpy()
        return out

    def stable_time_step(self):
        return self.exchange.min(min(b.stable_time_step() for b in self.backends),
                                 device=self.device)

    def set_time_step(self, dt):
        self.dt = float(dt)
        for b in self.backends:
            b.set_time_step(self.dt)

    # -- stepping ---------------------------------------------------------
    def solve_step(self):
        for b in self.backends:
            b.begin()
        for b, t in zip(self.backends, self._send):
            b.pack_forces(t)
        self.exchange.transfer(self._send, self._recv)
        for b, t in zip(self.backends, self._recv):
            b.end_exchange(t)

    def solve_steps(self, n):
        for _ in range(int(n)):
            self.solve_step()

    def close(self):
        for b in self.backends:
            if hasattr(b, "close"):
                b.close()
