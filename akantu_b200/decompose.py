"""A mesh partitioned over processes, one part (and one GPU) per process.

The reference distributes a SolidMechanicsModel over MPI ranks: each rank
holds its elements plus ghost elements, and the residual contributions of
nodes on the interface between ranks are summed by the synchronizers
(solid_mechanics_model.cc:94-100, 395-411; ElementSynchronizer,
NodeSynchronizer). Here a part is a model of its own elements and the nodes
they touch (`akb_model_create_part`); a node touched by elements of several
parts (an interface node) exists in each of them. Once per step every
process adds its parts' internal forces on the interface nodes into one
array over all interface nodes, an all-reduce (sum) adds the processes'
arrays, and each part finishes its copy of every interface node with the
total, so all copies stay equal. The lumped mass of the interface nodes is
summed the same way once, and every part steps with one time step, the
minimum of the parts' stable steps.

Exchange per step: 8 B x d per interface node, one all-reduce (NCCL on the
models' CUDA stream, or gloo on CPU tensors).
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
    (ascending; local node i is global node nodes[i]), its local mesh, and
    its interface nodes (local ids, their rows in the array over all
    interface nodes). owned[i]: this part reports node i (the lowest part
    holding a node owns it)."""

    def __init__(self, index, elements, nodes, mesh, iface_local, iface_rows, owned):
        self.index = index
        self.elements = elements
        self.nodes = nodes
        self.mesh = mesh
        self.iface_local = iface_local
        self.iface_rows = iface_rows
        self.owned = owned


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
    parts = []
    for p, nodes in enumerate(node_sets):
        elements = np.nonzero(part_of == p)[0]
        local_conn = np.searchsorted(nodes, conn[elements]).astype(np.uint32)
        pm = Mesh(mesh.spatial_dimension, mesh.element_type, x[nodes], local_conn)
        iface_local = np.nonzero(count[nodes] >= 2)[0]
        parts.append(MeshPart(p, elements, nodes, pm, iface_local.astype(np.uint32),
                              row[nodes[iface_local]], owner[nodes] == p))
    return parts, len(iface)


# ---------------------------------------------------------------------------
# the sum over processes
# ---------------------------------------------------------------------------
class Exchange:
    """Sums (and minima) over the processes of a torch.distributed group; a
    process alone (holding all parts itself) exchanges nothing."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1

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

    def begin(self):
        self._call("akb_part_step_begin")

    def export_forces(self, out):
        self._call("akb_part_export_forces", C.c_void_p(out.data_ptr()))

    def end(self, total):
        self._call("akb_part_step_end", C.c_void_p(total.data_ptr()))

    def export_mass(self, out):
        self._call("akb_part_export_mass", C.c_void_p(out.data_ptr()))

    def import_mass(self, total):
        self._call("akb_part_import_mass", C.c_void_p(total.data_ptr()))

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

    Every process of the group calls the same methods in the same order
    (each is a collective when the group has several processes). Fields are
    exchanged as whole-mesh arrays: set_field takes the global array,
    get_field returns it (each node from its owning part)."""

    def __init__(self, mesh, materials, nparts, precision=_abi.MODE_FP64, device=0, here=None,
                 group=None, part_of=None, backend=None, **patch):
        import torch
        self.exchange = Exchange(group)
        rank = self.exchange.dist.get_rank(group) if self.exchange.world > 1 else 0
        if here is None:
            here = [rank] if self.exchange.world > 1 else list(range(nparts))
        self.mesh = mesh
        self.dim = mesh.spatial_dimension
        self.part_of = partition_elements(mesh, nparts) if part_of is None else np.asarray(part_of)
        all_parts, self.n_interface = build_parts(mesh, self.part_of, nparts)
        self.parts = [all_parts[p] for p in here]
        if backend is None:
            def backend(part):
                return GpuPart(part, materials, precision, device, **patch)
        self.backends = [backend(p) for p in self.parts]
        self.device = getattr(self.backends[0], "device", torch.device("cpu"))
        self._rows = [torch.as_tensor(p.iface_rows, dtype=torch.int64, device=self.device)
                      for p in self.parts]
        self._out = [torch.zeros((len(p.iface_rows), self.dim), dtype=torch.float64,
                                 device=self.device) for p in self.parts]
        self._in = [torch.zeros_like(o) for o in self._out]
        # lumped mass of the interface nodes: the sum over the parts
        total = torch.zeros(self.n_interface, dtype=torch.float64, device=self.device)
        for b, r in zip(self.backends, self._rows):
            m = torch.zeros(len(r), dtype=torch.float64, device=self.device)
            b.export_mass(m)
            total.index_add_(0, r, m)
        self.exchange.sum_(total)
        for b, r in zip(self.backends, self._rows):
            b.import_mass(total.index_select(0, r).contiguous())
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
        out = np.zeros((len(self.mesh.nodes), self.dim))
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
        import torch
        for b in self.backends:
            b.begin()
        total = torch.zeros((self.n_interface, self.dim), dtype=torch.float64, device=self.device)
        for b, r, o in zip(self.backends, self._rows, self._out):
            b.export_forces(o)
            total.index_add_(0, r, o)  # parts in a fixed order: a deterministic sum
        self.exchange.sum_(total)
        for b, r, i in zip(self.backends, self._rows, self._in):
            torch.index_select(total, 0, r, out=i)
            b.end(i)

    def solve_steps(self, n):
        for _ in range(int(n)):
            self.solve_step()

    def close(self):
        for b in self.backends:
            if hasattr(b, "close"):
                b.close()
