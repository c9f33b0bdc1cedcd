"""Batches of independent meshes stepped together (akb_batch_create).

One BatchModel holds thousands of meshes of one element type, each with its
own material and time step. Each instance is split into patches on its own,
so the fused patch kernel advances every instance in the same launch and each
instance's state is bitwise the one a SolidMechanicsModel of that mesh alone
produces with the same patch options.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._lib import check, lib
from .mesh import Mesh
from .model import SolidMechanicsModel, material_from_dict


class BatchModel(SolidMechanicsModel):
    def __init__(self, meshes, materials, precision=_abi.MODE_FP64, device=0, stream=None,
                 patch_elements=0, patch_nodes=0, patch_grid=0):
        if len(meshes) != len(materials):
            raise ValueError("one material per instance")
        self.meshes = list(meshes)
        t = self.meshes[0].element_type
        d = self.meshes[0].spatial_dimension
        noff = np.cumsum([0] + [m.getNbNodes() for m in self.meshes])
        eoff = np.cumsum([0] + [m.getNbElement() for m in self.meshes])
        union = Mesh(d, t, np.concatenate([m.nodes for m in self.meshes]),
                     np.concatenate([m.connectivity.astype(np.int64) + o
                                     for m, o in zip(self.meshes, noff[:-1])]).astype(np.uint32))
        mats = [m if not isinstance(m, dict) else material_from_dict(m) for m in materials]
        super().__init__(union, mats, precision=precision, device=device, stream=stream,
                         patch_elements=patch_elements, patch_nodes=patch_nodes,
                         patch_grid=patch_grid)
        self.node_offsets = noff
        self.element_offsets = eoff

    @property
    def nb_instances(self):
        return len(self.meshes)

    def initFull(self, _analysis_method=0, precision=None):
        if precision is not None:
            self._precision = precision
        descs = []
        self._keep = []
        for m in self.meshes:
            nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
            conn = np.ascontiguousarray(m.connectivity, dtype=np.uint32)
            self._keep += [nodes, conn]
            descs.append(_abi.MeshDesc(m.spatial_dimension, m.element_type, nodes.shape[0],
                                       conn.shape[0], nodes.ctypes.data_as(C.POINTER(C.c_double)),
                                       conn.ctypes.data_as(C.POINTER(C.c_uint32))))
        mesh_arr = (_abi.MeshDesc * len(descs))(*descs)
        mat_arr = (_abi.MaterialDesc * len(self._materials))(*[m.desc() for m in self._materials])
        bd = _abi.BatchDesc(len(descs), mesh_arr, mat_arr)
        opt = _abi.ModelOptions(self._precision, self._device, self._stream, *self._patch)
        h = C.c_void_p()
        check(lib().akb_batch_create(C.byref(bd), C.byref(opt), C.byref(h)))
        self._h = h
        n = C.c_int32()
        no = (C.c_int64 * (len(descs) + 1))()
        eo = (C.c_int64 * (len(descs) + 1))()
        check(lib().akb_batch_get_layout(h, C.byref(n), no, eo))
        assert n.value == len(descs)
        assert list(no) == list(self.node_offsets) and list(eo) == list(self.element_offsets)

    def getStableTimeSteps(self):
        self._sync_in()
        out = np.zeros(self.nb_instances)
        check(lib().akb_batch_get_stable_time_steps(self.handle,
                                                    out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def setTimeSteps(self, dts):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        check(lib().akb_batch_set_time_steps(self.handle, dts.ctypes.data_as(C.POINTER(C.c_double))))

    def getEnergies(self, energy_id):
        self._sync_in()
        kind = {"kinetic": _abi.ENERGY_KINETIC, "potential": _abi.ENERGY_POTENTIAL}[energy_id]
        out = np.zeros(self.nb_instances)
        check(lib().akb_batch_get_energies(self.handle, kind,
                                           out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def instance_rows(self, i):
        return slice(int(self.node_offsets[i]), int(self.node_offsets[i + 1]))


def partition_instances(sizes, world):
    """Splits instances over `world` ranks by element count (longest
    processing time first: each instance, largest first, goes to the rank
    with the fewest elements so far; ties by rank). Independent instances
    need no collective in the step, so a batch shards with no data-path
    communication. Returns one ascending index list per rank."""
    sizes = np.asarray(sizes, dtype=np.int64)
    load = np.zeros(world, dtype=np.int64)
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]
