"""Mesh container, Gmsh reader (through libakb.so) and structured mesh
generators.

Mirrors the subset of akantu::Mesh the explicit path uses (mesh.hh:100):
nodal coordinates (getNodes, mesh.hh:293), one connectivity array of the
spatial dimension's element type (getConnectivity, mesh.hh:353) and node
groups for boundary conditions (GroupManager, group_manager.hh:63).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi

# element type properties: (name, dimension, nodes per element, quadrature points)
ELEMENT_TYPES = {
    _abi.SEGMENT_2: ("_segment_2", 1, 2, 1),
    _abi.TRIANGLE_3: ("_triangle_3", 2, 3, 1),
    _abi.TETRAHEDRON_4: ("_tetrahedron_4", 3, 4, 1),
    _abi.HEXAHEDRON_8: ("_hexahedron_8", 3, 8, 8),
}
NAME_TO_TYPE = {v[0]: k for k, v in ELEMENT_TYPES.items()}

# boundary facets of each element type (local node indices)
_FACETS = {
    _abi.SEGMENT_2: [(0,), (1,)],
    _abi.TRIANGLE_3: [(0, 1), (1, 2), (2, 0)],
    _abi.TETRAHEDRON_4: [(0, 2, 1), (1, 2, 3), (2, 0, 3), (0, 1, 3)],
    _abi.HEXAHEDRON_8: [(0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4),
                        (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)],
}


def element_properties(element_type):
    name, dim, nnpe, nqp = ELEMENT_TYPES[element_type]
    return dim, nnpe, nqp


# facet kinds (the element types of a group's boundary elements); the
# library has no quadrangle element, so the facet kind has a number of its own
QUADRANGLE_4 = 5
FACET_TYPES = {(2, 2): 1, (3, 3): 2, (3, 4): QUADRANGLE_4}  # (dim, nodes) -> type


class IntegrationPoint:
    """IntegrationPoint (element.hh): which Gauss point a NeumannFunctor is
    called at -- type (the facet kind), element (the facet's index in the
    group), num_point, ghost_type."""

    def __init__(self, type, element=0, num_point=0, ghost_type=0):
        self.type, self.element, self.num_point, self.ghost_type = type, element, num_point, ghost_type


class Mesh:
    """Nodes (N x d, float64) + connectivity (E x n, uint32) + node groups."""

    def __init__(self, spatial_dimension, element_type=None, nodes=None,
                 connectivity=None):
        self.spatial_dimension = int(spatial_dimension)
        self.element_type = element_type
        self.nodes = np.zeros((0, self.spatial_dimension)) if nodes is None \
            else np.ascontiguousarray(nodes, dtype=np.float64)
        self.connectivity = np.zeros((0, 0), dtype=np.uint32) if connectivity is None \
            else np.ascontiguousarray(connectivity, dtype=np.uint32)
        self.node_groups: dict[str, np.ndarray] = {}
        self.element_groups: dict[str, np.ndarray] = {}
        # per group, its facets (elements of one dimension less), n x nodes
        self.facet_groups: dict[str, np.ndarray] = {}
        self._mixed_facets: set[str] = set()  # groups with facets of two kinds

    # --- reference-style accessors -------------------------------------
    def getNodes(self):
        return self.nodes

    def getConnectivity(self, element_type=None):
        return self.connectivity

    def getNbNodes(self):
        return self.nodes.shape[0]

    def getNbElement(self, element_type=None):
        return self.connectivity.shape[0]

    def getSpatialDimension(self):
        return self.spatial_dimension

    def getNodeGroup(self, name):
        return self.node_groups[name]

    def createNodeGroup(self, name, nodes):
        self.node_groups[name] = np.unique(np.asarray(nodes, dtype=np.int64))
        return self.node_groups[name]

    # --- Gmsh reader (MeshIOMSH::read, mesh_io_msh.cc) ------------------
    def read(self, filename):
        """Mesh::read of a Gmsh ASCII 2.x file through libakb.so
        (include/akb_mesh.h): the elements of this mesh's spatial dimension,
        all nodes, and one node group and element group per physical name."""
        from . import _lib
        h = C.c_void_p()
        _lib.check(_lib.lib().akb_msh_read(os.fsencode(filename), self.spatial_dimension,
                                           C.byref(h)))
        self._take(h)

    def read_msh_text(self, text):
        """The same from the text of a Gmsh file."""
        from . import _lib
        data = text.encode() if isinstance(text, str) else bytes(text)
        h = C.c_void_p()
        _lib.check(_lib.lib().akb_msh_parse(data, len(data), self.spatial_dimension, C.byref(h)))
        self._take(h)

    def _take(self, h):
        from . import _abi, _lib
        L = _lib.lib()
        try:
            desc = _abi.MeshDesc()
            _lib.check(L.akb_msh_get_mesh(h, C.byref(desc)))
            d = desc.spatial_dimension
            n = ELEMENT_TYPES[desc.element_type][2]
            self.element_type = desc.element_type
            self.nodes = np.ctypeslib.as_array(desc.nodes, (desc.nb_nodes * d,)).reshape(-1, d).copy()
            self.connectivity = np.ctypeslib.as_array(
                desc.connectivity, (desc.nb_elements * n,)).reshape(-1, n).copy()
            ng = C.c_int32()
            _lib.check(L.akb_msh_get_nb_groups(h, C.byref(ng)))
            self.node_groups, self.element_groups, self.facet_groups = {}, {}, {}
            self._mixed_facets = set()
            for k in range(ng.value):
                name = C.c_char_p()
                nn, ne = C.c_int64(), C.c_int64()
                pn, pe = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
                _lib.check(L.akb_msh_get_group(h, k, C.byref(name), C.byref(nn), C.byref(pn),
                                               C.byref(ne), C.byref(pe)))
                key = name.value.decode()
                self.node_groups[key] = (np.ctypeslib.as_array(pn, (nn.value,)).astype(np.int64)
                                         if nn.value else np.zeros(0, np.int64))
                self.element_groups[key] = (np.ctypeslib.as_array(pe, (ne.value,)).astype(np.int64)
                                            if ne.value else np.zeros(0, np.int64))
                nf, npf = C.c_int64(), C.c_int32()
                pf = C.POINTER(C.c_uint32)()
                st = L.akb_msh_get_group_facets(h, k, C.byref(nf), C.byref(npf), C.byref(pf))
                if st == _abi.AKB_ERR_UNSUPPORTED:  # facets of two kinds
                    self._mixed_facets.add(key)
                    continue
                _lib.check(st)
                if nf.value:  # the group's elements of one dimension less
                    self.facet_groups[key] = np.ctypeslib.as_array(
                        pf, (nf.value * npf.value,)).reshape(-1, npf.value).astype(np.uint32)
        finally:
            L.akb_msh_destroy(h)

    def getElementGroup(self, name):
        return self.element_groups[name]

    def getFacetGroup(self, name):
        """The group's facets (its elements of one dimension less, as read
        from the file): (n, nodes per facet) node indices."""
        return self.facet_groups[name]

    def neumannForces(self, group, functor):
        """The nodal forces of a Neumann functor on a group's facets, (N, d):
        FromTraction / FromStress integrated by akb_neumann_forces, any other
        NeumannFunctor called at the facets' Gauss points
        (akb_facet_quadrature) as functor(quad_point, dual, coord, normals)."""
        from . import _lib
        from .model import FromStress, FromTraction
        if group in self._mixed_facets:
            raise ValueError("group '%s' has facets of two kinds (triangles and quadrangles)"
                             % group)
        X = np.ascontiguousarray(self.nodes, dtype=np.float64)
        n, d = X.shape
        facets = np.ascontiguousarray(self.facet_groups.get(group, np.zeros((0, 2), np.uint32)),
                                      dtype=np.uint32)
        nf, npf = facets.shape
        xp = X.ctypes.data_as(C.POINTER(C.c_double))
        fp = facets.ctypes.data_as(C.POINTER(C.c_uint32))
        out = np.zeros((n, d))
        if nf == 0:
            return out
        L = _lib.lib()
        if type(functor) in (FromTraction, FromStress):
            value = np.ascontiguousarray(functor.akb_value(d), dtype=np.float64)
            _lib.check(L.akb_neumann_forces(d, n, xp, nf, npf, fp, functor.kind,
                                            value.ctypes.data_as(C.POINTER(C.c_double)),
                                            out.ctypes.data_as(C.POINTER(C.c_double))))
            return out
        nq = L.akb_facet_points(npf)
        coords, normals = np.zeros((nf * nq, d)), np.zeros((nf * nq, d))
        shapes = np.zeros((nf * nq, npf))
        _lib.check(L.akb_facet_quadrature(d, n, xp, nf, npf, fp,
                                          coords.ctypes.data_as(C.POINTER(C.c_double)),
                                          normals.ctypes.data_as(C.POINTER(C.c_double)),
                                          shapes.ctypes.data_as(C.POINTER(C.c_double))))
        qp = IntegrationPoint(FACET_TYPES[(d, npf)])
        for f in range(nf):
            for q in range(nq):
                k = f * nq + q
                qp.element, qp.num_point = f, q
                dual = np.zeros(d)
                functor(qp, dual, coords[k], normals[k])
                out[facets[f]] += shapes[k][:, None] * dual[None, :]
        return out

    # --- boundary groups (Mesh::createBoundaryGroupFromGeometry) ---------
    def boundary_nodes(self):
        """Nodes of facets that belong to exactly one element."""
        counts = {}
        for elem in self.connectivity:
            for f in _FACETS[self.element_type]:
                key = tuple(sorted(int(elem[k]) for k in f))
                counts[key] = counts.get(key, 0) + 1
        nodes = set()
        for key, c in counts.items():
            if c == 1:
                nodes.update(key)
        return np.array(sorted(nodes), dtype=np.int64)

    def boundary_facets(self):
        """The facets that belong to exactly one element, each ordered so that
        its normal (the reference's: (t_y, -t_x) of a segment's tangent,
        t_xi x t_eta of a surface facet) points out of its element."""
        X = np.asarray(self.nodes, dtype=np.float64)
        owner = {}
        for e, elem in enumerate(self.connectivity):
            for f in _FACETS[self.element_type]:
                nodes = [int(elem[k]) for k in f]
                key = tuple(sorted(nodes))
                owner[key] = None if key in owner else (e, nodes)
        out = []
        for key, val in owner.items():
            if val is None:
                continue
            e, nodes = val
            P = X[nodes]
            if len(nodes) == 2:
                t = P[1] - P[0]
                n = np.array([t[1], -t[0]])
            elif len(nodes) >= 3:
                n = np.cross(P[1] - P[0], P[-1] - P[0]) if len(nodes) == 4 else \
                    np.cross(P[1] - P[0], P[2] - P[0])
            else:
                continue  # points: no facet orientation in 1D
            out_dir = P.mean(axis=0) - X[self.connectivity[e]].mean(axis=0)
            if np.dot(n, out_dir) < 0:
                nodes = nodes[::-1] if len(nodes) < 4 else [nodes[0]] + nodes[:0:-1]
            out.append(nodes)
        return np.array(out, dtype=np.uint32).reshape(len(out), -1 if out else 0)

    def createElementGroupFromNodeGroup(self, name, node_group, dimension=None):
        """Mesh::createElementGroupFromNodeGroup (group_manager.hh): of the
        spatial dimension, the elements whose nodes all lie in the node
        group; of one dimension less, the boundary facets whose nodes all lie
        in it (outward-oriented, for Neumann conditions). The group's node
        group is made of its elements' nodes, as an element group's is."""
        d = self.spatial_dimension
        dimension = d if dimension is None else int(dimension)
        inside = np.zeros(len(self.nodes), dtype=bool)
        inside[self.getNodeGroup(node_group) if isinstance(node_group, str)
               else np.asarray(node_group, dtype=np.int64)] = True
        if dimension == d:
            conn = np.asarray(self.connectivity, dtype=np.int64)
            elements = np.nonzero(inside[conn].all(axis=1))[0]
            self.element_groups[name] = elements
            self.node_groups[name] = np.unique(conn[elements])
        elif dimension == d - 1 and d >= 2:
            facets = self.boundary_facets()
            keep = facets[inside[facets.astype(np.int64)].all(axis=1)]
            self.facet_groups[name] = keep
            self.element_groups[name] = np.zeros(0, dtype=np.int64)
            self.node_groups[name] = np.unique(keep.astype(np.int64))
        else:
            raise ValueError("element groups of dimension %d or %d" % (d, d - 1))
        return self.node_groups[name]

    def createBoundaryGroupFromGeometry(self):
        """One node group 'boundary' with every node on a boundary facet
        (the reference splits it into connected surfaces; the explicit path
        only uses the union)."""
        return self.createNodeGroup("boundary", self.boundary_nodes())

    def iterateNodeGroups(self):
        return self.node_groups.items()


# --------------------------------------------------------------------------
# structured generators (seeded synthetic workloads)
# --------------------------------------------------------------------------
def bar_segment2(nb_nodes, length=1.0):
    """1D bar of nb_nodes-1 segment_2 elements on [0, length]."""
    x = np.arange(nb_nodes, dtype=np.float64) * (length / (nb_nodes - 1))
    conn = np.stack([np.arange(nb_nodes - 1), np.arange(1, nb_nodes)], 1)
    return Mesh(1, _abi.SEGMENT_2, x.reshape(-1, 1), conn)


def plate_triangle3(nx, ny, lx, ly, origin=(0.0, 0.0)):
    """nx x ny squares over lx x ly, each split along the (i,j)-(i+1,j+1)
    diagonal into two counter-clockwise triangle_3; nodes numbered x-fastest,
    elements cell by cell (x-fastest), two per cell."""
    xs = origin[0] + np.arange(nx + 1, dtype=np.float64) * (lx / nx)
    ys = origin[1] + np.arange(ny + 1, dtype=np.float64) * (ly / ny)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    nodes = np.stack([X.ravel(), Y.ravel()], 1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n00 = (j * (nx + 1) + i).ravel()
    n10 = n00 + 1
    n01 = n00 + (nx + 1)
    n11 = n01 + 1
    t1 = np.stack([n00, n10, n11], 1)
    t2 = np.stack([n00, n11, n01], 1)
    conn = np.stack([t1, t2], 1).reshape(-1, 3)
    return Mesh(2, _abi.TRIANGLE_3, nodes, conn)


def _grid_nodes_3d(nx, lx, ny=None, ly=None, nz=None, lz=None):
    ny, nz = ny or nx, nz or nx
    ly, lz = ly or lx, lz or lx
    xs = np.arange(nx + 1, dtype=np.float64) * (lx / nx)
    ys = np.arange(ny + 1, dtype=np.float64) * (ly / ny)
    zs = np.arange(nz + 1, dtype=np.float64) * (lz / nz)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)


def cube_tetrahedron4(n, length=1.0):
    """n^3 cubes, each split into 6 tetrahedra around the (0,0,0)-(1,1,1)
    diagonal (Kuhn split), all positively oriented; nodes x-fastest."""
    return box_tetrahedron4(n, n, n, length, length, length)


def box_tetrahedron4(nx, ny, nz, lx, ly, lz):
    """nx x ny x nz boxes over lx x ly x lz, each split into 6 tetrahedra
    around its (0,0,0)-(1,1,1) diagonal (Kuhn split), all positively
    oriented; nodes x-fastest, elements box by box (x-fastest), six per box."""
    nodes = _grid_nodes_3d(nx, lx, ny, ly, nz, lz)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = (k * (ny + 1) * (nx + 1) + j * (nx + 1) + i).ravel()
    off = {"x": 1, "y": nx + 1, "z": (nx + 1) * (ny + 1)}
    tets = []
    for perm in ("xyz", "xzy", "yxz", "yzx", "zxy", "zyx"):
        a = off[perm[0]]
        b = a + off[perm[1]]
        c = b + off[perm[2]]
        # even permutations are positively oriented; odd ones swap two nodes
        even = perm in ("xyz", "yzx", "zxy")
        t = (base, base + a, base + b, base + c) if even else \
            (base, base + b, base + a, base + c)
        tets.append(np.stack(t, 1))
    conn = np.stack(tets, 1).reshape(-1, 4)
    return Mesh(3, _abi.TETRAHEDRON_4, nodes, conn)


def block_hexahedron8(n, length=1.0):
    """n^3 hexahedron_8 (reference node order: bottom face counter-clockwise,
    then top face); nodes x-fastest, elements x-fastest."""
    return box_hexahedron8(n, n, n, length, length, length)


def box_hexahedron8(nx, ny, nz, lx, ly, lz):
    """nx x ny x nz hexahedron_8 over lx x ly x lz (reference node order);
    nodes x-fastest, elements x-fastest."""
    nodes = _grid_nodes_3d(nx, lx, ny, ly, nz, lz)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    p, q = nx + 1, (nx + 1) * (ny + 1)
    b = (k * q + j * p + i).ravel()
    conn = np.stack([b, b + 1, b + 1 + p, b + p,
                     b + q, b + 1 + q, b + 1 + p + q, b + p + q], 1)
    return Mesh(3, _abi.HEXAHEDRON_8, nodes, conn)
