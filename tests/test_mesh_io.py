"""The Gmsh reader of libakb.so (include/akb_mesh.h), no GPU needed.

Checked on the reference's own mesh files (tests/golden/msh, copied by
tests/golden/make_golden.py) against an independent parse written here, and
against the reference reader's rules (mesh_io_msh.cc:337-440, 692-906;
mesh_io.cc:98-122): node ids renumbered in order of appearance, the elements
of the mesh's dimension form the mesh, every physical tag becomes a group
named from $PhysicalNames (or by its number), holding the nodes of all its
elements and the mesh elements among them; no group without $PhysicalNames.
"""
import json
import os

import numpy as np
import pytest

from akantu_b200 import _abi
from akantu_b200.mesh import Mesh

HERE = os.path.dirname(os.path.abspath(__file__))
MSH = os.path.join(HERE, "golden", "msh")
DIM_OF_TYPE = {1: 1, 2: 2, 4: 3, 5: 3, 15: 0}


def independent_parse(path, dim):
    """Nodes, mesh elements (Gmsh type of dimension dim) and physical groups."""
    lines = [ln.strip() for ln in open(path).read().splitlines()]
    names, nodes, index, elems = {}, [], {}, []
    i = 0
    while i < len(lines):
        if lines[i] == "$PhysicalNames":
            for k in range(int(lines[i + 1])):
                d, tag, name = lines[i + 2 + k].split(maxsplit=2)
                names[int(tag)] = name.strip('"')
            i += int(lines[i + 1]) + 2
        elif lines[i] == "$Nodes":
            for k in range(int(lines[i + 1])):
                p = lines[i + 2 + k].split()
                index[int(p[0])] = k
                nodes.append([float(x) for x in p[1:1 + dim]])
            i += int(lines[i + 1]) + 2
        elif lines[i] == "$Elements":
            for k in range(int(lines[i + 1])):
                p = [int(x) for x in lines[i + 2 + k].split()]
                t, nt = p[1], p[2]
                if t in DIM_OF_TYPE:
                    elems.append((t, p[3] if nt else 0, [index[n] for n in p[3 + nt:]]))
            i += int(lines[i + 1]) + 2
        else:
            i += 1
    mesh_elems = [e for e in elems if DIM_OF_TYPE[e[0]] == dim]
    groups = {}
    if names:
        m = 0
        for t, tag, conn in elems:
            g = groups.setdefault(names.get(tag, str(tag)), (set(), []))
            g[0].update(conn)
            if DIM_OF_TYPE[t] == dim:
                g[1].append(m)
                m += 1
            # elements of other dimensions do not count in the mesh's numbering
    return np.array(nodes), np.array([e[2] for e in mesh_elems]), groups


CASES = [("_triangle_3.msh", 2, _abi.TRIANGLE_3), ("_tetrahedron_4.msh", 3, _abi.TETRAHEDRON_4),
         ("_hexahedron_8.msh", 3, _abi.HEXAHEDRON_8), ("1_tetrahedron.msh", 3, _abi.TETRAHEDRON_4),
         ("material_selector.msh", 1, _abi.SEGMENT_2),
         ("cohesive_strait_2D.msh", 2, _abi.TRIANGLE_3)]


@pytest.mark.parametrize("name,dim,etype", CASES)
def test_reader_matches_independent_parse(name, dim, etype):
    path = os.path.join(MSH, name)
    mesh = Mesh(dim)
    mesh.read(path)
    nodes, conn, groups = independent_parse(path, dim)
    assert mesh.element_type == etype
    assert np.array_equal(mesh.nodes, nodes)
    assert np.array_equal(mesh.connectivity, conn)
    assert set(mesh.node_groups) == set(groups)
    for g, (gn, ge) in groups.items():
        assert np.array_equal(mesh.getNodeGroup(g), np.array(sorted(gn)))
        assert np.array_equal(mesh.getElementGroup(g), np.array(ge, dtype=np.int64))


def test_reader_matches_committed_patch_meshes():
    golden = json.load(open(os.path.join(HERE, "golden", "patch_meshes.json")))
    for key, d in golden["meshes"].items():
        mesh = Mesh(d["spatial_dimension"])
        mesh.read(os.path.join(MSH, key + ".msh"))
        assert np.array_equal(mesh.nodes, np.array(d["nodes"]))
        assert np.array_equal(mesh.connectivity, np.array(d["connectivity"]))


def test_named_groups_of_the_cohesive_mesh():
    """cohesive_strait_2D.msh: 'body' holds every triangle, the three line
    groups hold nodes only."""
    mesh = Mesh(2)
    mesh.read(os.path.join(MSH, "cohesive_strait_2D.msh"))
    assert sorted(mesh.node_groups) == ["body", "fixed", "insertion", "loading"]
    assert len(mesh.getElementGroup("body")) == mesh.getNbElement()
    for g in ("fixed", "insertion", "loading"):
        assert len(mesh.getElementGroup(g)) == 0 and len(mesh.getNodeGroup(g)) > 0
    # 'fixed', 'insertion' and 'loading' are the lines y = -1, 0 and 1
    y = mesh.nodes[:, 1]
    assert np.allclose(y[mesh.getNodeGroup("fixed")], -1.0)
    assert np.allclose(y[mesh.getNodeGroup("insertion")], 0.0)
    assert np.allclose(y[mesh.getNodeGroup("loading")], 1.0)


TEXT = """$MeshFormat
2.2 0 8
$EndMeshFormat
$Comments
anything here is skipped
$EndComments
$Nodes
4
10 0 0 0
20 1 0 0
30 0 1 0
40 1 1 0
$EndNodes
$Elements
4
1 2 2 7 1 10 20 40
2 2 2 7 1 10 40 30
3 1 2 9 2 10 30
4 3 2 7 3 10 20 40 30
$EndElements
"""


def test_tags_without_names_and_unsupported_types():
    """Non-contiguous node ids, a skipped block, a quadrangle (skipped), and
    no $PhysicalNames: no group is made."""
    mesh = Mesh(2)
    mesh.read_msh_text(TEXT)
    assert mesh.element_type == _abi.TRIANGLE_3
    assert np.array_equal(mesh.connectivity, [[0, 1, 3], [0, 3, 2]])
    assert mesh.node_groups == {}
    named = TEXT.replace("$Nodes", "$PhysicalNames\n1\n2 7 \"plate\"\n$EndPhysicalNames\n$Nodes")
    mesh.read_msh_text(named)
    assert sorted(mesh.node_groups) == ["9", "plate"]  # tag 9 has no name
    assert np.array_equal(mesh.getNodeGroup("9"), [0, 2])
    assert np.array_equal(mesh.getElementGroup("plate"), [0, 1])


@pytest.mark.parametrize("text,status", [
    (TEXT.replace("2.2 0 8", "4.1 0 8"), _abi.AKB_ERR_UNSUPPORTED),
    (TEXT.replace("2.2 0 8", "2.2 1 8"), _abi.AKB_ERR_UNSUPPORTED),
    (TEXT.replace("1 2 2 7 1 10 20 40", "1 2 2 7 1 10 20 99"), _abi.AKB_ERR_BAD_MESH),
    (TEXT.replace("$EndNodes", "$EndNode"), _abi.AKB_ERR_BAD_MESH),
    (TEXT.replace("$Elements\n4\n1 2 2 7 1 10 20 40\n2 2 2 7 1 10 40 30\n", "$Elements\n2\n"),
     _abi.AKB_ERR_BAD_MESH),
])
def test_bad_files_are_rejected(text, status):
    from akantu_b200._lib import AkbError
    with pytest.raises(AkbError) as exc:
        Mesh(2).read_msh_text(text)
    assert exc.value.status == status
