"""Generates the golden fixtures of tests/golden/ from the Akantu 3.1.0 test
suite (run once, where the reference tree is available; the JSON files are
committed so the tests never read the reference at run time).

  model_solver_dynamic_explicit.json
      the 402-row table of
      test/test_model/test_common/test_model_solver/test_model_solver_dynamic_explicit.verified
      (time, wext, epot, ekin, total, max_disp, min_disp), produced by
      test_model_solver_dynamic.cc with EXPLICIT=true.
  patch_meshes.json
      nodes and connectivity of test/test_model/patch_tests/data/_{triangle_3,
      tetrahedron_4,hexahedron_8}.msh (Gmsh v2, parsed by akantu_b200.mesh)
      and the material sections of material_check_stress_plane_strain.dat and
      material_lumped.dat.

usage: python tests/golden/make_golden.py [reference_root]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from akantu_b200.mesh import Mesh  # noqa: E402


def parse_material_dat(path):
    """`material elastic [ key = value ... ]` -> dict of floats/bools."""
    text = open(path).read()
    m = re.search(r"material\s+(\w+)\s*\[(.*?)\]", text, re.S)
    params = {"law": m.group(1)}
    for line in m.group(2).splitlines():
        line = line.split("#")[0].strip()
        if "=" not in line:
            continue
        k, v = [s.strip() for s in line.split("=", 1)]
        if v in ("true", "false"):
            params[k] = v == "true"
        else:
            try:
                params[k] = float(v)
            except ValueError:
                params[k] = v
    return params


def main(ref):
    out = {}
    ver = os.path.join(ref, "test/test_model/test_common/test_model_solver/"
                            "test_model_solver_dynamic_explicit.verified")
    lines = [ln for ln in open(ver).read().splitlines() if ln.strip()]
    header = [h.strip() for h in lines[0].split(",")]
    rows = [[s.strip() for s in ln.split(",")] for ln in lines[1:]]
    out["model_solver"] = {
        "source": "test/test_model/test_common/test_model_solver/"
                  "test_model_solver_dynamic_explicit.verified",
        "header": header,
        "rows": rows,
    }
    with open(os.path.join(HERE, "model_solver_dynamic_explicit.json"), "w") as fh:
        json.dump(out["model_solver"], fh, indent=0)

    data = os.path.join(ref, "test/test_model/patch_tests/data")
    meshes = {}
    for name, dim in (("_triangle_3", 2), ("_tetrahedron_4", 3), ("_hexahedron_8", 3)):
        mesh = Mesh(dim)
        mesh.read(os.path.join(data, name + ".msh"))
        meshes[name] = {
            "source": "test/test_model/patch_tests/data/%s.msh" % name,
            "spatial_dimension": dim,
            "element_type": int(mesh.element_type),
            "nodes": mesh.nodes.tolist(),
            "connectivity": mesh.connectivity.astype(int).tolist(),
        }
    materials = {
        "plane_strain": parse_material_dat(os.path.join(data, "material_check_stress_plane_strain.dat")),
        "lumped": parse_material_dat(os.path.join(data, "material_lumped.dat")),
    }
    with open(os.path.join(HERE, "patch_meshes.json"), "w") as fh:
        json.dump({"meshes": meshes, "materials": materials}, fh, indent=0)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
