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
  msh/*.msh
      the Gmsh files themselves, as text, for the mesh reader's tests: the
      three patch-test meshes, test_materials/1_tetrahedron.msh (finite
      deformation test), material_selector.msh (named 1D groups) and
      test_cohesive/data/cohesive_strait_2D.msh (named 2D groups).
  reference_materials.json
      the material sections of test_materials/material_finite_deformation.dat,
      test_solid_mechanics_model_dynamics_material.dat and
      test_energies/test_solid_mechanics_model_work_material.dat.

usage: python tests/golden/make_golden.py REFERENCE_ROOT
"""
import json
import os
import re
import shutil
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

    smm = "test/test_model/test_solid_mechanics_model"
    msh_dir = os.path.join(HERE, "msh")
    os.makedirs(msh_dir, exist_ok=True)
    for src in ("test/test_model/patch_tests/data/_triangle_3.msh",
                "test/test_model/patch_tests/data/_tetrahedron_4.msh",
                "test/test_model/patch_tests/data/_hexahedron_8.msh",
                smm + "/test_materials/1_tetrahedron.msh",
                smm + "/material_selector.msh",
                smm + "/test_cohesive/data/cohesive_strait_2D.msh"):
        shutil.copyfile(os.path.join(ref, src), os.path.join(msh_dir, os.path.basename(src)))
    mats = {
        "finite_deformation": smm + "/test_materials/material_finite_deformation.dat",
        "dynamics": smm + "/test_solid_mechanics_model_dynamics_material.dat",
        "work": smm + "/test_energies/test_solid_mechanics_model_work_material.dat",
    }
    with open(os.path.join(HERE, "reference_materials.json"), "w") as fh:
        json.dump({k: dict(parse_material_dat(os.path.join(ref, v)), source=v)
                   for k, v in mats.items()}, fh, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
