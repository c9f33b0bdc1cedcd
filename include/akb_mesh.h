/*
 * akb_mesh.h -- Gmsh mesh input of libakb.so (Mesh::read with MeshIOMSH).
 *
 * Reads Gmsh ASCII files of format 2.x (mesh_io_msh.cc:692-906 and the
 * version-2 readers populateReaders2, mesh_io_msh.cc:337-440): the $Nodes
 * block (node ids renumbered in order of appearance, as file.node_tags), the
 * $Elements block (element type, tags, nodes; tag 0 is the physical tag) and
 * the $PhysicalNames block, from which named groups are built
 * (MeshIO::constructPhysicalNames, mesh_io.cc:98-122, then
 * GroupManager::createGroupsFromMeshData("physical_names"),
 * group_manager.hh:200): a physical tag without a name is named by its
 * decimal value, and without a $PhysicalNames block no group is made. Other
 * blocks are skipped up to their $End line.
 *
 * The mesh handed to akb_model_create is the set of elements of the
 * requested spatial dimension (one type: segment_2 in 1D, triangle_3 in 2D,
 * tetrahedron_4 or hexahedron_8 in 3D) and all nodes; elements of lower
 * dimension (points, lines, faces) only carry groups. Gmsh types 1, 2, 3, 4,
 * 5 and 15 are read, others are skipped, as the reference skips types it does
 * not know (quadrangle_4, type 3, is kept only as the facet of a 3D mesh and
 * skipped in a 2D one, where the library has no such element); a group keeps
 * the nodes of all its elements, the indices of its elements of the mesh's
 * dimension and the connectivity of its facets (elements of one dimension
 * less), on which Neumann conditions act.
 *
 * Format 4 files and binary files are rejected (AKB_ERR_UNSUPPORTED).
 */
#ifndef AKB_MESH_H
#define AKB_MESH_H

#include "akb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct akb_msh akb_msh;

/* Mesh::read(filename) for a Gmsh file (mesh_io_msh.cc:692). */
akb_status akb_msh_read(const char* path, int32_t spatial_dimension, akb_msh** mesh);
/* The same from the text of a file held in memory (length bytes). */
akb_status akb_msh_parse(const char* text, int64_t length, int32_t spatial_dimension,
                         akb_msh** mesh);
akb_status akb_msh_destroy(akb_msh* mesh);

/* The elements of the mesh's dimension and all nodes, ready for
 * akb_model_create; the pointers stay valid until akb_msh_destroy. */
akb_status akb_msh_get_mesh(const akb_msh* mesh, akb_mesh_desc* desc);

/* Named groups (GroupManager element groups and their node groups,
 * group_manager.hh:63), in order of name. nodes: ascending node indices of
 * all the group's elements; elements: ascending indices, into the mesh's
 * connectivity, of its elements of the mesh's dimension. Pointers stay valid
 * until akb_msh_destroy. */
akb_status akb_msh_get_nb_groups(const akb_msh* mesh, int32_t* nb_groups);
akb_status akb_msh_get_group(const akb_msh* mesh, int32_t index, const char** name,
                             int64_t* nb_nodes, const uint32_t** nodes, int64_t* nb_elements,
                             const uint32_t** elements);
/* The facets of group index (its elements of dimension d - 1, the boundary
 * elements of ElementGroup::getElements(facet type), group_manager.hh:63):
 * nb_facets x nodes_per_facet node indices in the file's node order --
 * segment_2 facets (2 nodes) of a 2D mesh, triangle_3 (3) or quadrangle_4
 * (4) facets of a 3D one; nb_facets = 0 when the group has none. For a
 * group whose facets are of two kinds (triangles and quadrangles) the call
 * returns AKB_ERR_UNSUPPORTED; the file itself reads. */
akb_status akb_msh_get_group_facets(const akb_msh* mesh, int32_t index, int64_t* nb_facets,
                                    int32_t* nodes_per_facet, const uint32_t** facets);

/* Neumann conditions (BoundaryCondition::applyBC with a Neumann functor,
 * boundary_condition_tmpl.hh:95-185): on every facet the functor's value at
 * the Gauss points of the boundary element (1 point on a segment_2 or a
 * triangle_3, 2 x 2 on a quadrangle_4), times the shape functions, integrated
 * over the facet and ADDED into forces (nb_nodes x d, row-major, the
 * model's external force). kind AKB_NEUMANN_TRACTION (FromTraction,
 * Neumann::FromSameDim): value is the traction, d doubles.
 * AKB_NEUMANN_STRESS (FromStress, Neumann::FromHigherDim): value is a
 * stress, d x d column-major, and the traction sigma n, n the facet's unit
 * normal as the reference forms it from the facet's node order
 * (ElementClass::computeNormalsOnNaturalCoordinates, element_class_tmpl.hh:
 * 359-380: (t_y, -t_x) for a segment's tangent t, t_xi x t_eta for a
 * surface facet). d is 2 or 3 (the reference has no 1D Neumann condition). */
enum akb_neumann_kind {
  AKB_NEUMANN_TRACTION = 0,
  AKB_NEUMANN_STRESS = 1
};
akb_status akb_neumann_forces(int32_t spatial_dimension, int64_t nb_nodes, const double* nodes,
                              int64_t nb_facets, int32_t nodes_per_facet, const uint32_t* facets,
                              int32_t kind, const double* value, double* forces);

/* The Gauss points of the same facets, for a Neumann functor evaluated by
 * the caller (a NeumannFunctor written in Python, py_boundary_conditions.cc):
 * akb_facet_points(nodes_per_facet) points per facet (1 or 4; 0 for an
 * unknown facet), and at facet f, point q (row k = f * points + q) its
 * coordinates (coords[k][d]), unit normal (normals[k][d]) and w |J| N_a
 * (weighted_shapes[k][nodes_per_facet]): the force of a functor value t there
 * on the facet's node a is weighted_shapes[k][a] t. */
int32_t akb_facet_points(int32_t nodes_per_facet);
akb_status akb_facet_quadrature(int32_t spatial_dimension, int64_t nb_nodes, const double* nodes,
                                int64_t nb_facets, int32_t nodes_per_facet,
                                const uint32_t* facets, double* coords, double* normals,
                                double* weighted_shapes);

#ifdef __cplusplus
}
#endif

#endif /* AKB_MESH_H */
