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
 * dimension (points, lines, faces) only carry groups. Gmsh types 1, 2, 4, 5
 * and 15 are read, others are skipped, as the reference skips types it does
 * not know; a group keeps the nodes of all its elements and the indices of
 * its elements of the mesh's dimension.
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

#ifdef __cplusplus
}
#endif

#endif /* AKB_MESH_H */
