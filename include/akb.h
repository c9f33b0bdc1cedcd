/*
 * akb.h -- C ABI of the B200-native explicit-dynamics library (libakb.so).
 *
 * This is the drop-in boundary for Akantu's explicit central-difference path
 * with lumped mass. The reference exposes that path only as a C++ class API
 * (no C ABI); every entry point below names the reference member function it
 * replaces, cited as file:line within the Akantu 3.1.0 source tree.
 *
 * Conventions
 *  - Plain pointers and sizes only; no CUDA or torch types in any signature
 *    (streams are passed as void*, holding a cudaStream_t).
 *  - Host arrays use the reference Array<T> layout: one row per node (or per
 *    element, or per quadrature point), components contiguous, row-major.
 *  - Every call returns an akb_status; AKB_OK is 0. On failure a message is
 *    stored per host thread and returned by akb_last_error().
 *  - A model handle may be used by one host thread at a time.
 */
#ifndef AKB_H
#define AKB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AKB_ABI_VERSION 1

typedef int32_t akb_status;
enum {
  AKB_OK = 0,
  AKB_ERR_INVALID_ARGUMENT = 1,
  AKB_ERR_BAD_MESH = 2,
  AKB_ERR_NEGATIVE_JACOBIAN = 3, /* integrator_gauss_inline_impl.hh:183-205 */
  AKB_ERR_NON_FINITE = 4,
  AKB_ERR_CUDA = 5,
  AKB_ERR_TIMEOUT = 6,
  AKB_ERR_STATE = 7,
  AKB_ERR_UNSUPPORTED = 8,
  AKB_ERR_OUT_OF_MEMORY = 9
};

/* Element types on the path (reference ElementType, aka_element_classes_info). */
enum {
  AKB_SEGMENT_2 = 1,
  AKB_TRIANGLE_3 = 2,
  AKB_TETRAHEDRON_4 = 3,
  AKB_HEXAHEDRON_8 = 4
};

/* Constitutive laws on the path. */
enum {
  AKB_MATERIAL_ELASTIC = 0,    /* materials/material_elastic.cc */
  AKB_MATERIAL_NEOHOOKEAN = 1, /* material_finite_deformation/material_neohookean.cc */
  AKB_MATERIAL_USER = 2        /* stresses written by the caller between
                                  akb_step_begin and akb_step_end (akb_fe2.h):
                                  the Material::computeStress plugin, material.hh:110 */
};

/* Arithmetic modes.
 * AKB_MODE_FP64_REFERENCE: FP64, the reference's own operation order (stored
 *   shape derivatives, B^T sigma, Gauss integration, element-order scatter),
 *   compiled without FMA contraction.
 * AKB_MODE_FP64: FP64 element and nodal arithmetic, fused kernels.
 * AKB_MODE_FP32_BULK: element gradient, stress and B^T sigma in FP32 with
 *   FP32 accumulation; nodal state, inverse lumped mass and energies FP64. */
enum {
  AKB_MODE_FP64_REFERENCE = 0,
  AKB_MODE_FP64 = 1,
  AKB_MODE_FP32_BULK = 2
};

/* Fields (reference getters, solid_mechanics_model.hh:364-397). */
enum {
  AKB_FIELD_DISPLACEMENT = 0,   /* N x d, read/write */
  AKB_FIELD_VELOCITY = 1,       /* N x d, read/write */
  AKB_FIELD_ACCELERATION = 2,   /* N x d, read/write */
  AKB_FIELD_EXTERNAL_FORCE = 3, /* N x d, read/write */
  AKB_FIELD_INTERNAL_FORCE = 4, /* N x d, read only */
  AKB_FIELD_MASS = 5,           /* N x d, read only (after mass assembly) */
  AKB_FIELD_NODES = 6,          /* N x d, read only */
  AKB_FIELD_GRAD_U = 7,         /* (E*q) x d*d column-major, read only */
  AKB_FIELD_STRESS = 8          /* (E*q) x d*d: Cauchy (small strain) or PK2 */
};

/* Energies (SolidMechanicsModel::getEnergy, solid_mechanics_model.cc:536-683). */
enum {
  AKB_ENERGY_KINETIC = 0,
  AKB_ENERGY_POTENTIAL = 1,
  AKB_ENERGY_EXTERNAL_WORK = 2
};

typedef struct {
  int32_t spatial_dimension;   /* 1, 2 or 3 */
  int32_t element_type;        /* AKB_SEGMENT_2 ... AKB_HEXAHEDRON_8 */
  int64_t nb_nodes;
  int64_t nb_elements;
  const double* nodes;          /* [nb_nodes][spatial_dimension] */
  const uint32_t* connectivity; /* [nb_elements][nodes_per_element] */
} akb_mesh_desc;

/* Parameters of one material section of the reference input file
 * (material elastic [ rho, E, nu, Plane_Stress, finite_deformation ]). */
typedef struct {
  int32_t kind;               /* AKB_MATERIAL_* */
  int32_t plane_stress;       /* 2D only; 0 = plane strain (reference default) */
  int32_t finite_deformation; /* elastic only; neo-Hookean is always finite */
  int32_t reserved;
  double rho;
  double E;
  double nu;
} akb_material_desc;

typedef struct {
  int32_t precision_mode; /* AKB_MODE_* */
  int32_t device;         /* CUDA device ordinal */
  void* stream;           /* cudaStream_t to run on; NULL = library-owned stream */
  int32_t patch_elements; /* fast modes: elements per patch (0 = per-type default) */
  int32_t patch_nodes;    /* fast modes: node cap of a patch (0 = per-type default) */
  int32_t patch_grid;     /* fast modes: 0 = one CTA per patch; > 0 = persistent grid
                             of that many CTAs striding over the patches */
} akb_model_options;

typedef struct {
  int32_t spatial_dimension;
  int32_t element_type;
  int32_t nodes_per_element;
  int32_t quadrature_points_per_element;
  int64_t nb_nodes;
  int64_t nb_elements;
  int32_t precision_mode;
  int32_t nb_materials;
  int64_t device_bytes; /* bytes of device memory the model holds */
} akb_model_info;

typedef struct akb_model akb_model;

/* Library version and the message of the last failed call on this thread. */
int32_t akb_abi_version(void);
const char* akb_last_error(void);

/* SolidMechanicsModel(mesh) + initFull(_analysis_method = _explicit_lumped_mass)
 * (solid_mechanics_model.hh:85-88, model.hh:78-99, solid_mechanics_model.cc:132-147).
 * element_material may be NULL (every element uses material 0); otherwise one
 * material index per element (the reference's material_index). */
akb_status akb_model_create(const akb_mesh_desc* mesh, int32_t nb_materials,
                            const akb_material_desc* materials,
                            const uint32_t* element_material,
                            const akb_model_options* options,
                            akb_model** model);
akb_status akb_model_destroy(akb_model* model);
akb_status akb_model_get_info(const akb_model* model, akb_model_info* info);

/* getDisplacement()/getVelocity()/... copies (solid_mechanics_model.hh:364-397).
 * count is the number of doubles in the host array. */
akb_status akb_set_field(akb_model* model, int32_t field, const double* values,
                         int64_t count);
akb_status akb_get_field(akb_model* model, int32_t field, double* values,
                         int64_t count);
/* Device address of a field, valid until akb_model_destroy. Quadrature-point
 * fields are in element order. Nodal fields (N x d doubles) are in the
 * model's own node order: in AKB_MODE_FP64 and AKB_MODE_FP32_BULK the fused
 * step keeps its nodes renumbered so that the nodes of each element patch are
 * contiguous; akb_get_node_numbering gives the row of each node. A caller
 * that writes a nodal field through this address calls akb_set_field (or
 * akb_apply_dirichlet) before the next step, which resets the state the step
 * derives from it. */
akb_status akb_field_device_pointer(akb_model* model, int32_t field,
                                    void** device_pointer);
/* Row of each node in the device arrays of the nodal fields:
 * row_of_node[i] for the caller's node i (the identity in
 * AKB_MODE_FP64_REFERENCE and for user materials). No reference
 * counterpart: the reference's nodal Arrays are in mesh order. */
akb_status akb_get_node_numbering(const akb_model* model, uint32_t* row_of_node,
                                  int64_t count);

/* getBlockedDOFs() (solid_mechanics_model.hh:397): N x d bytes, 0 or 1. */
akb_status akb_set_blocked_dofs(akb_model* model, const uint8_t* blocked,
                                int64_t count);
akb_status akb_get_blocked_dofs(akb_model* model, uint8_t* blocked,
                                int64_t count);

/* SolidMechanicsModel::assembleMassLumped (solid_mechanics_model_mass.cc:58-133). */
akb_status akb_assemble_mass_lumped(akb_model* model);

/* SolidMechanicsModel::getStableTimeStep (solid_mechanics_model.cc:482-533). */
akb_status akb_get_stable_time_step(akb_model* model, double* time_step);

/* setTimeStep / getTimeStep (solid_mechanics_model.cc:109-115, model_solver.cc:321-325). */
akb_status akb_set_time_step(akb_model* model, double time_step);
akb_status akb_get_time_step(const akb_model* model, double* time_step);

/* ModelSolver::solveStep (model_solver.cc:265-278) for the explicit lumped
 * solver: NonLinearSolverLumped::solve (non_linear_solver_lumped.cc:58-82). */
akb_status akb_solve_step(akb_model* model);
/* nb_steps consecutive solveStep() calls, replayed from a CUDA graph. */
akb_status akb_solve_steps(akb_model* model, int64_t nb_steps);
/* akb_solve_steps timed with CUDA events on the model's stream; *elapsed_ms
 * is the device time of the whole sequence. */
akb_status akb_time_solve_steps(akb_model* model, int64_t nb_steps,
                                double* elapsed_ms);

/* SolidMechanicsModel::assembleInternalForces (solid_mechanics_model.cc:375-414)
 * at the current displacement. */
akb_status akb_assemble_internal_forces(akb_model* model);
/* Material::computeAllStresses (material.cc:254-279) at the current
 * displacement; fills AKB_FIELD_GRAD_U and AKB_FIELD_STRESS. */
akb_status akb_compute_stresses(akb_model* model);

/* SolidMechanicsModel::getEnergy (solid_mechanics_model.cc:665-683). */
akb_status akb_get_energy(akb_model* model, int32_t kind, double* value);
/* The same without waiting: the reduction and the copy of its result to
 * *value are queued on the model's stream, and *value is written when the
 * stream reaches them; read it after akb_synchronize (the copy itself runs
 * on a stream of the library's, so an event of the model's stream does not
 * cover it). value: host memory (pinned, for the copy to run
 * asynchronously) or device memory. Lets a time loop that records the
 * energies of every step (examples/explicit/explicit_dynamic.cc:87-99) run
 * without a host round trip per step. No reference counterpart. */
akb_status akb_get_energy_async(akb_model* model, int32_t kind, double* value);

/* applyBC(BC::Dirichlet::FixedValue(value, component), group)
 * (boundary_condition_functor_inline_impl.hh:85-93, boundary_condition_tmpl.hh:63-88):
 * for each listed node, blocks DOF (node, component) and sets its
 * displacement to values[k]. nodes and values are host arrays of nb_nodes
 * entries; they are copied before the call returns (and may be reused
 * then), while the upload and the update are queued on the model's stream:
 * an error of the update is reported by the next call that synchronises.
 * component AKB_ALL_COMPONENTS: every component of the listed nodes at once,
 * values then holding nb_nodes x spatial_dimension entries (row per node),
 * the functor applied to every axis of a group in one call. */
#define AKB_ALL_COMPONENTS (-1)
akb_status akb_apply_dirichlet(akb_model* model, const uint32_t* nodes,
                               int64_t nb_nodes, int32_t component,
                               const double* values);

/* Kernel slots of one step, for akb_time_kernels. */
enum { AKB_MAX_KERNEL_SLOTS = 8 };
/* Runs nb_steps steps one launch at a time, with CUDA events recorded on the
 * model's stream around every kernel; ms_per_launch[k] receives the mean
 * device time of the step's k-th kernel (0 past the last one). No reference
 * counterpart: the reference has no timers (it measures nothing). */
akb_status akb_time_kernels(akb_model* model, int64_t nb_steps,
                            double* ms_per_launch, int32_t nb_slots);
/* Name of the step's k-th kernel, or "" past the last one. */
const char* akb_kernel_name(const akb_model* model, int32_t slot);

/* ------------------------------------------------------------------------
 * Batches: many independent meshes of one element type stepped together.
 * No counterpart in the reference (it runs one SolidMechanicsModel per
 * process); each instance follows the single-model path exactly: its own
 * material (one per instance), its own time step, the same per-instance
 * patches, so its state is bitwise the one a model of that mesh alone gives.
 * The batch is an akb_model over the union mesh (instances concatenated in
 * order; fields, blocked DOFs, Dirichlet values and akb_solve_steps work on
 * the union arrays). Fast modes only (AKB_MODE_FP64, AKB_MODE_FP32_BULK). */
typedef struct {
  int32_t nb_instances;
  const akb_mesh_desc* meshes;        /* nb_instances meshes, same element type */
  const akb_material_desc* materials; /* one material per instance */
} akb_batch_desc;

akb_status akb_batch_create(const akb_batch_desc* batch, const akb_model_options* options,
                            akb_model** model);
/* node_offsets / element_offsets: nb_instances + 1 entries each, or NULL. */
akb_status akb_batch_get_layout(const akb_model* model, int32_t* nb_instances,
                                int64_t* node_offsets, int64_t* element_offsets);
/* Per-instance time steps (nb_instances values). */
akb_status akb_batch_set_time_steps(akb_model* model, const double* time_steps);
/* getStableTimeStep of every instance (solid_mechanics_model.cc:482-533). */
akb_status akb_batch_get_stable_time_steps(akb_model* model, double* time_steps);
/* getEnergy of every instance, AKB_ENERGY_KINETIC or AKB_ENERGY_POTENTIAL. */
akb_status akb_batch_get_energies(akb_model* model, int32_t kind, double* values);

/* Kinetic energy 1/2 sum(m v^2) of device arrays, allocating no memory.
 * No counterpart in the reference: it serves callers that cannot call
 * cudaMalloc mid-run (inside CUDA stream capture, or under a device-memory
 * budget owned by another allocator). mass and velocity are device arrays of
 * nb_nodes x spatial_dimension doubles (e.g. from akb_field_device_pointer),
 * result a device double the caller provides; work is queued on stream
 * (cudaStream_t, NULL = default stream) and not waited for. The partial sums
 * use a fixed 16 KiB array inside the library, held by every GPU that loads
 * it until exit: nb_nodes above 8 388 608 is rejected
 * (AKB_ERR_INVALID_ARGUMENT); calls that overlap on the GPU race on that
 * array; its device address is looked up again on every call made outside
 * stream capture and cached per device for calls made during one, so one
 * call per device should come before the first capture. */
akb_status akb_kinetic_energy_static(const double* mass, const double* velocity,
                                     int64_t nb_nodes, int32_t spatial_dimension,
                                     double* result, void* stream);

/* Waits for all work queued on the model's stream. */
akb_status akb_synchronize(akb_model* model);

/* ---- Partitioned meshes (one process and GPU per part) -------------------
 * The reference distributes a mesh over MPI ranks with ghost elements and
 * sums the interface nodes' residual contributions across ranks
 * (solid_mechanics_model.cc:94-100, 395-411; ElementSynchronizer). Here a
 * part is a model of its own elements and the nodes they touch;
 * interface_nodes lists its nodes that other parts' elements touch too
 * (local ids, in an order of the caller's choice). Fast modes only
 * (AKB_MODE_FP64, AKB_MODE_FP32_BULK), built-in materials; akb_solve_steps
 * is refused. A step is
 *   akb_part_step_begin   predictor, element forces, this part's nodes
 *                         finished, the interface nodes' partial forces kept;
 *   akb_part_export_forces  out[i*d + c] = this part's internal force on
 *                         interface node i (device array, nb_interface x d);
 *   (the caller sums the exported arrays over all parts, e.g. an all-reduce
 *   on the model's stream, akb_model_get_stream)
 *   akb_part_step_end     in = the summed forces: lumped solve and corrector
 *                         of the interface nodes and the other shared nodes.
 * The lumped mass of an interface node is also a sum over parts: after
 * creation, export it (out[i], nb_interface doubles), sum over parts and
 * import the sum; and set one time step for all parts (the minimum of the
 * parts' stable steps). All calls only queue work on the model's stream. */
akb_status akb_model_create_part(const akb_mesh_desc* mesh, int32_t nb_materials,
                                 const akb_material_desc* materials,
                                 const uint32_t* element_material,
                                 const akb_model_options* options,
                                 const uint32_t* interface_nodes, int64_t nb_interface,
                                 akb_model** model);
akb_status akb_part_step_begin(akb_model* model);
akb_status akb_part_export_forces(akb_model* model, double* device_out);
akb_status akb_part_step_end(akb_model* model, const double* device_in);
akb_status akb_part_export_mass(akb_model* model, double* device_out);
akb_status akb_part_import_mass(akb_model* model, const double* device_in);

/* Neighbour exchange (the send and receive schemes of the reference's
 * ElementSynchronizer, element_synchronizer.hh:52, used by the _smm_stress
 * synchronisation of solid_mechanics_model.cc:395-411): each part sends only
 * the interface rows it shares with each neighbour and sums what it receives.
 *   send_rows[k], k < nb_send: the interface row (index into the
 *       interface_nodes given at creation) of the k-th packed value, the
 *       blocks for the neighbours concatenated in the caller's order;
 *   sum_ptr[i] .. sum_ptr[i+1] (nb_interface + 1 entries): the terms of
 *       interface row i's sum, in the order they are added; sum_src[t] = -1
 *       for this part's own value (exactly once per row), else a row of the
 *       received buffer (nb_recv rows, the neighbours' blocks concatenated).
 * With the terms in ascending part order on every part, all copies of an
 * interface node's sum are equal. Arrays are host arrays, copied. A step is
 * then akb_part_step_begin, akb_part_pack_forces (device_send: nb_send x d
 * doubles), the transfer (e.g. grouped NCCL send/recv on the model's
 * stream), akb_part_step_end_exchange (device_recv: nb_recv x d doubles);
 * the masses are summed once by akb_part_pack_mass (nb_send doubles), the
 * transfer, akb_part_import_mass_exchange (nb_recv doubles). */
akb_status akb_part_set_exchange(akb_model* model, int64_t nb_send, const uint32_t* send_rows,
                                 int64_t nb_recv, const int64_t* sum_ptr,
                                 const int64_t* sum_src);
akb_status akb_part_pack_forces(akb_model* model, double* device_send);
akb_status akb_part_step_end_exchange(akb_model* model, const double* device_recv);
akb_status akb_part_pack_mass(akb_model* model, double* device_send);
akb_status akb_part_import_mass_exchange(akb_model* model, const double* device_recv);

#ifdef __cplusplus
}
#endif

#endif /* AKB_H */
