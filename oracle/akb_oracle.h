/*
 * akb_oracle.h -- CPU restatement of Akantu's explicit lumped-mass path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle the CUDA library is checked
 * against, and the timed CPU baseline. Nothing in the product links it.
 *
 * It restates, in FP64 and in the reference's operation order, the functions
 * listed in akb_oracle.cc (each cites the reference file:line it follows). It
 * is pinned by the reference's own golden data: the 402-row explicit
 * model-solver table, the explicit linear patch test, the lumped-mass test.
 */
#ifndef AKB_ORACLE_H
#define AKB_ORACLE_H

#include <stdint.h>

#include "../include/akb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_model oracle_model;

/* Builds the model and runs initFull(_explicit_lumped_mass): shape
 * derivatives and detJ*w on the reference coordinates. Returns NULL and sets
 * *status on failure (AKB_ERR_NEGATIVE_JACOBIAN, AKB_ERR_BAD_MESH). */
oracle_model* oracle_create(const akb_mesh_desc* mesh, int32_t nb_materials,
                            const akb_material_desc* materials,
                            const uint32_t* element_material,
                            int32_t* status);
void oracle_destroy(oracle_model* m);

/* Direct pointers to the model-owned arrays (reference Array layout). */
double* oracle_field(oracle_model* m, int32_t field);
uint8_t* oracle_blocked(oracle_model* m);
int64_t oracle_field_size(oracle_model* m, int32_t field);

void oracle_assemble_mass_lumped(oracle_model* m);
double oracle_stable_time_step(oracle_model* m);
void oracle_set_time_step(oracle_model* m, double dt);
/* Host threads (OpenMP builds only); the multi-threaded path is bitwise
 * equal to the single-threaded one. */
void oracle_set_threads(oracle_model* m, int32_t threads);
void oracle_solve_step(oracle_model* m);
void oracle_solve_steps(oracle_model* m, int64_t n);
void oracle_assemble_internal_forces(oracle_model* m);
void oracle_compute_stresses(oracle_model* m);
double oracle_energy(oracle_model* m, int32_t kind);

/* Seconds of wall time for n steps (steady_clock), for the CPU baseline. */
double oracle_time_steps(oracle_model* m, int64_t n);

#ifdef __cplusplus
}
#endif

#endif
