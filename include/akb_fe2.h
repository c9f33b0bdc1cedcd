/*
 * akb_fe2.h -- FE^2 entry points of libakb.so.
 *
 * 1. User materials. A model whose materials are AKB_MATERIAL_USER takes its
 *    quadrature-point stresses from the caller: the explicit step is split
 *    around Material::computeStress (material.hh:110, called from
 *    Material::computeAllStresses, material.cc:254-279), so a material
 *    written outside the library -- here the FE^2 macro material that asks
 *    RVEs or their learned surrogate for the stress -- plugs into the same
 *    step as the built-in laws.
 *
 * 2. Periodic RVEs. The micro problem of FE^2 (the reference's MaterialFE2 /
 *    SolidMechanicsModelRVE, extra_packages/extra-materials/src/material_FE2/
 *    material_FE2.cc:84-199 and solid_mechanics_model_RVE.hh:44-93, which
 *    apply the macroscopic displacement gradient to an RVE and homogenise):
 *    a cube of n^3 hexahedron_8 voxels with periodic nodes, loaded by a
 *    macroscopic displacement gradient H, relaxed to equilibrium by damped
 *    dynamic relaxation, returning the volume average of the first
 *    Piola-Kirchhoff stress. Thousands of RVEs are solved in one launch.
 *
 * Tensors are 3 x 3 column-major per point, like the reference's Matrix
 * (aka_types.hh:929-944): entry (i, j) at [i + 3 j]; grad_u(i, j) = du_i/dX_j.
 */
#ifndef AKB_FE2_H
#define AKB_FE2_H

#include "akb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ user */

/* First half of a step of a model whose materials are AKB_MATERIAL_USER
 * (AKB_MODE_FP64 only): the central-difference predictor, then the
 * displacement gradient at every quadrature point into AKB_FIELD_GRAD_U
 * (device: akb_field_device_pointer). The caller then writes, on the model's
 * stream (akb_model_get_stream), the stress conjugate to grad u into
 * AKB_FIELD_STRESS: Cauchy stress for a small-strain material
 * (finite_deformation = 0), first Piola-Kirchhoff stress for a finite one. */
akb_status akb_step_begin(akb_model* model);
/* Second half: internal forces -sum_q stress grad N_a detJ w from
 * AKB_FIELD_STRESS, lumped solve and corrector. */
akb_status akb_step_end(akb_model* model);
/* The cudaStream_t the model's work is queued on. */
akb_status akb_model_get_stream(akb_model* model, void** stream);

/* ------------------------------------------------------------------- RVE */

typedef struct {
  int32_t cells;                      /* n voxels per side (even, 2..64) */
  int32_t nb_materials;               /* 1..8 */
  double length;                      /* side L of the cube */
  const uint8_t* voxel_material;      /* [n^3], voxel (x, y, z) at x + n (y + n z) */
  const akb_material_desc* materials; /* elastic (small strain) or neo-Hookean */
} akb_rve_desc;

typedef struct {
  int32_t precision_mode;   /* AKB_MODE_FP32_BULK (default) or AKB_MODE_FP64 (n <= 12) */
  int32_t device;           /* CUDA device ordinal */
  void* stream;             /* cudaStream_t; NULL = library-owned stream */
  int32_t max_iterations;   /* 0: 2000 */
  int32_t check_interval;   /* residual checked every k updates; 0: 10 */
  double tolerance;         /* relative residual to stop at; 0: 1e-4; < 0: run
                               exactly max_iterations updates */
  double time_step_factor;  /* 0: 0.6 */
  double damping_factor;    /* 0: 0.6 */
} akb_rve_options;

typedef struct {
  int32_t cells;
  int32_t precision_mode;
  int64_t nb_nodes;          /* n^3 unique periodic nodes */
  double volume_fraction[8]; /* voxel fraction of each material */
  int64_t shared_bytes;      /* shared memory of one RVE solve */
} akb_rve_info;

typedef struct akb_rve akb_rve;

akb_status akb_rve_create(const akb_rve_desc* desc, const akb_rve_options* options,
                          akb_rve** out);
akb_status akb_rve_destroy(akb_rve* rve);
akb_status akb_rve_get_info(const akb_rve* rve, akb_rve_info* info);

/* Solves nb RVE problems, all arrays on the device, queued on stream (NULL =
 * the RVE's stream) and not waited for:
 *   grad_u     [nb][9]        macroscopic displacement gradients H (F = I + H);
 *   fluctuation [nb][n^3][3]  periodic fluctuation, float (FP32 mode) or
 *                             double (FP64): read as the start, overwritten by
 *                             the solution; NULL starts from zero;
 *   stress     [nb][9]        homogenised first Piola-Kirchhoff stress;
 *   iterations [nb]           updates done (may be NULL);
 *   residual   [nb]           final max|f| / (h^2 max(mu) max(|H_ij|, 1e-6))
 *                             (may be NULL; +inf if the relaxation diverged). */
akb_status akb_rve_solve(akb_rve* rve, int64_t nb, const double* grad_u, void* fluctuation,
                         double* stress, int32_t* iterations, double* residual, void* stream);

/* akb_rve_solve for the points index[0 .. min(*count, capacity)) of arrays
 * over capacity points (grad_u [capacity][9], fluctuation
 * [capacity][n^3][3] or NULL, stress [capacity][9], iterations / residual
 * [capacity] or NULL; entries of other points are left alone). index and
 * count are device arrays read by the kernel (e.g. written by
 * akb_mlp_stress earlier on the same stream): no host round trip, and an
 * empty list costs one short launch. */
akb_status akb_rve_solve_indexed(akb_rve* rve, int64_t capacity, const int32_t* index,
                                 const int32_t* count, const double* grad_u, void* fluctuation,
                                 double* stress, int32_t* iterations, double* residual,
                                 void* stream);

/* Homogenised stress and internal force of given states, no relaxation
 * (internal_force [nb][n^3][3] double, may be NULL). */
akb_status akb_rve_stress(akb_rve* rve, int64_t nb, const double* grad_u,
                          const void* fluctuation, double* stress, double* internal_force,
                          void* stream);

/* ---------------------------------------------------------- surrogate */

/* A multilayer perceptron nb_inputs -> width (SiLU) x nb_hidden -> nb_outputs
 * run on the tensor cores (BF16 operands, FP32 accumulation, FP32 master
 * weights): the learned map grad_u -> homogenised stress that replaces RVE
 * solves inside its training envelope. Inputs and outputs are normalised
 * inside (x' = (x - in_shift) in_scale, y = y' out_scale + out_shift).
 * Parameters are FP32, layer by layer: W_l (rows = outputs, row-major), then
 * b_l. Supported: 1..16 inputs and outputs, width 128 or 256, 1..5 hidden
 * layers. */
typedef struct akb_mlp akb_mlp;

akb_status akb_mlp_create(int32_t nb_inputs, int32_t nb_outputs, int32_t width,
                          int32_t nb_hidden, int32_t device, void* stream, akb_mlp** out);
akb_status akb_mlp_destroy(akb_mlp* mlp);
akb_status akb_mlp_get_parameter_count(const akb_mlp* mlp, int64_t* count);
/* Host arrays; setting the parameters resets the optimiser state. */
akb_status akb_mlp_set_parameters(akb_mlp* mlp, const float* values, int64_t count);
akb_status akb_mlp_get_parameters(akb_mlp* mlp, float* values, int64_t count);
akb_status akb_mlp_set_scaling(akb_mlp* mlp, const float* in_shift, const float* in_scale,
                               const float* out_shift, const float* out_scale);
/* y[nb][nb_outputs] = network(x[nb][nb_inputs]), device FP64 arrays, queued
 * on stream (NULL = the network's stream). */
akb_status akb_mlp_forward(akb_mlp* mlp, int64_t nb, const double* x, double* y, void* stream);
/* The surrogate as MaterialFE2's stress map, in one launch: for nb Gauss
 * points, grad_u [nb][9] (column-major H = du/dX per point, as
 * AKB_FIELD_GRAD_U) -> stress [nb][9] (column-major first Piola-Kirchhoff
 * P = |H| y, y the network's output for the inputs (H / r, log r),
 * r = max(|H|, 1e-8), |H| the Frobenius norm). Needs 10 inputs and 9
 * outputs. With fallback_index / fallback_count (device int32, nb entries /
 * one), the points outside the training envelope (max |H_ij| > amplitude or
 * det(I + H) < min_det) are listed in fallback_index[0 .. *fallback_count)
 * (in no particular order; the count is zeroed first), ready for
 * akb_rve_solve_indexed; both NULL skips the test. Queued on stream. */
akb_status akb_mlp_stress(akb_mlp* mlp, int64_t nb, const double* grad_u, double* stress,
                          double amplitude, double min_det, int32_t* fallback_index,
                          int32_t* fallback_count, void* stream);
/* Mean squared error of the normalised outputs against target (device FP64
 * [nb][nb_outputs]) and its gradient (host, parameter layout; may be NULL). */
akb_status akb_mlp_gradients(akb_mlp* mlp, int64_t nb, const double* x, const double* target,
                             float* grad, float* loss);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on that loss. */
akb_status akb_mlp_train_step(akb_mlp* mlp, int64_t nb, const double* x, const double* target,
                              float learning_rate, float* loss);
/* The same step in two halves, for data-parallel training (one process and
 * GPU per rank, each with its share of the minibatch): compute_gradients
 * leaves the gradient of the mean loss over its nb samples in a device array
 * of nb_parameters floats (parameter layout, gradient_device_pointer; valid
 * until the next call on this network), which the caller may average over
 * ranks in place (e.g. an all-reduce on the network's stream), then
 * apply_gradients takes one Adam step with it. compute + apply is
 * akb_mlp_train_step. */
akb_status akb_mlp_compute_gradients(akb_mlp* mlp, int64_t nb, const double* x,
                                     const double* target, float* loss);
akb_status akb_mlp_gradient_device_pointer(akb_mlp* mlp, float** grad);
akb_status akb_mlp_apply_gradients(akb_mlp* mlp, float learning_rate);

#ifdef __cplusplus
}
#endif

#endif /* AKB_FE2_H */
