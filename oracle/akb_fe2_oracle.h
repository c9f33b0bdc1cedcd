/*
 * akb_fe2_oracle.h -- CPU restatement of the FE^2 building blocks.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA RVE solver and of the
 * MLP kernels, never linked by the product.
 *
 * The reference has no periodic-RVE relaxation and no learned surrogate (its
 * MaterialFE2, extra_packages/extra-materials/src/material_FE2/material_FE2.cc:
 * 84-199, linearises each RVE into a homogenised stiffness); these routines
 * restate the algorithms the CUDA library documents, in FP64 with plain
 * loops, so parity here is "the same algorithm in FP64", not "the
 * reference's numbers": parity unpinned by reference data.
 */
#ifndef AKB_FE2_ORACLE_H
#define AKB_FE2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One periodic voxel RVE solved by damped dynamic relaxation.
 *   n cells per side (even), side L, voxel_material[n^3] (x fastest),
 *   lambda/mu/kind per material (kind 0 small-strain elastic, 1 neo-Hookean),
 *   grad_u: macroscopic displacement gradient H, column-major (H[i + 3 j] =
 *   du_i/dX_j), F = I + H;
 *   fluct: n^3 x 3 periodic fluctuation, node-major (in: start, out: end);
 *   stress: homogenised first Piola-Kirchhoff stress, column-major.
 * tolerance < 0 runs exactly max_iterations updates. Returns the number of
 * updates; *residual is the final relative residual. */
int32_t oracle_rve_solve(int32_t n, double L, const uint8_t* voxel_material,
                         int32_t nb_materials, const double* lambda, const double* mu,
                         const int32_t* kind, const double* grad_u, double* fluct,
                         int32_t max_iterations, int32_t check_interval, double tolerance,
                         double time_step_factor, double damping_factor, double* stress,
                         double* residual);

/* Per-instance time step and damping coefficient of the relaxation. */
void oracle_rve_parameters(int32_t n, double L, int32_t nb_materials, const double* lambda,
                           const double* mu, const int32_t* kind, const double* grad_u,
                           double time_step_factor, double damping_factor, double* dt,
                           double* damping);

/* Homogenised stress of one RVE state (no relaxation). */
void oracle_rve_stress(int32_t n, double L, const uint8_t* voxel_material,
                       const double* lambda, const double* mu, const int32_t* kind,
                       const double* grad_u, const double* fluct, double* stress,
                       double* internal_force /* n^3 x 3 or null */);

/* The surrogate MLP (akantu_b200/csrc/akb_mlp.cu) in FP64: nin -> width
 * (SiLU) x nhidden -> nout, parameters in the library's layout (per layer
 * W row-major [out][in], then b). With emulate_bf16 the values the tensor
 * cores consume are rounded to BF16 where the CUDA kernels round them (the
 * normalised input, weights, hidden activations, dY and dZ) and the output
 * and pre-activations to FP32; sums stay FP64. scaling: in_shift, in_scale
 * [nin], out_shift, out_scale [nout]. y: [nb][nout]. */
void oracle_mlp_forward(int32_t nin, int32_t nout, int32_t width, int32_t nhidden,
                        const float* params, const float* scaling, int64_t nb, const double* x,
                        double* y, int32_t emulate_bf16);
/* Loss (mean squared error of the normalised outputs) and its gradient. */
double oracle_mlp_gradients(int32_t nin, int32_t nout, int32_t width, int32_t nhidden,
                            const float* params, const float* scaling, int64_t nb,
                            const double* x, const double* target, double* grad,
                            int32_t emulate_bf16);

#ifdef __cplusplus
}
#endif

#endif
