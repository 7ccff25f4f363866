/*
 * lod_oracle.h -- CPU restatement of BioFVM-B's diffusion-decay hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle). Used by tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg as the checker; the product library never
 * links or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks every restated reference
 * function here bit-for-bit against the reference library compiled from its own sources
 * (oracle/_ref, see oracle/Makefile) and against the committed golden fixtures
 * in tests/golden/ that were produced by that library.
 *
 * Field layout everywhere: rho[((i*ny + j)*nz + k)*S + d]   (BioFVM_mesh.cpp:659-665)
 * Face order for masks/values: 0 = x-low, 1 = x-high, 2 = y-low, 3 = y-high,
 * 4 = z-low, 5 = z-high.
 */
#ifndef BFB_LOD_ORACLE_H
#define BFB_LOD_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Thomas factors for one axis of length n (BioFVM_parallel.cpp:780-912). */
void orc_factors(int n, int S, double dt, double dx, const double *D, const double *lambda,
                 double *denom /* n*S */, double *c /* n*S */);

/* apply_dirichlet_conditions (BioFVM_microenvironment.cpp:381-484) with a
 * per-face activation mask face_mask[f*S + d]; the reference is the mask with
 * all six faces equal to dirichlet_activation_vector[d]. values is V*S. */
void orc_dirichlet(double *rho, int nx, int ny, int nz, int S, const double *values,
                   const uint8_t *face_mask);

/* One LOD diffusion-decay step: Dir, X, Dir, Y, Dir, Z, Dir
 * (diffusion_decay_solver__constant_coefficients_LOD_3D, BioFVM_parallel.cpp:693-1395,
 * single rank). Factors come from orc_factors with the same dt. */
void orc_lod_step(double *rho, int nx, int ny, int nz, int S,
                  const double *denx, const double *cx, const double *deny, const double *cy,
                  const double *denz, const double *cz, const double *c1,
                  const double *dir_values, const uint8_t *face_mask);

/* c1[d] = dt*D[d]/dx/dx, evaluated as in BioFVM_parallel.cpp:780-788. */
void orc_constant1(int S, double dt, double dx, const double *D, double *c1);

/* simulate_bulk_sources_and_sinks (BioFVM_microenvironment.cpp:1110-1153). */
void orc_bulk_step(double *rho, int64_t V, int S, double dt, const double *S_rate,
                   const double *T_target, const double *U_rate);

/* Agent binning: is_position_valid (BioFVM_mesh.cpp:204-213) and
 * nearest_voxel_local_index at rank 0 / dims {1,1,1} (BioFVM_parallel.cpp:418-522)
 * followed by the clamp in Basic_Agent::update_voxel_index
 * (BioFVM_basic_agent.cpp:137-153). bbox = {x0, y0, z0, x1, y1, z1}.
 * out_voxel[a] = voxel index, or -1 when assign_position would reject the
 * position (the reference then leaves the agent's previous index in place). */
void orc_bin_agents(int n, const double *pos, const double *bbox, double dx, double dy, double dz,
                    int nx, int ny, int nz, int *out_voxel);

/* Basic_Agent::set_internal_uptake_constants (BioFVM_basic_agent.cpp:155-176). */
void orc_agent_constants(int n, int S, double dt, double dx, double dy, double dz,
                         const double *volume, const double *secretion, const double *uptake,
                         const double *saturation, double *temp1, double *temp2);

/* simulate_secretion_and_uptake for every active agent in list order
 * (BioFVM_basic_agent.cpp:279-300), serial. */
void orc_cells_step(double *rho, int S, int n, const int *voxel, const double *temp1,
                    const double *temp2, const uint8_t *active);

/* Per-substrate sum of rho over voxels, FP64, voxel order. */
void orc_checksum(const double *rho, int64_t V, int S, double *out);

/* Gradient vectors of every substrate at every voxel, out[(n*S + q)*3 + c]
 * (compute_all_gradient_vectors, BioFVM_microenvironment.cpp:1243-1402). */
void orc_gradients(const double *rho, int nx, int ny, int nz, int S, double dx, double *out);

/* Reverse-mode of one orc_lod_step: given lam = dL/d(rho_out), on return
 * lam = dL/d(rho_in); gD[d], gL[d] are incremented by dL/dD_d, dL/dlambda_d.
 * rho_in is the step's input field (left unchanged). */
void orc_lod_step_adjoint(const double *rho_in, double *lam, int nx, int ny, int nz, int S,
                          double dt, double dx, const double *D, const double *lambda,
                          const double *dir_values, const uint8_t *face_mask,
                          double *gD, double *gL);

/* The product's FP32 path restated (not a reference function): n_steps LOD
 * steps Dir, X, Dir, Y, Dir, Z, Dir on an FP32 field, with the reference's
 * FP64 factors (orc_factors) rounded once into FP32 tables, and each line
 * solved in the deviation form u - u_ref with the reciprocal 1/den carried as
 * a hi + lo pair, in exactly the FP32 operations of the CUDA line solver.
 * dir_values (V*S FP64, rounded to FP32 like the device face values) and
 * face_mask (6*S) may both be NULL for no Dirichlet faces. */
void orc_lod_steps_f32(float *rho, int nx, int ny, int nz, int S, double dt, double dx, const double *D,
                       const double *lambda, int n_steps, const double *dir_values, const uint8_t *face_mask);

/* The FP32 path's bulk update and agent update (not reference functions):
 * the arithmetic of orc_bulk_step / orc_cells_step in IEEE binary32, with the
 * FP64 inputs rounded once as the product's host code rounds them. */
void orc_bulk_step_f32(float *rho, int64_t V, int S, double dt, const double *S_rate, const double *T_target,
                       const double *U_rate);
void orc_cells_step_f32(float *rho, int S, int n, const int *voxel, const double *temp1, const double *temp2,
                        const uint8_t *active);

#ifdef __cplusplus
}
#endif
#endif
