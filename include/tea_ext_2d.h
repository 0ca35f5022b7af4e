/*
 * tea_ext_2d.h -- the drop-in C ABI of libtea2d_b200.so.
 *
 * Each declaration replaces the same-named extern "C" function of the reference's
 * 2D extension layer (crtrott/TeaLeaf-Kokkos, tealeaf_2d/ext_chunk.cpp and
 * tealeaf_2d/ext_core.cpp), cited per entry.  Signatures, argument meaning and
 * call order are the reference's: gfortran name mangling (trailing underscore),
 * every argument by pointer, 1-based chunk ids.  A call that returns data to the
 * host (a reduction, the field summary, a packed face) returns when its kernels
 * have finished; a call that only updates fields returns when its kernels are
 * queued on the chunk's stream, like the reference's Kokkos parallel_for
 * (tealeaf_2d/ext_core.cpp:21-24).  The fields live in device memory (one B200)
 * instead of Kokkos Views; results are the same numbers (see the parity tests).
 *
 * Two arguments are declared `bool*` in the reference but receive Fortran
 * INTEGER literals 1/0 from the driver (tealeaf_2d/tea_solve.f90:262,670); they
 * are declared `const void*` here and read as the reference reads them: the first
 * byte, non-zero = true.
 *
 * Additive entry points (no reference counterpart) are in tea_b200.h.
 */
#ifndef TEA_EXT_2D_H
#define TEA_EXT_2D_H

#include "tea_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* tealeaf_2d/ext_chunk.cpp:19 -- create chunk (xMax x yMax interior cells); the next
 * chunk id is returned implicitly (1 for the first call, as in the reference). */
void ext_init_(int* xMax, int* yMax, int* rank);
/* tealeaf_2d/ext_chunk.cpp:29 -- release every chunk. */
void ext_finalise_(void);

/* tealeaf_2d/ext_core.cpp:33 -- vertex/cell coordinates, volume and face areas. */
void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin,
                           const double* dx, const double* dy);
/* tealeaf_2d/ext_core.cpp:57 -- paint states 1..numStates (last wins); u = energy0*density. */
void ext_generate_chunk_(const int* chunk, const int* numStates,
                         const double* stateDensity, const double* stateEnergy,
                         const double* stateXMin, const double* stateXMax,
                         const double* stateYMin, const double* stateYMax,
                         const double* stateRadius, const int* stateGeometry,
                         const int* rectParam, const int* circParam, const int* pointParam);
/* tealeaf_2d/ext_core.cpp:130 -- (sum vol, sum vol*rho, sum vol*rho*e0, sum vol*rho*u). */
void ext_field_summary_kernel_(const int* chunk, double* vol, double* mass, double* ie,
                               double* temp);
/* tealeaf_2d/ext_core.cpp:151 -- pack (pack != 0) or unpack a face of the selected fields
 * to/from the host buffer at the given per-field offsets. */
void ext_pack_message_(const int* chunk, const int* fields, const int* offsets,
                       const int* depth, const int* face, double* buffer, const void* pack);
/* tealeaf_2d/ext_core.cpp:249 -- energy = energy0 over the padded array. */
void ext_set_field_kernel_(const int* chunk);
/* tealeaf_2d/ext_core.cpp:260 -- u0 = u on the inner domain. */
void ext_solver_copy_u_(const int* chunk);
/* tealeaf_2d/ext_core.cpp:271 -- r = u0 - A u on the inner domain. */
void ext_calculate_residual_(const int* chunk);
/* tealeaf_2d/ext_core.cpp:282 -- norm = sum buf^2, buf = r if *normArray else u0. */
void ext_calculate_2norm_(const int* chunk, double* norm, const void* normArray);
/* tealeaf_2d/ext_core.cpp:295 -- energy = u / density on the inner domain. */
void ext_solver_finalise_(const int* chunk);
/* tealeaf_2d/ext_core.cpp:305 -- reflective halo update of the selected fields on every
 * face whose neighbour is EXTERNAL_FACE (-1), depth 1 or 2. */
void ext_update_halo_kernel_(const int* chunk, const int* chunkNeighbours,
                             const int* fields, const int* depth);
/* tealeaf_2d/ext_core.cpp:340 -- Jacobi set-up: u0 = u = rho*e, Kx/Ky from rho or 1/rho. */
void ext_jacobi_kernel_init_(const int* chunk, const int* coefficient, const double* dt);
/* tealeaf_2d/ext_core.cpp:362 -- one Jacobi sweep; error = sum |u_new - u_old|. */
void ext_jacobi_kernel_solve_(const int* chunk, double* error);
/* tealeaf_2d/ext_core.cpp:377 -- CG set-up: u = rho*e, Kx/Ky, w = A u, r = u - w,
 * p = r (or z = Mi r), rro = sum r.p. */
void ext_cg_solver_init_(const int* chunk, const int* coefficient, const int* preconditioner,
                         double* dt, double* rro);
/* tealeaf_2d/ext_core.cpp:417 -- w = A p, pw = sum p.w. */
void ext_cg_calc_w_(const int* chunk, double* pw);
/* tealeaf_2d/ext_core.cpp:433 -- u += alpha p, r -= alpha w, rrn = sum r.r (or r.z). */
void ext_cg_calc_ur_(const int* chunk, const double* alpha, double* rrn);
/* tealeaf_2d/ext_core.cpp:451 -- p = beta p + r (or z). */
void ext_cg_calc_p_(const int* chunk, const double* beta);
/* tealeaf_2d/ext_core.cpp:468 -- store Chebyshev alphas/betas, first Chebyshev step. */
void ext_cheby_solver_init_(const int* chunk, double* alphas, double* betas,
                            const double* theta, const int* preconditioner,
                            const int* maxChebyIters);
/* tealeaf_2d/ext_core.cpp:501 -- one Chebyshev iteration with coefficient index step-1. */
void ext_cheby_solver_iterate_(const int* chunk, const int* chebyCalcStep);
/* tealeaf_2d/ext_core.cpp:519 -- store PPCG alphas/betas and theta. */
void ext_ppcg_init_(const int* chunk, double* alphas, double* betas, const double* theta,
                    const int* maxChebyIters);
/* tealeaf_2d/ext_core.cpp:543 -- sd = (Mi r or r) / theta. */
void ext_ppcg_init_sd_(const int* chunk);
/* tealeaf_2d/ext_core.cpp:554 -- r -= A sd, u += sd, sd = alpha sd + beta (Mi r or r). */
void ext_ppcg_inner_(const int* chunk, int* currentStep);

#ifdef __cplusplus
}
#endif

#endif /* TEA_EXT_2D_H */
