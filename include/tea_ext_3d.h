/*
 * tea_ext_3d.h -- the drop-in C ABI of libtea3d_b200.so.
 *
 * Each declaration replaces the same-named extern "C" function of the reference's
 * 3D extension layer (crtrott/TeaLeaf-Kokkos, tealeaf_3d/ext_chunk.cpp and
 * tealeaf_3d/ext_core.cpp), cited per entry.  Conventions as in tea_ext_2d.h:
 * gfortran mangling, by-pointer arguments, 1-based chunk ids, field-only calls
 * returning once their kernels are queued;
 * `bool*` arguments of the reference are `const void*` read by their first byte.
 * The 3D ABI differs from the 2D one in ext_init_ (z extent), ext_initialise_chunk_
 * (zMin, dz), ext_generate_chunk_ (stateZMin/stateZMax), ext_pack_message_
 * (fieldType) and in having six faces (BACK=5, FRONT=6).
 */
#ifndef TEA_EXT_3D_H
#define TEA_EXT_3D_H

#include "tea_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* tealeaf_3d/ext_chunk.cpp:20 */
void ext_init_(int* xMax, int* yMax, int* zMax, int* rank);
/* tealeaf_3d/ext_chunk.cpp:31 */
void ext_finalise_(void);

/* tealeaf_3d/ext_core.cpp:33 */
void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin,
                           const double* zMin, const double* dx, const double* dy,
                           const double* dz);
/* tealeaf_3d/ext_core.cpp:61 */
void ext_generate_chunk_(const int* chunk, const int* numStates,
                         const double* stateDensity, const double* stateEnergy,
                         const double* stateXMin, const double* stateXMax,
                         const double* stateYMin, const double* stateYMax,
                         const double* stateZMin, const double* stateZMax,
                         const double* stateRadius, const int* stateGeometry,
                         const int* rectParam, const int* circParam, const int* pointParam);
/* tealeaf_3d/ext_core.cpp:147 */
void ext_field_summary_kernel_(const int* chunk, double* vol, double* mass, double* ie,
                               double* temp);
/* tealeaf_3d/ext_core.cpp:168 */
void ext_pack_message_(const int* chunk, const int* fields, const int* offsets,
                       const int* depth, const int* face, const int* fieldType,
                       double* buffer, const void* pack);
/* tealeaf_3d/ext_core.cpp:276 */
void ext_set_field_kernel_(const int* chunk);
/* tealeaf_3d/ext_core.cpp:287 */
void ext_solver_copy_u_(const int* chunk);
/* tealeaf_3d/ext_core.cpp:298 */
void ext_calculate_residual_(const int* chunk);
/* tealeaf_3d/ext_core.cpp:310 */
void ext_calculate_2norm_(const int* chunk, double* norm, const void* normArray);
/* tealeaf_3d/ext_core.cpp:323 */
void ext_solver_finalise_(const int* chunk);
/* tealeaf_3d/ext_core.cpp:334 -- 6 neighbours; only the inner part of each face. */
void ext_update_halo_kernel_(const int* chunk, const int* chunkNeighbours,
                             const int* fields, const int* depth);
/* tealeaf_3d/ext_core.cpp:371 */
void ext_jacobi_kernel_init_(const int* chunk, const int* coefficient, const double* dt);
/* tealeaf_3d/ext_core.cpp:394 */
void ext_jacobi_kernel_solve_(const int* chunk, double* error);
/* tealeaf_3d/ext_core.cpp:409 */
void ext_cg_solver_init_(const int* chunk, const int* coefficient, const int* preconditioner,
                         double* dt, double* rro);
/* tealeaf_3d/ext_core.cpp:450 */
void ext_cg_calc_w_(const int* chunk, double* pw);
/* tealeaf_3d/ext_core.cpp:462 */
void ext_cg_calc_ur_(const int* chunk, const double* alpha, double* rrn);
/* tealeaf_3d/ext_core.cpp:476 */
void ext_cg_calc_p_(const int* chunk, const double* beta);
/* tealeaf_3d/ext_core.cpp:488 */
void ext_cheby_solver_init_(const int* chunk, double* alphas, double* betas,
                            const double* theta, const int* preconditioner,
                            const int* maxChebyIters);
/* tealeaf_3d/ext_core.cpp:521 */
void ext_cheby_solver_iterate_(const int* chunk, const int* chebyCalcStep);
/* tealeaf_3d/ext_core.cpp:539 */
void ext_ppcg_init_(const int* chunk, double* alphas, double* betas, const double* theta,
                    const int* maxChebyIters);
/* tealeaf_3d/ext_core.cpp:563 */
void ext_ppcg_init_sd_(const int* chunk);
/* tealeaf_3d/ext_core.cpp:574 */
void ext_ppcg_inner_(const int* chunk, int* currentStep);

#ifdef __cplusplus
}
#endif

#endif /* TEA_EXT_3D_H */
