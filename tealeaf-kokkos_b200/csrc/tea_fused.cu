// Whole-solve path (ext_tea_leaf_solve_): provisional entry point until the fused
// kernels land; it records TEA_ERR_BAD_ARGUMENT.
#include "tea_chunk.cuh"
#include "../../include/tea_b200.h"

namespace tea {
void destroy_fused(Chunk* c) { (void)c; }
}  // namespace tea

extern "C" __attribute__((visibility("default"))) void ext_tea_leaf_solve_(const int* chunk,
                                                                           const tea_solve_params* params,
                                                                           tea_solve_result* result)
{
    (void)chunk;
    (void)params;
    if (result) result->status = 2;
    tea::set_status(2, "ext_tea_leaf_solve_ is not available in this build");
}
