/*
 * tea_b200.h -- additive C-ABI entry points shared by the 2D and 3D libraries
 * (libtea2d_b200.so, libtea3d_b200.so).  The reference's own ext_* entry points
 * are declared in tea_ext_2d.h / tea_ext_3d.h; everything here is new and has
 * no counterpart in tealeaf_2d|3d/ext_core.cpp unless a line says otherwise.
 *
 * Conventions follow the reference ABI: Fortran-callable names carry a trailing
 * underscore, every argument is passed by pointer, chunk ids are 1-based.
 */
#ifndef TEA_B200_H
#define TEA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Field ids.  1..6 are the reference's FIELD_* ids (tealeaf_2d/ext_shared.hpp:19-25,
 * tealeaf_3d/ext_shared.hpp:21-27); 7..15 name the remaining chunk arrays of
 * TeaLeafChunk (tealeaf_2d/ext_chunk.hpp:28-53). */
enum {
    TEA_FIELD_DENSITY = 1,
    TEA_FIELD_ENERGY0 = 2,
    TEA_FIELD_ENERGY1 = 3,
    TEA_FIELD_U = 4,
    TEA_FIELD_P = 5,
    TEA_FIELD_SD = 6,
    TEA_FIELD_U0 = 7,
    TEA_FIELD_R = 8,
    TEA_FIELD_W = 9,
    TEA_FIELD_Z = 10,
    TEA_FIELD_MI = 11,
    TEA_FIELD_KX = 12,
    TEA_FIELD_KY = 13,
    TEA_FIELD_KZ = 14, /* 3D only */
    TEA_FIELD_VOLUME = 15
};

/* Status codes reported by ext_get_status_.  The reference aborts the process on
 * misuse (abort(), tealeaf_2d/ext_core.cpp:571-584); this library still aborts on
 * the same fatal misuse but records device-side and numerical failures here. */
enum {
    TEA_OK = 0,
    TEA_ERR_BAD_CHUNK = 1,      /* chunk id not initialised */
    TEA_ERR_BAD_ARGUMENT = 2,   /* unknown field/face/solver, sizes out of range */
    TEA_ERR_CUDA = 3,           /* a CUDA runtime call failed */
    TEA_ERR_NONFINITE = 4,      /* NaN/Inf reached a reduction (pw, rrn, error) */
    TEA_ERR_EIGEN = 5,          /* tqli failed or produced a negative eigenvalue */
    TEA_ERR_NO_DEVICE = 6,      /* no CUDA device visible */
    TEA_ERR_NOT_CONVERGED = 7   /* informational: max_iters reached */
};

/* Inspection: copy a whole chunk array between the device and a host buffer laid
 * out as the reference lays it out (flat, x fastest, HALO_PAD=2 on every side:
 * dims = {nx+4, ny+4, nz+4 (1 in 2D)}).  Return 0 on success. */
int tea_chunk_dims_(const int* chunk, int* dims);
int tea_read_field_(const int* chunk, const int* field, double* out);
int tea_write_field_(const int* chunk, const int* field, const double* in);

/* Last recorded status (0 = TEA_OK) and clear it.  Waits for the kernels still queued
 * on every chunk's stream first, so that their faults are included. */
void ext_get_status_(int* status);
/* Message for the last non-zero status (empty string if none). */
const char* tea_last_error(void);

/* The chunk's CUDA stream (a cudaStream_t); every entry point of the chunk runs on it. */
int tea_chunk_stream_(const int* chunk, void** stream);

/* Measurement hook: `reps` back-to-back launches of one fused kernel of the whole-solve
 * path on the chunk's stream, between two CUDA events, on the chunk's current fields
 * (which it modifies).  kernel: 1 PPCG inner step, 2 CG/PPCG sweep A, 3 Chebyshev
 * iteration, 4 Jacobi sweep, 5 CG sweep B, 6 two Chebyshev iterations in one pass (2D;
 * in 3D one iteration), and the FP32 inner-solve kernels of the precision form: 7 CG
 * sweep A, 8 CG sweep B, 9 two Chebyshev iterations (3D: one); 10 two PPCG inner steps
 * in one pass.  Writes the mean milliseconds per launch. */
void tea_kernel_timing_(const int* chunk, const int* kernel, const int* reps, double* ms_per_launch);

/* Host<->device bytes the library has moved for the chunk so far: state tables,
 * coefficients, scalars and results (the field arrays never leave the device). */
int tea_transfer_bytes_(const int* chunk, long long* h2d, long long* d2h);

/* Allocation-free 2-norm, for callers whose device memory belongs to their own pool
 * allocator and who therefore cannot let a library call cudaMalloc (and who hold their
 * fields in their own buffers, not in a chunk of this library).  No counterpart in the
 * reference: it computes what ext_calculate_2norm_ computes (sum of v^2 over the inner
 * domain, Calculate2Norm of tealeaf_2d/ext_solver_methods.hpp) on the caller's device
 * array `field`, laid out as the reference lays out a chunk array (flat, x fastest,
 * HALO_PAD = 2 on every side: (nx+4) x (ny+4) [x (nz+4)]; nz is ignored in 2D), and
 * writes the result to the caller's device double `norm`, on `stream` (NULL: the legacy
 * default stream); the call returns without waiting.  It allocates nothing: its
 * reduction scratch is a static device array of 128 KB per GPU, held until the process
 * exits, which limits one call to at most 16,777,216 inner cells (larger sizes return
 * TEA_ERR_BAD_ARGUMENT with a message).  The first call on each device looks the array up
 * (cudaGetSymbolAddress) and should come before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race.  Returns a TEA_* status. */
int tea_2norm_noalloc_(const double* field, const int* nx, const int* ny, const int* nz, double* norm,
                       void* stream);

/* Face packing for a halo exchange between ranks: the arguments and meaning of the 2D
 * ext_pack_message_ (tealeaf_2d/ext_core.cpp:151; the 3D library takes the same seven
 * arguments, without fieldType) with one difference: in 2D the bottom (3) and top (4) faces
 * are packed from, and unpacked into, the inner columns 2..nx+1.  The reference's 2D
 * packer (TopBottomPacker, tealeaf_2d/ext_pack_kernel.hpp:17-44) starts those rows at padded
 * column 0, so the last two inner columns of each exchanged halo row are never sent;
 * ext_pack_message_ keeps that behaviour for parity, and the slab driver uses this one.
 * Every other face, and every 3D face, is packed exactly as ext_pack_message_ packs it. */
void tea_pack_face_(const int* chunk, const int* fields, const int* offsets, const int* depth, const int* face,
                    double* buffer, const void* pack);

/* Solver ids for the whole-solve entry point. */
enum {
    TEA_SOLVER_JACOBI = 1,
    TEA_SOLVER_CG = 2,
    TEA_SOLVER_CHEBYSHEV = 3,
    TEA_SOLVER_PPCG = 4
};

/* Inputs of one implicit solve: the tea.in keywords that tea_leaf() reads
 * (tealeaf_2d/tea_solve.f90:36-605, defaults at tealeaf_2d/read_input.f90:49-80), plus the
 * precision form. */
typedef struct {
    int solver;             /* TEA_SOLVER_* */
    int coefficient;        /* 1 = CONDUCTIVITY (w = rho), 2 = RECIP_CONDUCTIVITY (w = 1/rho) */
    int preconditioner;     /* tl_preconditioner_on: diagonal (Jacobi) preconditioner */
    int max_iters;          /* tl_max_iters */
    int ch_cg_presteps;     /* tl_ch_cg_presteps */
    int ch_cg_errswitch;    /* tl_ch_cg_errswitch */
    int ppcg_inner_steps;   /* tl_ppcg_inner_steps */
    int check_result;       /* tl_check_result */
    double dt;              /* timestep */
    double eps;             /* absolute threshold on the solver's error (sum r^2 or sum r.z) */
    double ch_cg_epslim;    /* tl_ch_cg_epslim */
    double eps_rel;         /* > 0: replace eps by eps_rel^2 * sum(u0^2) each solve */
    int precision;          /* TEA_PRECISION_FP64 (the reference's arithmetic) or
                               TEA_PRECISION_FP32_REFINED */
    int inner_max_iters;    /* FP32_REFINED: inner iterations per correction, 0 = no limit */
    double inner_tol;       /* FP32_REFINED: relative drop of the inner residual per
                               correction, 0 = 1e-4; a correction also stops once its
                               sum r^2 is below a tenth of the outer target */
    int inner_solver;       /* FP32_REFINED, corrections after the first (CG) one:
                               TEA_INNER_DECK (0) the deck's method -- Chebyshev for
                               Chebyshev decks, PPCG for PPCG decks (an even number
                               of inner steps; else Chebyshev); TEA_INNER_CHEBYSHEV (1) Chebyshev
                               for both */
    int reserved[3];        /* must be zero */
} tea_solve_params;

enum { TEA_INNER_DECK = 0, TEA_INNER_CHEBYSHEV = 1 };

/* Precision forms of ext_tea_leaf_solve_. */
enum {
    /* FP64 throughout, bit-identical to the per-call ext_* sequence. */
    TEA_PRECISION_FP64 = 0,
    /* Defect correction: the outer residual r = b - A u, the update u += d, the sums
     * that decide convergence (tested on the true FP64 residual) and everything after
     * the solve stay FP64; each correction A d = r is solved by CG in FP32 storage and
     * arithmetic, with its dot products accumulated in double-double.  The solver
     * setting selects nothing here (the inner solver is CG); max_iters bounds the total
     * of inner iterations. */
    TEA_PRECISION_FP32_REFINED = 1
};

/* Outputs of one implicit solve. */
typedef struct {
    int iterations;         /* the "Iteration count" that tea_leaf() prints (n-1); for
                               FP32_REFINED the inner iterations in total */
    int status;             /* TEA_* status of this solve */
    int cg_steps;           /* CG iterations before a Chebyshev/PPCG switch */
    int cheby_steps;        /* Chebyshev iterations or PPCG outer iterations after it */
    int switch_step;        /* n at the switch, 0 if none */
    int est_itc;            /* Chebyshev iteration estimate, 0 if none */
    double error;           /* final error (FP32_REFINED: true residual sum r^2) */
    double exact_error;     /* sum (u0 - A u)^2 when check_result is set, else 0 */
    double eps_used;        /* the absolute threshold that was applied */
    double eigmin, eigmax;  /* scaled eigenvalue bounds at the switch (0 if none) */
    int corrections;        /* FP32_REFINED: outer corrections */
    int warm_start_used;    /* 1 when the solve started from an attached network's guess */
    double warm_r0_plain;   /* with a network attached: sum r^2 of the start u = u0
                               (0 on a timestep the back-off skipped) */
    double warm_r0_guess;   /* ... and of the start u = u0 + the network's du */
    int inner_solver;       /* FP32_REFINED: inner solver of the last correction: 0 CG,
                               1 Chebyshev, 2 PPCG */
    int pad;
    double reserved[4];
} tea_solve_result;

/* Whole implicit solve of one timestep on the device: the control flow of
 * tea_leaf() (tealeaf_2d/tea_solve.f90:36-605, tealeaf_3d/tea_solve.f90:36-653),
 * from the depth-2 halo update of energy/density to ext_solver_finalise_ and the
 * final energy halo update, with the iteration loop captured in CUDA graphs and
 * the scalar recurrences and convergence test evaluated on the device.  Single
 * chunk only (every face external).  Replaces the per-iteration sequence of
 * ext_cg_calc_w_/ext_cg_calc_ur_/ext_cg_calc_p_/... calls that the Fortran driver
 * makes; produces the same fields and iteration counts. */
void ext_tea_leaf_solve_(const int* chunk, const tea_solve_params* params,
                         tea_solve_result* result);

/* ---------------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference).  A U-Net of `levels` levels and
 * `base` channels at full resolution (doubling per level), bfloat16 weights and
 * activations with float32 accumulation, predicts the timestep increment
 * du = u(n+1) - u0 from u0 = density*energy, density, Kx, Ky (and Kz) -- through the plain
 * start's residual r0 = u0 - A u0, which scales input and output.  The 2D library's
 * network is made of 3x3 convolutions and 2x2 average pooling over [ny][nx] images, the 3D
 * library's of 3x3x3 convolutions and 2x2x2 pooling over [nz][ny][nx] volumes, with 5
 * input features instead of 4 (log10(1 + Kz) added).  A chunk with a network
 * attached starts each ext_tea_leaf_solve_ from u0 + du, smoothed by 8 damped Jacobi
 * sweeps in FP64, when that start has the smaller FP64 residual (else from u0, as the
 * reference does) and converges to the same tolerance.  After three rejected guesses in a
 * row the chunk solves 4 timesteps without predicting, then tries again (8, 16, at most 32
 * timesteps after further rejections); an accepted guess ends the back-off.  All functions
 * return a TEA_* status.
 * --------------------------------------------------------------------------------- */

/* New network with seeded He-initialised weights on the current device: levels 2..5,
 * base 16, 24, 32 or 64.  Writes its id (1-based).  tea_ws_create_capped_ stops the
 * doubling of the channel count at max_channels (0: no limit; 4 levels of base 32 capped
 * at 64 give 32/64/64/64 channels, about half a million parameters). */
int tea_ws_create_(const int* levels, const int* base, const int* seed, int* net);
int tea_ws_create_capped_(const int* levels, const int* base, const int* max_channels, const int* seed, int* net);
int tea_ws_destroy_(const int* net);
/* Records a training pair from the chunk's last ext_tea_leaf_solve_ (its features and
 * (u - u0) / max|u0|), kept in device memory by the network. */
int tea_ws_record_(const int* net, const int* chunk);
int tea_ws_pairs_(const int* net, int* count);
/* Adam training: `steps` steps on `batch` random crop x crop windows (crop^3 in 3D) of
 * the recorded pairs (crop a multiple of 2^(levels-1)).  The loss is, per crop, the energy norm of the
 * smoothed guess's error relative to that of the plain start, e.A e / du.A du with
 * e = M^8 (du_pred - du), A the solver's operator on the crop and M the smoothing sweep.
 * Writes that loss averaged over the first and over the last 10 steps (below 1: the guess
 * beats u0 on average), and the device milliseconds per step. */
int tea_ws_train_(const int* net, const int* steps, const int* batch, const int* crop, const double* lr,
                  const int* seed, double* loss_first, double* loss_last, double* ms_per_step);
/* Attaches the network to a chunk (net 0 detaches) and clears its back-off; sides must
 * be multiples of 2^(levels-1) for the guess to be used. */
int tea_ws_attach_(const int* chunk, const int* net);
/* The network's du for the chunk's current step, into a host array [ny][nx] ([nz][ny][nx]
 * in 3D), and the device milliseconds of the prediction. */
int tea_ws_predict_(const int* net, const int* chunk, double* du, double* ms);
/* Test hooks: parameters in the order of the CPU oracle (per layer w[co][taps][cin], 9
 * taps in 2D and 27 in 3D, then b; head w, head b), the choice of convolution (0 tensor
 * cores, fed by TMA where the image width is a multiple of 128; 1 CUDA cores; 2 tensor cores
 * without TMA), and forward/backward on host images [n][D][H][W][F] (F = 4 input
 * features in 2D, where D must be 1, and 5 in 3D; target null: forward only; kxy null:
 * mean squared error, else the residual loss with face coefficients [n][D][H][W][K],
 * K = 2 in 2D and 3 in 3D).  tea_ws_eval_host_ is tea_ws_eval_volume_ with D = 1. */
int tea_ws_param_count_(const int* net, long long* count);
int tea_ws_get_params_(const int* net, float* params);
int tea_ws_set_params_(const int* net, const float* params);
int tea_ws_set_conv_(const int* net, const int* reference);
int tea_ws_eval_volume_(const int* net, const float* x, const float* target, const float* kxy, const int* n,
                        const int* D, const int* H, const int* W, float* y, double* loss, float* grads);
int tea_ws_eval_host_(const int* net, const float* x, const float* target, const float* kxy, const int* n,
                      const int* H, const int* W, float* y, double* loss, float* grads);

#ifdef __cplusplus
}
#endif

#endif /* TEA_B200_H */
