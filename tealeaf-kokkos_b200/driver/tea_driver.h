/*
 * tea_driver.h -- C API of libtea_driver.so, the host-side restatement of the
 * reference's Fortran driver (tealeaf_2d|3d: tea_leaf.f90, start.f90, diffuse.f90,
 * timestep.f90, tea_solve.f90, field_summary.f90, read_input.f90, parse.f90).
 *
 * The driver runs a tea.in deck against any library that exports the reference's
 * ext_* C ABI (include/tea_ext_2d.h or tea_ext_3d.h), loaded with dlopen: the CUDA
 * library libtea{2,3}d_b200.so is the product backend.  No Fortran compiler exists
 * in this image, so this C++ restatement stands in for the Fortran caller.
 */
#ifndef TEA_DRIVER_H
#define TEA_DRIVER_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int dim;                 /* 2 or 3 */
    const char* backend;     /* path of the ext_* library */
    int use_fused_solve;     /* call ext_tea_leaf_solve_ instead of the per-call sequence */
    int summary_every_step;  /* call ext_field_summary_kernel_ after every step */
    int end_step_override;   /* > 0: stop after this many steps */
    int quiet;               /* 1: no tea.out lines on stdout */
    const char* out_path;    /* write the tea.out log here (NULL: none) */
    double eps_override;     /* > 0: replace tl_eps */
    double eps_rel_override; /* > 0: replace tl_eps_rel */
    int keep_chunk;          /* 1: skip ext_finalise_ so the caller can inspect the fields */
    int precision;           /* > 0: TEA_PRECISION_* for the whole-solve path (deck: tl_precision) */
    int ws_net;              /* a learned warm-start network id (tea_ws_create_), or 0 */
    int ws_mode;             /* with ws_net: 1 record a training pair after every solve,
                                2 warm-start every solve from the network */
    int reserved[4];
} tea_run_options;

typedef struct {
    int step;
    int iterations;          /* "Iteration count" printed by tea_leaf (n-1) */
    int status;
    int cheby_steps;
    double time;
    double dt;
    double error;
    double exact_error;
    double eps_used;
    double solve_seconds;    /* wall time of tea_leaf() for this step */
    double vol, mass, ie, temp; /* field summary after the step (0 unless computed) */
    int has_summary;
    int switch_step;
    int est_itc;
    int warm_start_used;     /* 1 when the solve started from the network's guess */
    double wall_end;         /* seconds since the start of the timestep loop, at the step's end */
    long long h2d_bytes;     /* backend host->device bytes so far (0 if not reported) */
    long long d2h_bytes;     /* backend device->host bytes so far */
    int corrections;         /* FP32-refined solves: outer corrections */
    int inner_solver;        /* FP32-refined solves: inner solver of the last correction
                                (0 CG, 1 Chebyshev, 2 PPCG) */
    double warm_r0_plain;    /* with a network attached: sum r^2 of the plain start u0 ... */
    double warm_r0_guess;    /* ... and of the network's guess (0 when none was made) */
} tea_step_record;

typedef struct {
    int steps;
    int test_problem;
    int kat_available;
    int kat_passed;
    double qa_diff;          /* percent difference to the known answer */
    double kat_expected;
    double vol, mass, ie, temp;  /* final field summary */
    double wall_seconds;     /* whole run (set-up excluded) */
    double solve_seconds;    /* sum of tea_leaf() wall times */
    long total_iterations;
    int x_cells, y_cells, z_cells;
    int solver;              /* TEA_SOLVER_* */
} tea_run_summary;

/* Run a deck (the text of a tea.in file).  `steps` may be NULL; at most `max_steps`
 * records are written.  Returns 0 on success, non-zero on a driver or backend error
 * (message in tea_driver_last_error()). */
int tea_run_deck(const char* deck_text, const tea_run_options* options,
                 tea_run_summary* summary, tea_step_record* steps, int max_steps);

/* A run split into slabs over `size` ranks -- the reference's MPI layer (tea_decompose,
 * tea_exchange, tea_allsum of tealeaf_2d/tea.f90, tealeaf_3d/tea.f90) with the transport
 * supplied by the caller (e.g. torch.distributed over NCCL or gloo).  Rank r owns the
 * r-th slab of the slowest axis (y in 2D, z in 3D; the remainder cells go to the first
 * ranks, as in tea_decompose).  allreduce_sum sums n doubles over all ranks in place;
 * sendrecv sends `send` to rank `to` and receives into `recv` from rank `from`, both
 * completing before it returns.  Faces are exchanged with the backend's tea_pack_face_
 * when it exports one (else ext_pack_message_, whose 2D bottom/top faces miss two inner
 * columns, as the reference's do).  The per-call path only (use_fused_solve must be 0). */
typedef struct {
    int rank, size;
    void (*allreduce_sum)(double* values, int n, void* ctx);
    void (*sendrecv)(const double* send, int nsend, int to, double* recv, int nrecv, int from, void* ctx);
    void* ctx;
} tea_comm;

int tea_run_deck_comm(const char* deck_text, const tea_run_options* options, const tea_comm* comm,
                      tea_run_summary* summary, tea_step_record* steps, int max_steps);

const char* tea_driver_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* TEA_DRIVER_H */
